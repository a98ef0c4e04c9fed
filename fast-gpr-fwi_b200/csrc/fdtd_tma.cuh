// Row-streaming time-step kernels: rows of state, coefficients and history
// are moved into a shared-memory ring by cp.async.bulk (TMA bulk copies)
// issued by a producer warp, completing on mbarriers; the consumer warps of
// the CTA compute one row of a tile per iteration from shared memory and store
// the new state straight to global memory.
//
// Tile = (shot group of G shots, row chunk [i0, i1), column band [b0, b0+W)),
// W = (consumer warps) * 32 * V.  Each ring stage holds, for one row r, the
// coefficient rows uE0 uE1 uH1 and, per shot, the old Ez, Hx, Hy rows (and in
// the adjoint the two stored forward Ez rows), each with 4 halo columns on
// either side.  The per-cell arithmetic is the same device code as the
// register-march kernels (fdtd_device.cuh): results are bit-identical.
//
// Forward, per row i:  H of row i (Hx written back into the stage in place),
// consumer barrier, E of row i reading Hx_new[j-1] from the stage.
// Adjoint, per row i:  E of row i+1 (written back into the stage in place,
// plus the column just past the band, recomputed), consumer barrier, H of
// row i and imaging from the stage.
#pragma once

#include "fdtd_device.cuh"

namespace fg {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bulk global -> shared copy completing on `bar` (no multicast).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void consumer_sync(int nthreads) {
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

// Error codes written to GridDev::err by bounded waits.
constexpr int ERR_WAIT_FULL = 201;
constexpr int ERR_WAIT_EMPTY = 202;
constexpr unsigned long long WAIT_LIMIT_NS = 2000000000ull;  // 2 s: a row takes microseconds

// Wait for `parity` on `bar`, for at most WAIT_LIMIT_NS; on timeout record
// `code`, raise the CTA's abort flag and return false.  Once the flag is up
// every later wait returns false at once, so all threads drain to the end of
// the kernel through the same barriers (no thread can be left waiting).
__device__ __forceinline__ bool wait_bounded(const GridDev& g, uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                             int code) {
    if (*abort_flag) return false;
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    while (!mbar_try_wait(bar, parity)) {
        if (*abort_flag) return false;
        if (globaltimer() - t0 > WAIT_LIMIT_NS) {
            atomicCAS(g.err, 0, code);
            *abort_flag = 1;
            return false;
        }
        __nanosleep(32);
    }
    return true;
}

struct Ring {
    float* base;      // D stages of SROWS rows of RW floats
    uint64_t* full;   // D barriers, count 1 (+tx)
    uint64_t* empty;  // D barriers, count = consumer warps
    volatile int* abort_flag;
    int D, SROWS, RW;
    __device__ __forceinline__ float* row(int n, int k) const { return base + ((long long)(n % D) * SROWS + k) * RW; }
};

// Carve the dynamic shared memory: barriers first (8-byte aligned), then the
// ring at a 128-byte boundary.
__device__ __forceinline__ Ring carve_ring(unsigned char* smem, int D, int SROWS, int RW) {
    Ring R;
    R.full = reinterpret_cast<uint64_t*>(smem);
    R.empty = R.full + D;
    R.abort_flag = reinterpret_cast<volatile int*>(R.empty + D);
    R.base = reinterpret_cast<float*>(smem + 128 * ((2 * D * 8 + 16 + 127) / 128));
    R.D = D;
    R.SROWS = SROWS;
    R.RW = RW;
    return R;
}

__host__ __device__ inline size_t ring_smem_bytes(int D, int SROWS, int RW) {
    return 128 * ((2 * (size_t)D * 8 + 16 + 127) / 128) + (size_t)D * SROWS * RW * sizeof(float);
}

struct TileTma {
    int band, chunk, grp, i0, i1, b0, W, lo, hi, soff;
};

__device__ __forceinline__ TileTma tma_tile(const GridDev& g, int W) {
    TileTma t;
    const int tile = blockIdx.x;
    t.band = tile % g.nb;
    const int rest = tile / g.nb;
    t.chunk = rest % g.nc;
    t.grp = rest / g.nc;
    t.i0 = g.chunk_row[t.chunk];
    t.i1 = g.chunk_row[t.chunk + 1];
    t.W = W;
    t.b0 = t.band * W;
    t.lo = max(t.b0 - 4, 0);
    t.hi = min(t.b0 + W + 4, g.P);
    t.soff = t.lo - (t.b0 - 4);
    return t;
}

// Producer: stream rows r_first..r_last of the tile into the ring.
// Stage rows: 0 uE0, 1 uE1, 2 uH1, then per shot q: 3+3q Ez, 4+3q Hx, 5+3q Hy,
// and for the adjoint 3+3G+2q Ez_fwd[it], 4+3G+2q Ez_fwd[it-1].
template <int G, bool ADJ>
__device__ void tma_producer(const GridDev& g, const Ring& R, const TileTma& T, int r_first, int r_last, int rp,
                             int it) {
    const int s0 = T.grp * G;
    const uint32_t seg = (uint32_t)(T.hi - T.lo) * 4u;
    const int hw_hi = min(T.b0 + T.W, g.Ph);
    const uint32_t hseg = (uint32_t)max(hw_hi - T.b0, 0) * 4u;
    int issued = 0;
    for (int r = r_first; r <= r_last; ++r) {
        const int n = r - r_first;
        if (n >= R.D) {
            if (!wait_bounded(g, &R.empty[n % R.D], ((n / R.D) - 1) & 1, R.abort_flag, ERR_WAIT_EMPTY)) break;
        }
        fence_proxy_async();
        int rows = 3;
        for (int q = 0; q < G; ++q) rows += (s0 + q < g.S) ? 3 : 0;
        const bool hrow = ADJ && r >= T.i0 && r < T.i1 && r < g.nx;
        uint32_t bytes = seg * rows;
        if (hrow)
            for (int q = 0; q < G; ++q)
                if (s0 + q < g.S) bytes += 2 * hseg;
        uint64_t* bar = &R.full[n % R.D];
        mbar_expect_tx(bar, bytes);
        const long long ro = (long long)r * g.P + T.lo;
        bulk_g2s(R.row(n, 0) + T.soff, g.ca + ro, seg, bar);
        bulk_g2s(R.row(n, 1) + T.soff, g.cb + ro, seg, bar);
        bulk_g2s(R.row(n, 2) + T.soff, g.ch + ro, seg, bar);
        for (int q = 0; q < G; ++q) {
            const int s = s0 + q;
            if (s >= g.S) continue;
            const long long so = (long long)s * g.plane + ro;
            bulk_g2s(R.row(n, 3 + 3 * q) + T.soff, g.ez[rp] + so, seg, bar);
            bulk_g2s(R.row(n, 4 + 3 * q) + T.soff, g.hx[rp] + so, seg, bar);
            bulk_g2s(R.row(n, 5 + 3 * q) + T.soff, g.hy[rp] + so, seg, bar);
            if (hrow) {
                const long long ho = (((long long)it * g.S + s) * g.nx + r) * g.Ph + T.b0;
                const long long hs = (long long)g.S * g.nx * g.Ph;
                bulk_g2s(R.row(n, 3 + 3 * G + 2 * q) + 4, g.hist + ho, hseg, bar);
                bulk_g2s(R.row(n, 4 + 3 * G + 2 * q) + 4, g.hist + ho - hs, hseg, bar);
            }
        }
        ++issued;
    }
    if (*R.abort_flag) {
        // drain: let every copy already issued land before the CTA retires
        for (int n = 0; n < issued; ++n) {
            const uint64_t t0 = globaltimer();
            while (!mbar_try_wait(&R.full[n % R.D], (n / R.D) & 1) && globaltimer() - t0 < WAIT_LIMIT_NS) {
            }
        }
    }
}

template <int V>
__device__ __forceinline__ void lds(float (&x)[V], const float* p) {
    if constexpr (V == 4) {
        const float4 q = *reinterpret_cast<const float4*>(p);
        x[0] = q.x; x[1] = q.y; x[2] = q.z; x[3] = q.w;
    } else if constexpr (V == 2) {
        const float2 q = *reinterpret_cast<const float2*>(p);
        x[0] = q.x; x[1] = q.y;
    } else {
        x[0] = *p;
    }
}

// ---------------------------------------------------------------------------
// Forward step
// ---------------------------------------------------------------------------
template <int V, int G>
__global__ void k_forward_tma(const GridDev g, const int t, const int D) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int nw = (blockDim.x >> 5) - 1;      // consumer warps
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int W = nw * 32 * V, RW = W + 8;
    const int SROWS = 3 + 3 * G;
    const Ring R = carve_ring(smem, D, SROWS, RW);
    const TileTma T = tma_tile(g, W);
    if (T.grp * G >= g.S) return;
    const int rp = t & 1, wp = rp ^ 1;
    const int r_first = T.i0 >= 1 ? T.i0 - 1 : T.i0, r_last = T.i1;
    if (threadIdx.x == 0) {
        for (int k = 0; k < D; ++k) {
            mbar_init(&R.full[k], 1);
            mbar_init(&R.empty[k], nw);
        }
        *R.abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();
    if (warp == nw) {
        if (lane == 0) tma_producer<G, false>(g, R, T, r_first, r_last, rp, 0);
        return;
    }

    const int nx = g.nx, ny = g.ny, P = g.P;
    const int tid = threadIdx.x;           // consumer thread index
    const int c0 = 4 + tid * V;            // smem column of this thread's first cell
    const int jb = T.b0 + tid * V;         // its global column
    const int s0 = T.grp * G;
    const int ncons = nw * 32;
    const long long hstride = (long long)nx * g.Ph;

    float hyu[G][V];
#pragma unroll
    for (int q = 0; q < G; ++q)
#pragma unroll
        for (int v = 0; v < V; ++v) hyu[q][v] = 0.f;

    int n = 0;  // ring index of the current row
    if (T.i0 >= 1) {
        wait_bounded(g, &R.full[0], 0, R.abort_flag, ERR_WAIT_FULL);
        wait_bounded(g, &R.full[1 % D], (1 / D) & 1, R.abort_flag, ERR_WAIT_FULL);
        const int ih = T.i0 - 1;
        const float* chr = R.row(0, 2);
#pragma unroll
        for (int q = 0; q < G; ++q) {
            if (s0 + q >= g.S) continue;
            const PsiShot rd = psi_shot(g, rp, s0 + q);
            const float* ezh = R.row(0, 3 + 3 * q);
            const float* hyh = R.row(0, 5 + 3 * q);
            const float* ez0 = R.row(1, 3 + 3 * q);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int j = jb + v;
                float hx_unused = 0.f, hy = hyh[c0 + v];
                if (j < ny)
                    h_update<false, false, true>(g, ih, j, hx_unused, hy, 0.f, __fsub_rn(ez0[c0 + v], ezh[c0 + v]),
                                                 chr[c0 + v], rd, rd);
                hyu[q][v] = hy;
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&R.empty[0]);
        n = 1;
    } else {
        wait_bounded(g, &R.full[0], 0, R.abort_flag, ERR_WAIT_FULL);
    }

    int sc = g.src_off[blockIdx.x];
    const int se = g.src_off[blockIdx.x + 1];
    int rc = g.rx_off[blockIdx.x];
    const int re = g.rx_off[blockIdx.x + 1];

    for (int i = T.i0; i < T.i1; ++i, ++n) {
        wait_bounded(g, &R.full[(n + 1) % D], ((n + 1) / D) & 1, R.abort_flag, ERR_WAIT_FULL);
        const float* car = R.row(n, 0);
        const float* cbr = R.row(n, 1);
        const float* chr = R.row(n, 2);
        float hyn[G][V];
        // --- H of row i
#pragma unroll
        for (int q = 0; q < G; ++q) {
            if (s0 + q >= g.S) continue;
            const int s = s0 + q;
            const PsiShot rd = psi_shot(g, rp, s), wr = psi_shot(g, wp, s);
            const float* ezc = R.row(n, 3 + 3 * q);
            float* hxr = R.row(n, 4 + 3 * q);
            const float* hyr = R.row(n, 5 + 3 * q);
            const float* ezn = R.row(n + 1, 3 + 3 * q);
            float ez[V + 1], en[V], hx[V], hy[V], ch[V];
            lds<V>(en, ezn + c0);
            lds<V>(hx, hxr + c0);
            lds<V>(hy, hyr + c0);
            lds<V>(ch, chr + c0);
#pragma unroll
            for (int v = 0; v < V; ++v) ez[v] = ezc[c0 + v];
            ez[V] = ezc[c0 + V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int j = jb + v;
                if (j < ny)
                    h_update<true, true, true>(g, i, j, hx[v], hy[v], __fsub_rn(ez[v + 1], ez[v]),
                                               __fsub_rn(en[v], ez[v]), ch[v], rd, wr);
                hyn[q][v] = hy[v];
            }
            // Hx of the column left of the band: from the old state, read-only auxiliaries
            if (tid == 0 && T.b0 > 0) {
                float hxl = hxr[3], hy_unused = 0.f;
                h_update<false, true, false>(g, i, T.b0 - 1, hxl, hy_unused, __fsub_rn(ez[0], ezc[3]), 0.f, chr[3],
                                             rd, rd);
                hxr[3] = hxl;
            }
#pragma unroll
            for (int v = 0; v < V; ++v) hxr[c0 + v] = hx[v];
        }
        consumer_sync(ncons);
        // --- E of row i
#pragma unroll
        for (int q = 0; q < G; ++q) {
            if (s0 + q >= g.S) continue;
            const int s = s0 + q;
            const PsiShot rd = psi_shot(g, rp, s), wr = psi_shot(g, wp, s);
            const float* ezc = R.row(n, 3 + 3 * q);
            const float* hxr = R.row(n, 4 + 3 * q);
            float ez[V], hx[V], ca[V], cb[V];
            lds<V>(ez, ezc + c0);
            lds<V>(hx, hxr + c0);
            lds<V>(ca, car + c0);
            lds<V>(cb, cbr + c0);
            const float hxl0 = hxr[c0 - 1];
            float ezw[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int j = jb + v;
                ezw[v] = ez[v];
                if (j < ny) {
                    const float hxl = (v > 0) ? hx[(v + V - 1) % V] : hxl0;
                    ezw[v] = e_update<true>(g, i, j, ez[v], __fsub_rn(hyn[q][v], hyu[q][v]), __fsub_rn(hx[v], hxl),
                                            ca[v], cb[v], rd, wr);
                }
            }
            while (sc < se) {
                const Ev e = __ldg(g.src_ev + sc);
                if (e.x != i || e.y != q) break;
#pragma unroll
                for (int v = 0; v < V; ++v)
                    if (jb + v == e.z) {
                        const float cd = ldc1(g, g.cd + (long long)i * P + e.z);
                        ezw[v] = __fmaf_rn(-cd, ldc1(g, g.srcw + (long long)e.w * g.nt + t), ezw[v]);
                    }
                ++sc;
            }
            if (jb < P) {
                const long long ro = (long long)s * g.plane + (long long)i * P + jb;
                st_state<V>(g, g.ez[wp] + ro, ezw);
                st_state<V>(g, g.hx[wp] + ro, hx);
                st_state<V>(g, g.hy[wp] + ro, hyn[q]);
            }
            if (g.hist && jb < g.Ph) {
                float* hrow = g.hist + ((long long)t * g.S + s) * hstride + (long long)i * g.Ph + jb;
                st_state<V>(g, hrow, ezw);
            }
            while (rc < re) {
                const Ev e = __ldg(g.rx_ev + rc);
                if (e.x != i || e.y != q) break;
                if (t + 1 < g.nt) {
#pragma unroll
                    for (int v = 0; v < V; ++v)
                        if (jb + v == e.z) g.traces[((long long)s * g.nt + t + 1) * g.nrx + e.w] = ezw[v];
                }
                ++rc;
            }
#pragma unroll
            for (int v = 0; v < V; ++v) hyu[q][v] = hyn[q][v];
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&R.empty[n % D]);
    }
}

// ---------------------------------------------------------------------------
// Reference-mode adjoint step
// ---------------------------------------------------------------------------

// E_new of one row of one shot for this thread's columns, written back into
// the stage's Ez row.  hyp: the stage row holding Hy_old of row r-1 (NULL when
// r == 0).  STORE selects whether the CPML auxiliaries are written (owned
// rows).  Events consumed from *cur.
template <int V>
__device__ __forceinline__ void adj_e_row(const GridDev& g, int r, int q, int s, int jb, int c0, float* ezr,
                                          const float* hxr, const float* hyr, const float* hyp, const float* car,
                                          const float* cbr, const PsiShot& rd, const PsiShot& wr, bool store,
                                          const float* resid_t, int& cur, int end) {
    float ez[V], hx[V], hy[V], hu[V], ca[V], cb[V];
    lds<V>(ez, ezr + c0);
    lds<V>(hx, hxr + c0);
    lds<V>(hy, hyr + c0);
    lds<V>(ca, car + c0);
    lds<V>(cb, cbr + c0);
    if (hyp) {
        lds<V>(hu, hyp + c0);
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v) hu[v] = 0.f;
    }
    const float hxl0 = hxr[c0 - 1];
    while (cur < end) {
        const Ev e = __ldg(g.inj_ev + cur);
        if (e.x != r || e.y != q) break;
#pragma unroll
        for (int v = 0; v < V; ++v)
            if (jb + v == e.z) ez[v] = __fsub_rn(ez[v], resid_t[(long long)s * g.nt * g.nrx + e.w]);
        ++cur;
    }
    float out[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const int j = jb + v;
        out[v] = ez[v];
        if (j < g.ny) {
            const float hxl = (v > 0) ? hx[(v + V - 1) % V] : hxl0;
            out[v] = store ? e_update<true>(g, r, j, ez[v], __fsub_rn(hy[v], hu[v]), __fsub_rn(hx[v], hxl), ca[v],
                                            cb[v], rd, wr)
                           : e_update<false>(g, r, j, ez[v], __fsub_rn(hy[v], hu[v]), __fsub_rn(hx[v], hxl), ca[v],
                                             cb[v], rd, rd);
        }
    }
#pragma unroll
    for (int v = 0; v < V; ++v) ezr[c0 + v] = out[v];
}

// E_new of the column just past the band (be), from the stage (old values),
// with the halo-column injections of row r.
__device__ __forceinline__ void adj_e_halo(const GridDev& g, int r, int q, int s, int be, int cbe, float* ezr,
                                           const float* hxr, const float* hyr, const float* hyp, const float* car,
                                           const float* cbr, const PsiShot& rd, const float* resid_t, int& cur,
                                           int end, bool active) {
    float ez = active ? ezr[cbe] : 0.f;
    while (cur < end) {
        const Ev e = __ldg(g.injh_ev + cur);
        if (e.x != r || e.y != q) break;
        if (active) ez = __fsub_rn(ez, resid_t[(long long)s * g.nt * g.nrx + e.w]);
        ++cur;
    }
    if (!active) return;
    if (be < g.ny) {
        const float hu = hyp ? hyp[cbe] : 0.f;
        ez = e_update<false>(g, r, be, ez, __fsub_rn(hyr[cbe], hu), __fsub_rn(hxr[cbe], hxr[cbe - 1]), car[cbe],
                             cbr[cbe], rd, rd);
    } else {
        ez = 0.f;
    }
    ezr[cbe] = ez;
}

template <int V, int G>
__global__ void k_adjoint_tma(const GridDev g, const int it, const int rp, const int D) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int nw = (blockDim.x >> 5) - 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int W = nw * 32 * V, RW = W + 8;
    const int SROWS = 3 + 5 * G;
    const Ring R = carve_ring(smem, D, SROWS, RW);
    const TileTma T = tma_tile(g, W);
    if (T.grp * G >= g.S) return;
    const int wp = rp ^ 1;
    const int r_first = T.i0 >= 1 ? T.i0 - 1 : T.i0;
    const int r_last = min(T.i1, g.nx - 1);   // row nx is the zero frame: never loaded
    if (threadIdx.x == 0) {
        for (int k = 0; k < D; ++k) {
            mbar_init(&R.full[k], 1);
            mbar_init(&R.empty[k], nw);
        }
        *R.abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();
    if (warp == nw) {
        if (lane == 0) tma_producer<G, true>(g, R, T, r_first, r_last, rp, it);
        return;
    }

    const int nx = g.nx, ny = g.ny, P = g.P;
    const int tid = threadIdx.x;
    const int c0 = 4 + tid * V;
    const int jb = T.b0 + tid * V;
    const int s0 = T.grp * G;
    const int ncons = nw * 32;
    const int be = T.b0 + W;
    const int cbe = 4 + W;
    const bool halo_thread = (tid == ncons - 1);
    const float* resid_t = g.resid + (long long)it * g.nrx;
    int ic = g.inj_off[blockIdx.x];
    const int ie = g.inj_off[blockIdx.x + 1];
    int hc = g.injh_off[blockIdx.x];
    const int he = g.injh_off[blockIdx.x + 1];
    double* gae = g.gacc + (long long)T.grp * 2 * ((long long)nx * ny);
    double* gas = gae + (long long)nx * ny;

    // Prologue: E_new of row i0.
    int n = 0;
    if (T.i0 >= 1) {
        wait_bounded(g, &R.full[0], 0, R.abort_flag, ERR_WAIT_FULL);
        wait_bounded(g, &R.full[1 % D], (1 / D) & 1, R.abort_flag, ERR_WAIT_FULL);
        n = 1;
    } else {
        wait_bounded(g, &R.full[0], 0, R.abort_flag, ERR_WAIT_FULL);
    }
#pragma unroll
    for (int q = 0; q < G; ++q) {
        const int s = s0 + q;
        if (s >= g.S) continue;
        const PsiShot rd = psi_shot(g, rp, s), wr = psi_shot(g, wp, s);
        const float* hyp = (T.i0 >= 1) ? R.row(0, 5 + 3 * q) : nullptr;
        adj_e_row<V>(g, T.i0, q, s, jb, c0, R.row(n, 3 + 3 * q), R.row(n, 4 + 3 * q), R.row(n, 5 + 3 * q), hyp,
                     R.row(n, 0), R.row(n, 1), rd, wr, true, resid_t, ic, ie);
        adj_e_halo(g, T.i0, q, s, be, cbe, R.row(n, 3 + 3 * q), R.row(n, 4 + 3 * q), R.row(n, 5 + 3 * q), hyp,
                   R.row(n, 0), R.row(n, 1), rd, resid_t, hc, he, halo_thread);
    }
    if (T.i0 >= 1) {
        __syncwarp();
        if (lane == 0) mbar_arrive(&R.empty[0]);
    }

    for (int i = T.i0; i < T.i1; ++i, ++n) {
        const int r = i + 1;
        const bool have_r = r < nx;
        if (have_r) wait_bounded(g, &R.full[(n + 1) % D], ((n + 1) / D) & 1, R.abort_flag, ERR_WAIT_FULL);
        // --- E of row r (row i1 is the next chunk's: computed, auxiliaries not stored)
        if (have_r) {
#pragma unroll
            for (int q = 0; q < G; ++q) {
                const int s = s0 + q;
                if (s >= g.S) continue;
                const PsiShot rd = psi_shot(g, rp, s), wr = psi_shot(g, wp, s);
                const float* hyp = R.row(n, 5 + 3 * q);
                adj_e_row<V>(g, r, q, s, jb, c0, R.row(n + 1, 3 + 3 * q), R.row(n + 1, 4 + 3 * q),
                             R.row(n + 1, 5 + 3 * q), hyp, R.row(n + 1, 0), R.row(n + 1, 1), rd, wr, r < T.i1,
                             resid_t, ic, ie);
                if (r < T.i1)
                    adj_e_halo(g, r, q, s, be, cbe, R.row(n + 1, 3 + 3 * q), R.row(n + 1, 4 + 3 * q),
                               R.row(n + 1, 5 + 3 * q), hyp, R.row(n + 1, 0), R.row(n + 1, 1), rd, resid_t, hc, he,
                               halo_thread);
            }
        }
        consumer_sync(ncons);
        // --- H of row i and imaging
        const float* chr = R.row(n, 2);
        float acc_e[V], acc_s[V];
#pragma unroll
        for (int v = 0; v < V; ++v) { acc_e[v] = 0.f; acc_s[v] = 0.f; }
#pragma unroll
        for (int q = 0; q < G; ++q) {
            const int s = s0 + q;
            if (s >= g.S) continue;
            const PsiShot rd = psi_shot(g, rp, s), wr = psi_shot(g, wp, s);
            const float* ezc = R.row(n, 3 + 3 * q);
            float ez[V + 1], en[V], hx[V], hy[V], ch[V], f1[V], f0[V];
#pragma unroll
            for (int v = 0; v <= V; ++v) ez[v] = ezc[c0 + v];
            if (have_r) {
                lds<V>(en, R.row(n + 1, 3 + 3 * q) + c0);
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) en[v] = 0.f;
            }
            lds<V>(hx, R.row(n, 4 + 3 * q) + c0);
            lds<V>(hy, R.row(n, 5 + 3 * q) + c0);
            lds<V>(ch, chr + c0);
            lds<V>(f1, R.row(n, 3 + 3 * G + 2 * q) + c0);
            lds<V>(f0, R.row(n, 4 + 3 * G + 2 * q) + c0);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int j = jb + v;
                if (j < ny) {
                    h_update<true, true, true>(g, i, j, hx[v], hy[v], __fsub_rn(ez[v + 1], ez[v]),
                                               __fsub_rn(en[v], ez[v]), ch[v], rd, wr);
                    acc_e[v] = __fadd_rn(acc_e[v], __fmul_rn(__fsub_rn(f1[v], f0[v]), ez[v]));
                    acc_s[v] = __fadd_rn(acc_s[v], __fmul_rn(__fmul_rn(f1[v], ez[v]), g.dt));
                }
            }
            if (jb < P) {
                const long long ro = (long long)s * g.plane + (long long)i * P + jb;
                float ezo[V];
#pragma unroll
                for (int v = 0; v < V; ++v) ezo[v] = ez[v];
                st_state<V>(g, g.ez[wp] + ro, ezo);
                st_state<V>(g, g.hx[wp] + ro, hx);
                st_state<V>(g, g.hy[wp] + ro, hy);
            }
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int j = jb + v;
            if (j < ny) {
                const long long o = (long long)i * ny + j;
                gae[o] += (double)acc_e[v];
                gas[o] += (double)acc_s[v];
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&R.empty[n % D]);
    }
}

}  // namespace fg
