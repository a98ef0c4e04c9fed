// Row-streaming time-step kernels: every operand of a row -- coefficient
// rows, the old Ez/Hx/Hy rows, the CPML auxiliaries of that row and, in the
// adjoint, the stored forward Ez rows -- is moved into a shared-memory ring by
// cp.async.bulk (TMA bulk copies) issued by a producer warp and completing on
// mbarriers.  The consumer warps compute one row of the tile per iteration
// entirely from shared memory and store the new state (and new CPML
// auxiliaries) straight to global memory, so no global load sits in the
// dependency chain of a row.
//
// Tile = (shot group of G shots, row chunk [i0, i1), column band [b0, b0+W)),
// W = (consumer warps) * 32 * V.  Stage slots (SW floats each):
//   0..4             uE0 uE1 uE4 uH1 uH4 of the row
//   5+6q .. 10+6q    shot q: Ez, Hx, Hy, x-slab E auxiliary row, x-slab H
//                    auxiliary row, y-slab block [E y0 | E ymax | H y0 | H ymax]
//   5+6G+2q, +1      adjoint only: forward Ez of steps it and it-1
// Field and coefficient slots hold columns b0-4 .. b0+W+3 (4 halo columns on
// each side).  The per-cell arithmetic is the same operation sequence as
// fdtd_device.cuh, so results are bit-identical to the register-march
// kernels and to the reference.
//
// Forward, per row i:  H of row i (Hx written back into the stage in place),
// consumer barrier, E of row i reading Hx_new[j-1] from the stage.
// Adjoint, per row i:  E of row i+1 (written back into the stage in place,
// plus the column just past the band, recomputed), consumer barrier, H of
// row i and imaging from the stage.
//
// Requires 2*th < nx (a row lies in at most one x-slab); the plan falls back
// to the register-march kernels otherwise.
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
    float* base;      // D stages of SROWS slots of SW floats
    uint64_t* full;   // D barriers, count 1 (+tx)
    uint64_t* empty;  // D barriers, count = consumer warps
    volatile int* abort_flag;
    float* pml;       // (8, th) CPML vectors
    int D, SROWS, SW;
    __device__ __forceinline__ float* row(int n, int k) const { return base + ((long long)(n % D) * SROWS + k) * SW; }
};

__host__ __device__ inline int ring_slot_width(int W, int TY) {
    const int rw = W + 8;
    const int yw = 4 * TY;
    return rw > yw ? rw : yw;
}
__host__ __device__ inline size_t ring_head_bytes(int D, int th) {
    return 128 * ((2 * (size_t)D * 8 + 16 + 8 * (size_t)th * 4 + 127) / 128);
}
__host__ __device__ inline size_t ring_smem_bytes(int D, int SROWS, int SW, int th) {
    return ring_head_bytes(D, th) + (size_t)D * SROWS * SW * sizeof(float);
}

// Carve the dynamic shared memory: barriers, abort flag and CPML vectors,
// then the ring at a 128-byte boundary.
__device__ __forceinline__ Ring carve_ring(unsigned char* smem, int D, int SROWS, int SW, int th) {
    Ring R;
    R.full = reinterpret_cast<uint64_t*>(smem);
    R.empty = R.full + D;
    R.abort_flag = reinterpret_cast<volatile int*>(R.empty + D);
    R.pml = reinterpret_cast<float*>(smem + 2 * D * 8 + 16);
    R.base = reinterpret_cast<float*>(smem + ring_head_bytes(D, th));
    R.D = D;
    R.SROWS = SROWS;
    R.SW = SW;
    return R;
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

// x-slab membership of row r for the E (1..th, nx-th..nx-1) and H
// (0..th-1, nx-th..nx-1) auxiliaries: returns the auxiliary row index
// slab*th + k, or -1.
__device__ __forceinline__ int ex_row(const GridDev& g, int r) {
    if (g.th <= 0 || r >= g.nx) return -1;
    if (r >= 1 && r <= g.th) return g.th - r;
    if (r >= g.nx - g.th) return g.th + (r - (g.nx - g.th));
    return -1;
}
__device__ __forceinline__ int hx_row(const GridDev& g, int r) {
    if (g.th <= 0 || r >= g.nx) return -1;
    if (r <= g.th - 1) return g.th - 1 - r;
    if (r >= g.nx - g.th) return g.th + (r - (g.nx - g.th));
    return -1;
}

// Producer: stream rows r_first..r_last of the tile into the ring.
template <int G, bool ADJ>
__device__ void tma_producer(const GridDev& g, const Ring& R, const TileTma& T, int r_first, int r_last, int rp,
                             int it) {
    const int s0 = T.grp * G;
    const uint32_t seg = (uint32_t)(T.hi - T.lo) * 4u;
    const int hw_hi = min(T.b0 + T.W, g.Ph);
    const uint32_t hseg = (uint32_t)max(hw_hi - T.b0, 0) * 4u;
    const uint32_t yseg = (uint32_t)g.TY * 4u;
    int issued = 0;
    for (int r = r_first; r <= r_last; ++r) {
        const int n = r - r_first;
        if (n >= R.D) {
            if (!wait_bounded(g, &R.empty[n % R.D], ((n / R.D) - 1) & 1, R.abort_flag, ERR_WAIT_EMPTY)) break;
        }
        fence_proxy_async();
        const int ek = ex_row(g, r), hk = hx_row(g, r);
        const bool ypsi = g.th > 0 && r < g.nx;
        const bool hrow = ADJ && r >= T.i0 && r < T.i1 && r < g.nx;
        int nsh = 0;
        for (int q = 0; q < G; ++q) nsh += (s0 + q < g.S) ? 1 : 0;
        uint32_t per_shot = 3 * seg + (ek >= 0 ? seg : 0) + (hk >= 0 ? seg : 0) + (ypsi ? 4 * yseg : 0) +
                            (hrow ? 2 * hseg : 0);
        uint64_t* bar = &R.full[n % R.D];
        mbar_expect_tx(bar, 5 * seg + nsh * per_shot);
        const long long ro = (long long)r * g.P + T.lo;
        bulk_g2s(R.row(n, 0) + T.soff, g.ca + ro, seg, bar);
        bulk_g2s(R.row(n, 1) + T.soff, g.cb + ro, seg, bar);
        bulk_g2s(R.row(n, 2) + T.soff, g.cd + ro, seg, bar);
        bulk_g2s(R.row(n, 3) + T.soff, g.ch + ro, seg, bar);
        bulk_g2s(R.row(n, 4) + T.soff, g.ci + ro, seg, bar);
        for (int q = 0; q < G; ++q) {
            const int s = s0 + q;
            if (s >= g.S) continue;
            const int b = 5 + 6 * q;
            const long long so = (long long)s * g.plane + ro;
            bulk_g2s(R.row(n, b + 0) + T.soff, g.ez[rp] + so, seg, bar);
            bulk_g2s(R.row(n, b + 1) + T.soff, g.hx[rp] + so, seg, bar);
            bulk_g2s(R.row(n, b + 2) + T.soff, g.hy[rp] + so, seg, bar);
            if (ek >= 0)
                bulk_g2s(R.row(n, b + 3) + T.soff, g.pex[rp] + (long long)s * g.pxs + (long long)ek * g.P + T.lo, seg,
                         bar);
            if (hk >= 0)
                bulk_g2s(R.row(n, b + 4) + T.soff, g.phx[rp] + (long long)s * g.pxs + (long long)hk * g.P + T.lo, seg,
                         bar);
            if (ypsi) {
                float* yb = R.row(n, b + 5);
                const long long y0 = (long long)s * g.pys + (long long)r * g.TY;
                const long long y1 = (long long)s * g.pys + (long long)(g.nx + 1 + r) * g.TY;
                bulk_g2s(yb, g.pey[rp] + y0, yseg, bar);
                bulk_g2s(yb + g.TY, g.pey[rp] + y1, yseg, bar);
                bulk_g2s(yb + 2 * g.TY, g.phy[rp] + y0, yseg, bar);
                bulk_g2s(yb + 3 * g.TY, g.phy[rp] + y1, yseg, bar);
            }
            if (hrow) {
                const long long ho = (((long long)it * g.S + s) * g.nx + r) * g.Ph + T.b0;
                const long long hs = (long long)g.S * g.nx * g.Ph;
                bulk_g2s(R.row(n, 5 + 6 * G + 2 * q) + 4, g.hist + ho, hseg, bar);
                bulk_g2s(R.row(n, 6 + 6 * G + 2 * q) + 4, g.hist + ho - hs, hseg, bar);
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

// One HORIPML correction with the coefficient vectors in shared memory.
template <bool PLUS>
__device__ __forceinline__ float cpml_s(float f, float deriv, float u4, float& psi, const float* R, int th, int k) {
    const float ra1 = __fsub_rn(R[k], 1.0f);
    const float t = madd2(ra1, deriv, R[th + k], psi);
    const float out = __fmaf_rn(PLUS ? u4 : -u4, t, f);
    psi = msub2(R[2 * th + k], psi, R[3 * th + k], deriv);
    return out;
}

// x-slab auxiliary row index of row r, or -1 (see ex_row / hx_row): rows
// 0..th-1 of the auxiliary array are slab x0 (k = index), rows th..2th-1 slab
// xmax (k = index - th).

// E update of cell (i, j), operands in shared memory; same operation
// sequence as e_update.  ek: x-slab E auxiliary row of row i (or -1);
// y0 / ym: this column lies in the y0 / ymax E slab.  New auxiliaries of
// shot s go to parity wp.
template <bool STORE>
__device__ __forceinline__ float e_cell_s(const GridDev& g, const float* pml, int i, int j, int c, float ez, float dhy,
                                          float dhx, float ca, float cb, const float* cdr, int ek, bool y0, bool ym,
                                          const float* pE, const float* yp, int s, int wp) {
    if (i >= 1 && j >= 1) ez = __fmaf_rn(-cb, dhx, madd2(ca, ez, cb, dhy));
    if (ek >= 0 || y0 || ym) {
        const int th = g.th;
        const float cd = cdr[c];
        if (ek >= 0 && ek < th) {
            float psi = pE[c];
            ez = cpml_s<true>(ez, __fdiv_rn(dhy, g.d), cd, psi, pml, th, ek);
            if (STORE) __stcg(g.pex[wp] + (long long)s * g.pxs + (long long)ek * g.P + j, psi);
        }
        if (y0) {
            const int k = th - j;
            float psi = yp[k];
            ez = cpml_s<false>(ez, __fdiv_rn(dhx, g.d), cd, psi, pml, th, k);
            if (STORE) __stcg(g.pey[wp] + (long long)s * g.pys + (long long)i * g.TY + k, psi);
        }
        if (ek >= th) {
            float psi = pE[c];
            ez = cpml_s<true>(ez, __fdiv_rn(dhy, g.d), cd, psi, pml, th, ek - th);
            if (STORE) __stcg(g.pex[wp] + (long long)s * g.pxs + (long long)ek * g.P + j, psi);
        }
        if (ym) {
            const int k = j - (g.ny - th);
            float psi = yp[g.TY + k];
            ez = cpml_s<false>(ez, __fdiv_rn(dhx, g.d), cd, psi, pml, th, k);
            if (STORE) __stcg(g.pey[wp] + (long long)s * g.pys + (long long)(g.nx + 1 + i) * g.TY + k, psi);
        }
    }
    return ez;
}

// H update of cell (i, j), operands in shared memory; same operation
// sequence as h_update.  hk: x-slab H auxiliary row of row i (or -1);
// y0 / ym: this column lies in the y0 / ymax H slab.
template <bool STORE, bool DO_HX, bool DO_HY>
__device__ __forceinline__ void h_cell_s(const GridDev& g, const float* pml, int i, int j, int c, float& hx, float& hy,
                                         float dzx, float dzy, float ch, const float* cir, int hk, bool y0, bool ym,
                                         const float* pH, const float* yp, int s, int wp) {
    if (DO_HX && i >= 1) hx = msub2(1.0f, hx, ch, dzx);
    if (DO_HY && j >= 1) hy = madd2(1.0f, hy, ch, dzy);
    const bool xs = DO_HY && hk >= 0;
    const bool ys0 = DO_HX && y0, ysm = DO_HX && ym;
    if (xs || ys0 || ysm) {
        const int th = g.th;
        const float* HR = pml + 4 * th;
        const float ci = cir[c];
        if (xs && hk < th) {
            float psi = pH[c];
            hy = cpml_s<true>(hy, __fdiv_rn(dzy, g.d), ci, psi, HR, th, hk);
            if (STORE) __stcg(g.phx[wp] + (long long)s * g.pxs + (long long)hk * g.P + j, psi);
        }
        if (ys0) {
            const int k = th - 1 - j;
            float psi = yp[2 * g.TY + k];
            hx = cpml_s<false>(hx, __fdiv_rn(dzx, g.d), ci, psi, HR, th, k);
            if (STORE) __stcg(g.phy[wp] + (long long)s * g.pys + (long long)i * g.TY + k, psi);
        }
        if (xs && hk >= th) {
            float psi = pH[c];
            hy = cpml_s<true>(hy, __fdiv_rn(dzy, g.d), ci, psi, HR, th, hk - th);
            if (STORE) __stcg(g.phx[wp] + (long long)s * g.pxs + (long long)hk * g.P + j, psi);
        }
        if (ysm) {
            const int k = j - (g.ny - th);
            float psi = yp[3 * g.TY + k];
            hx = cpml_s<false>(hx, __fdiv_rn(dzx, g.d), ci, psi, HR, th, k);
            if (STORE) __stcg(g.phy[wp] + (long long)s * g.pys + (long long)(g.nx + 1 + i) * g.TY + k, psi);
        }
    }
}

// y-slab membership bits of a thread's V columns (bit v for column jb+v).
struct YBits {
    unsigned valid, e0, em, h0, hm;
};
template <int V>
__device__ __forceinline__ YBits ybits(const GridDev& g, int jb) {
    YBits b{0u, 0u, 0u, 0u, 0u};
    const int th = g.th, ny = g.ny;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const int j = jb + v;
        if (j < ny) b.valid |= 1u << v;
        if (th > 0 && j < ny) {
            if (j >= 1 && j <= th) b.e0 |= 1u << v;
            if (j >= ny - th) b.em |= 1u << v;
            if (j <= th - 1) b.h0 |= 1u << v;
            if (j >= ny - th) b.hm |= 1u << v;
        }
    }
    return b;
}

// Shared set-up of both kernels: barriers, CPML vectors.
__device__ __forceinline__ void ring_init(const GridDev& g, const Ring& R, int nw) {
    for (int k = threadIdx.x; k < 8 * g.th; k += blockDim.x) R.pml[k] = g.pml[k];
    if (threadIdx.x == 0) {
        for (int k = 0; k < R.D; ++k) {
            mbar_init(&R.full[k], 1);
            mbar_init(&R.empty[k], nw);
        }
        *R.abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Forward step
// ---------------------------------------------------------------------------
template <int V, int G>
__global__ void __launch_bounds__(512) k_forward_tma(const GridDev g, const int t, const int D) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int nw = (blockDim.x >> 5) - 1;      // consumer warps
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int W = nw * 32 * V;
    const int SROWS = 5 + 6 * G;
    const int SW = ring_slot_width(W, g.TY);
    const Ring R = carve_ring(smem, D, SROWS, SW, g.th);
    const TileTma T = tma_tile(g, W);
    if (T.grp * G >= g.S) return;
    const int rp = t & 1, wp = rp ^ 1;
    const int r_first = T.i0 >= 1 ? T.i0 - 1 : T.i0, r_last = T.i1;
    ring_init(g, R, nw);
    if (warp == nw) {
        if (lane == 0) tma_producer<G, false>(g, R, T, r_first, r_last, rp, 0);
        return;
    }

    const int P = g.P;
    const int tid = threadIdx.x;           // consumer thread index
    const int c0 = 4 + tid * V;            // smem column of this thread's first cell
    const int jb = T.b0 + tid * V;         // its global column
    const int s0 = T.grp * G;
    const int ncons = nw * 32;
    const int stage_floats = SROWS * SW;
    const YBits yb = ybits<V>(g, jb);
    const bool act = jb < P;
    const bool hist_act = g.hist != nullptr && jb < g.Ph;
    const float* pml = R.pml;

    float hyu[G][V];
#pragma unroll
    for (int q = 0; q < G; ++q)
#pragma unroll
        for (int v = 0; v < V; ++v) hyu[q][v] = 0.f;

    int slot = 0;  // ring slot of the current row
    if (T.i0 >= 1) {
        wait_bounded(g, &R.full[0], 0, R.abort_flag, ERR_WAIT_FULL);
        wait_bounded(g, &R.full[1 % D], (1 / D) & 1, R.abort_flag, ERR_WAIT_FULL);
        const int ih = T.i0 - 1;
        const float* st0 = R.base;
        const float* st1 = R.base + (1 % D) * stage_floats;
        const int hk = hx_row(g, ih);
#pragma unroll
        for (int q = 0; q < G; ++q) {
            if (s0 + q >= g.S) continue;
            const int b = 5 + 6 * q;
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int c = c0 + v;
                float hx_unused = 0.f, hy = st0[b * SW + 2 * SW + c];
                if (yb.valid >> v & 1)
                    h_cell_s<false, false, true>(g, pml, ih, jb + v, c, hx_unused, hy, 0.f,
                                                 __fsub_rn(st1[b * SW + c], st0[b * SW + c]), st0[3 * SW + c],
                                                 st0 + 4 * SW, hk, false, false, st0 + (b + 4) * SW,
                                                 st0 + (b + 5) * SW, s0 + q, wp);
                hyu[q][v] = hy;
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&R.empty[0]);
        slot = 1 % D;
    } else {
        wait_bounded(g, &R.full[0], 0, R.abort_flag, ERR_WAIT_FULL);
    }
    int n = slot;  // ring sequence number of the current row (for barrier parity)

    int sc = g.src_off[blockIdx.x];
    const int se = g.src_off[blockIdx.x + 1];
    int rc = g.rx_off[blockIdx.x];
    const int re = g.rx_off[blockIdx.x + 1];
    const long long hplane = (long long)g.nx * g.Ph;

    for (int i = T.i0; i < T.i1; ++i, ++n) {
        const int nslot = (slot + 1 == D) ? 0 : slot + 1;
        wait_bounded(g, &R.full[nslot], ((n + 1) / D) & 1, R.abort_flag, ERR_WAIT_FULL);
        float* st = R.base + slot * stage_floats;
        const float* stn = R.base + nslot * stage_floats;
        const int hk = hx_row(g, i), ek = ex_row(g, i);
        float hyn[G][V];
        // --- H of row i
#pragma unroll
        for (int q = 0; q < G; ++q) {
            if (s0 + q >= g.S) continue;
            const int s = s0 + q;
            const int b = 5 + 6 * q;
            const float* ezc = st + b * SW;
            float* hxr = st + (b + 1) * SW;
            float ez[V + 1], en[V], hx[V], hy[V], ch[V];
            lds<V>(en, stn + b * SW + c0);
            lds<V>(hx, hxr + c0);
            lds<V>(hy, st + (b + 2) * SW + c0);
            lds<V>(ch, st + 3 * SW + c0);
            lds<V>(*reinterpret_cast<float(*)[V]>(ez), ezc + c0);
            ez[V] = ezc[c0 + V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                if (yb.valid >> v & 1)
                    h_cell_s<true, true, true>(g, pml, i, jb + v, c0 + v, hx[v], hy[v], __fsub_rn(ez[v + 1], ez[v]),
                                               __fsub_rn(en[v], ez[v]), ch[v], st + 4 * SW, hk, yb.h0 >> v & 1,
                                               yb.hm >> v & 1, st + (b + 4) * SW, st + (b + 5) * SW, s, wp);
                hyn[q][v] = hy[v];
            }
            // Hx of the column left of the band: from the old state, auxiliaries read only
            if (tid == 0 && T.b0 > 0) {
                const int j = T.b0 - 1;
                float hxl = hxr[3], hy_unused = 0.f;
                h_cell_s<false, true, false>(g, pml, i, j, 3, hxl, hy_unused, __fsub_rn(ez[0], ezc[3]), 0.f,
                                             st[3 * SW + 3], st + 4 * SW, -1, g.th > 0 && j <= g.th - 1,
                                             g.th > 0 && j >= g.ny - g.th, st + (b + 4) * SW, st + (b + 5) * SW, s, wp);
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
            const int b = 5 + 6 * q;
            const float* hxr = st + (b + 1) * SW;
            float ez[V], hx[V], ca[V], cb[V];
            lds<V>(ez, st + b * SW + c0);
            lds<V>(hx, hxr + c0);
            lds<V>(ca, st + c0);
            lds<V>(cb, st + SW + c0);
            const float hxl0 = hxr[c0 - 1];
            float ezw[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                ezw[v] = ez[v];
                if (yb.valid >> v & 1) {
                    const float hxl = (v > 0) ? hx[(v + V - 1) % V] : hxl0;
                    ezw[v] = e_cell_s<true>(g, pml, i, jb + v, c0 + v, ez[v], __fsub_rn(hyn[q][v], hyu[q][v]),
                                            __fsub_rn(hx[v], hxl), ca[v], cb[v], st + 2 * SW, ek, yb.e0 >> v & 1,
                                            yb.em >> v & 1, st + (b + 3) * SW, st + (b + 5) * SW, s, wp);
                }
            }
            while (sc < se) {
                const Ev e = __ldg(g.src_ev + sc);
                if (e.x != i || e.y != q) break;
#pragma unroll
                for (int v = 0; v < V; ++v)
                    if (jb + v == e.z)
                        ezw[v] = __fmaf_rn(-st[2 * SW + c0 + v], __ldg(g.srcw + (long long)e.w * g.nt + t), ezw[v]);
                ++sc;
            }
            if (act) {
                const long long ro = (long long)s * g.plane + (long long)i * P + jb;
                st_state<V>(g, g.ez[wp] + ro, ezw);
                st_state<V>(g, g.hx[wp] + ro, hx);
                st_state<V>(g, g.hy[wp] + ro, hyn[q]);
            }
            if (hist_act)
                st_state<V>(g, g.hist + ((long long)t * g.S + s) * hplane + (long long)i * g.Ph + jb, ezw);
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
        if (lane == 0) mbar_arrive(&R.empty[slot]);
        slot = nslot;
    }
}

// ---------------------------------------------------------------------------
// Reference-mode adjoint step
// ---------------------------------------------------------------------------

// E_new of row r of one shot for this thread's columns, written back into the
// stage's Ez slot.  sr: row r's stage; hyp: Hy_old of row r-1 (NULL when
// r == 0).  Injection events consumed from *cur.
template <int V>
__device__ __forceinline__ void adj_e_row(const GridDev& g, const float* pml, float* sr, int SW, int r, int q, int s,
                                          int jb, int c0, const YBits& yb, const float* hyp, bool store, int wp,
                                          const float* resid_s, int& cur, int end) {
    const int b = 5 + 6 * q;
    float* ezr = sr + b * SW;
    const float* hxr = sr + (b + 1) * SW;
    float ez[V], hx[V], hy[V], hu[V], ca[V], cb[V];
    lds<V>(ez, ezr + c0);
    lds<V>(hx, hxr + c0);
    lds<V>(hy, sr + (b + 2) * SW + c0);
    lds<V>(ca, sr + c0);
    lds<V>(cb, sr + SW + c0);
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
            if (jb + v == e.z) ez[v] = __fsub_rn(ez[v], resid_s[e.w]);
        ++cur;
    }
    const int ek = ex_row(g, r);
    float out[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        out[v] = ez[v];
        if (yb.valid >> v & 1) {
            const float hxl = (v > 0) ? hx[(v + V - 1) % V] : hxl0;
            const float dhy = __fsub_rn(hy[v], hu[v]), dhx = __fsub_rn(hx[v], hxl);
            out[v] = store ? e_cell_s<true>(g, pml, r, jb + v, c0 + v, ez[v], dhy, dhx, ca[v], cb[v], sr + 2 * SW, ek,
                                            yb.e0 >> v & 1, yb.em >> v & 1, sr + (b + 3) * SW, sr + (b + 5) * SW, s, wp)
                           : e_cell_s<false>(g, pml, r, jb + v, c0 + v, ez[v], dhy, dhx, ca[v], cb[v], sr + 2 * SW,
                                             ek, yb.e0 >> v & 1, yb.em >> v & 1, sr + (b + 3) * SW, sr + (b + 5) * SW,
                                             s, wp);
        }
    }
#pragma unroll
    for (int v = 0; v < V; ++v) ezr[c0 + v] = out[v];
}

// E_new of the column just past the band (be) of row r, from the stage (old
// values), with the halo-column injections of row r.
__device__ __forceinline__ void adj_e_halo(const GridDev& g, const float* pml, float* sr, int SW, int r, int q, int s,
                                           int be, int cbe, const float* hyp, const float* resid_s, int& cur, int end,
                                           bool active, int wp) {
    const int b = 5 + 6 * q;
    float* ezr = sr + b * SW;
    float ez = active ? ezr[cbe] : 0.f;
    while (cur < end) {
        const Ev e = __ldg(g.injh_ev + cur);
        if (e.x != r || e.y != q) break;
        if (active) ez = __fsub_rn(ez, resid_s[e.w]);
        ++cur;
    }
    if (!active) return;
    if (be < g.ny) {
        const float* hxr = sr + (b + 1) * SW;
        const float hu = hyp ? hyp[cbe] : 0.f;
        const int th = g.th;
        ez = e_cell_s<false>(g, pml, r, be, cbe, ez, __fsub_rn(sr[(b + 2) * SW + cbe], hu),
                             __fsub_rn(hxr[cbe], hxr[cbe - 1]), sr[cbe], sr[SW + cbe], sr + 2 * SW, ex_row(g, r),
                             th > 0 && be >= 1 && be <= th, th > 0 && be >= g.ny - th, sr + (b + 3) * SW,
                             sr + (b + 5) * SW, s, wp);
    } else {
        ez = 0.f;
    }
    ezr[cbe] = ez;
}

template <int V, int G>
__global__ void __launch_bounds__(512) k_adjoint_tma(const GridDev g, const int it, const int rp, const int D) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int nw = (blockDim.x >> 5) - 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int W = nw * 32 * V;
    const int SROWS = 5 + 8 * G;
    const int SW = ring_slot_width(W, g.TY);
    const Ring R = carve_ring(smem, D, SROWS, SW, g.th);
    const TileTma T = tma_tile(g, W);
    if (T.grp * G >= g.S) return;
    const int wp = rp ^ 1;
    const int r_first = T.i0 >= 1 ? T.i0 - 1 : T.i0;
    const int r_last = min(T.i1, g.nx - 1);   // row nx is the zero frame: never loaded
    ring_init(g, R, nw);
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
    const int stage_floats = SROWS * SW;
    const YBits yb = ybits<V>(g, jb);
    const bool act = jb < P;
    const float* pml = R.pml;
    int ic = g.inj_off[blockIdx.x];
    const int ie = g.inj_off[blockIdx.x + 1];
    int hc = g.injh_off[blockIdx.x];
    const int he = g.injh_off[blockIdx.x + 1];
    double* gae = g.gacc + (long long)T.grp * 2 * ((long long)nx * ny);
    double* gas = gae + (long long)nx * ny;
    const long long rstride = (long long)g.nt * g.nrx;
    const float* resid_t = g.resid + (long long)it * g.nrx;

    // Prologue: E_new of row i0.
    int slot = 0;
    if (T.i0 >= 1) {
        wait_bounded(g, &R.full[0], 0, R.abort_flag, ERR_WAIT_FULL);
        wait_bounded(g, &R.full[1 % D], (1 / D) & 1, R.abort_flag, ERR_WAIT_FULL);
        slot = 1 % D;
    } else {
        wait_bounded(g, &R.full[0], 0, R.abort_flag, ERR_WAIT_FULL);
    }
    {
        float* st = R.base + slot * stage_floats;
#pragma unroll
        for (int q = 0; q < G; ++q) {
            const int s = s0 + q;
            if (s >= g.S) continue;
            const float* hyp = (T.i0 >= 1) ? R.base + (5 + 6 * q + 2) * SW : nullptr;
            adj_e_row<V>(g, pml, st, SW, T.i0, q, s, jb, c0, yb, hyp, true, wp, resid_t + s * rstride, ic, ie);
            adj_e_halo(g, pml, st, SW, T.i0, q, s, be, cbe, hyp, resid_t + s * rstride, hc, he, halo_thread, wp);
        }
    }
    if (T.i0 >= 1) {
        __syncwarp();
        if (lane == 0) mbar_arrive(&R.empty[0]);
    }
    int n = slot;

    for (int i = T.i0; i < T.i1; ++i, ++n) {
        const int r = i + 1;
        const bool have_r = r < nx;
        const int nslot = (slot + 1 == D) ? 0 : slot + 1;
        float* st = R.base + slot * stage_floats;
        float* stn = R.base + nslot * stage_floats;
        if (have_r) wait_bounded(g, &R.full[nslot], ((n + 1) / D) & 1, R.abort_flag, ERR_WAIT_FULL);
        // --- E of row r (row i1 is the next chunk's: computed, auxiliaries not stored)
        if (have_r) {
#pragma unroll
            for (int q = 0; q < G; ++q) {
                const int s = s0 + q;
                if (s >= g.S) continue;
                const float* hyp = st + (5 + 6 * q + 2) * SW;
                adj_e_row<V>(g, pml, stn, SW, r, q, s, jb, c0, yb, hyp, r < T.i1, wp, resid_t + s * rstride, ic,
                             ie);
                if (r < T.i1)
                    adj_e_halo(g, pml, stn, SW, r, q, s, be, cbe, hyp, resid_t + s * rstride, hc, he, halo_thread,
                               wp);
            }
        }
        consumer_sync(ncons);
        // --- H of row i and imaging
        const int hk = hx_row(g, i);
        float acc_e[V], acc_s[V];
#pragma unroll
        for (int v = 0; v < V; ++v) { acc_e[v] = 0.f; acc_s[v] = 0.f; }
#pragma unroll
        for (int q = 0; q < G; ++q) {
            const int s = s0 + q;
            if (s >= g.S) continue;
            const int b = 5 + 6 * q;
            const float* ezc = st + b * SW;
            float ez[V + 1], en[V], hx[V], hy[V], ch[V], f1[V], f0[V];
            lds<V>(*reinterpret_cast<float(*)[V]>(ez), ezc + c0);
            ez[V] = ezc[c0 + V];
            if (have_r) {
                lds<V>(en, stn + b * SW + c0);
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) en[v] = 0.f;
            }
            lds<V>(hx, st + (b + 1) * SW + c0);
            lds<V>(hy, st + (b + 2) * SW + c0);
            lds<V>(ch, st + 3 * SW + c0);
            lds<V>(f1, st + (5 + 6 * G + 2 * q) * SW + c0);
            lds<V>(f0, st + (6 + 6 * G + 2 * q) * SW + c0);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                if (yb.valid >> v & 1) {
                    h_cell_s<true, true, true>(g, pml, i, jb + v, c0 + v, hx[v], hy[v], __fsub_rn(ez[v + 1], ez[v]),
                                               __fsub_rn(en[v], ez[v]), ch[v], st + 4 * SW, hk, yb.h0 >> v & 1,
                                               yb.hm >> v & 1, st + (b + 4) * SW, st + (b + 5) * SW, s, wp);
                    acc_e[v] = __fadd_rn(acc_e[v], __fmul_rn(__fsub_rn(f1[v], f0[v]), ez[v]));
                    acc_s[v] = __fadd_rn(acc_s[v], __fmul_rn(__fmul_rn(f1[v], ez[v]), g.dt));
                }
            }
            if (act) {
                const long long ro = (long long)s * g.plane + (long long)i * P + jb;
                st_state<V>(g, g.ez[wp] + ro, *reinterpret_cast<float(*)[V]>(ez));
                st_state<V>(g, g.hx[wp] + ro, hx);
                st_state<V>(g, g.hy[wp] + ro, hy);
            }
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
            if (yb.valid >> v & 1) {
                const long long o = (long long)i * ny + jb + v;
                gae[o] += (double)acc_e[v];
                gas[o] += (double)acc_s[v];
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&R.empty[slot]);
        slot = nslot;
    }
}

}  // namespace fg
