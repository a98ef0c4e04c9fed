// Lane-march time-step kernels: one launch per time step, persistent warps
// that fetch tiles from a counter, no synchronisation between warps.
//
// Tile = (shot group, row chunk [i0, i1), column band).  Each thread owns W
// consecutive columns j0 .. j0+W-1 of one shot and marches down the rows of
// the chunk, carrying the previous row's values in registers, so every cell's
// Ez/Hx/Hy is read once and written once per step.  The one-cell halo a
// thread needs from outside its columns (column j0-1 / j0+W, row i0-1 / i1)
// is recomputed from the previous step's state, which lives in the other
// buffer of a ping-pong pair, so tiles never wait on each other.
//
//   shot lanes   (SHOT = true):  lane l is shot slot l of the group (CS = 32);
//                all lanes of a warp touch the same cells, so each access is
//                one 128-byte line, coefficients are warp-uniform and every
//                boundary branch is uniform across the warp.
//   column lanes (SHOT = false): one shot per group (CS = 1); lane l owns
//                columns b0 + l*W .. b0 + l*W + W-1.
//
// Scheduling: the grid holds as many warps as fit on the GPU; each warp takes
// the next tile position from a per-launch counter (CPML-heavy tiles come
// first in the order table), so the slow boundary tiles start early and the
// light interior tiles fill in behind them.
//
// Operand delivery (RING):
//   false  each row's operands are loaded from global memory into registers
//          when the row is computed;
//   true   lane 0 of each warp streams the warp's row segments -- contiguous
//          runs of whole cells (all 32 shots of a cell are adjacent) -- into
//          a D-stage shared-memory ring with cp.async.bulk, D rows ahead and
//          across tile boundaries, completing on one mbarrier per stage.
//          Bytes in flight then cost no registers.  Waits are bounded: a
//          stage that does not complete within 2 s sets the device error
//          word, the warp waits (bounded) for its copies in flight and
//          leaves, and later launches of the solve return at once.
//
// Forward step t (src/compute.py:574-712), per row i: Hx (columns j0-1 ..
// j0+W-1) and Hy from the old Ez, then Ez from the new H, the CPML
// corrections of each, the source injection, the stores, the Ez history and
// the receiver samples (trace[t+1] = Ez after step t, which is what the
// reference's store_outputs reads at the start of step t+1).
//
// Reference-mode adjoint step (src/compute.py:1048-1172): residual injection
// at the receivers, E (Ucgeta's uE0) from the old H, then H from the new E,
// then the imaging sums with the stored forward Ez.  The march computes E one
// row ahead of H; the imaging products of a warp's 32 shots are summed by a
// reduce-scatter over the lanes and added to the group's fp64 accumulator.
#pragma once

#include "fdtd_common.cuh"
#include "fdtd_shot.cuh"

namespace fg {


// ---------------------------------------------------------------------------
// mbarrier / bulk-copy primitives (no multicast anywhere)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
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
// Bulk global -> shared copy completing on `bar`.
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

// Arm `bar` for the copies `each` enumerates and issue them.  `each(f)` calls
// f(dst, src, bytes) for every copy of the stage; the byte count is summed in
// a first pass, so the barrier always expects exactly what is issued (the
// checked build drops -- and records -- a copy whose source is out of range).
template <class Each>
__device__ __forceinline__ void issue_stage(const Dev& g, uint64_t* bar, Each&& each) {
    uint32_t total = 0;
    each([&](void*, const void* s, uint32_t b) {
        if (b && FG_OK_PTR(g, s, (int)b)) total += b;
    });
    mbar_expect_tx(bar, total);
    each([&](void* d, const void* s, uint32_t b) {
        if (b && FG_OK_PTR(g, s, (int)b)) bulk_g2s(d, s, b, bar);
    });
}

constexpr int ERR_WAIT_STAGE = 201;                          // device error word: a stage never completed
constexpr unsigned long long WAIT_LIMIT_NS = 2000000000ull;  // 2 s; a stage normally lands in microseconds

// Bounded wait of one thread for phase `parity` of `bar`.
__device__ __forceinline__ bool wait_stage(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    while (!mbar_try_wait(bar, parity)) {
        if (globaltimer() - t0 > WAIT_LIMIT_NS) return false;
        __nanosleep(20);
    }
    return true;
}

// Geometry of a warp's ring stage.
template <int W, bool SHOT>
struct RingGeom {
    static constexpr int CS = SHOT ? 32 : 1;
    static constexpr int BW = SHOT ? W : 32 * W;        // columns of a band
    static constexpr int NS = SHOT ? W + 2 : BW + 8;    // cells of a state segment
    static constexpr int NH = BW;                       // cells of a history segment
    static constexpr int NCF = SHOT ? W + 8 : BW + 8;   // floats of a coefficient segment
    static constexpr int FWD = 3 * NS * CS + 3 * NCF;   // floats of a forward stage
    static constexpr int ADJ = 3 * NS * CS + NH * CS + 3 * NCF;   // floats of an adjoint stage
};

// Dynamic shared memory: the CPML profile, then (RING) the barriers and the
// stages of every warp of the block.
__host__ __device__ inline size_t prof_bytes(int th) { return ((size_t)8 * th * 4 + 127) / 128 * 128; }
__host__ __device__ inline size_t ring_bar_bytes(int wpb, int D) { return (((size_t)wpb * D * 8) + 127) / 128 * 128; }

// Copy the CPML profile (8 x th) into shared memory; every thread of the
// block passes the barrier.
__device__ __forceinline__ const float* stage_profile(const Dev& g, unsigned char* smem) {
    float* R = reinterpret_cast<float*>(smem);
    for (int k = threadIdx.x; k < 8 * g.th; k += blockDim.x) R[k] = __ldg(g.pml + k);
    __syncthreads();
    return R;
}

// Bulk prefetch of [p, p + bytes) into L2 (no data returned).
__device__ __forceinline__ void prefetch_l2(const float* p, long long first, long long last) {
    // [first, last] in floats, widened to 16-byte boundaries
    const long long a = first & ~3LL, b = (last | 3LL) + 1;
    if (b <= a) return;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p + a), "r"((uint32_t)((b - a) * 4)) : "memory");
}

// Prefetch into L2 the CPML auxiliaries (read parity) a tile of rows
// [r0, r1] and columns [jlo, jhi] touches, so that the consumers' gather
// loads of a CPML tile hit L2.  Issued by the producer, S tiles ahead.
template <int CS>
__device__ __forceinline__ void prefetch_tile_psi(const Dev& g, int grp, int rp, int r0, int r1, int jlo, int jhi) {
    const int th = g.th, nx = g.nx, ny = g.ny, P = g.P, TY = g.TY;
    if (th <= 0) return;
    r0 = max(r0, 0);
    r1 = min(r1, nx - 1);
    jlo = max(jlo, 0);
    jhi = min(jhi, ny - 1);
    if (r0 > r1 || jlo > jhi) return;
    const PsiG rd = psi_group(g, rp, grp);
    // x slabs: E rows 1..th (k = th-i), H rows 0..th-1 (k = th-1-i), both nx-th.. (k = th+i-(nx-th))
    for (int i = r0; i <= r1; ++i) {
        const int ke = (i >= 1 && i <= th) ? th - i : (i >= nx - th ? th + i - (nx - th) : -1);
        const int kh = (i <= th - 1) ? th - 1 - i : (i >= nx - th ? th + i - (nx - th) : -1);
        if (ke >= 0) prefetch_l2(rd.ex, ((long long)ke * P + jlo) * CS, ((long long)ke * P + jhi) * CS + CS - 1);
        if (kh >= 0) prefetch_l2(rd.hx, ((long long)kh * P + jlo) * CS, ((long long)kh * P + jhi) * CS + CS - 1);
    }
    // y slabs: y0 columns 0..th (k = th-j for E, th-1-j for H), ymax columns ny-th.. (k = j-(ny-th))
    const bool y0 = jlo <= th, ym = jhi >= ny - th;
    if (!y0 && !ym) return;
    const int k0lo = max(0, th - 1 - jhi), k0hi = min(th - 1, th - jlo);
    const int kmlo = max(jlo, ny - th) - (ny - th), kmhi = jhi - (ny - th);
    for (int i = r0; i <= r1; ++i) {
        if (y0 && k0lo <= k0hi) {
            const long long o = (long long)i * TY;
            prefetch_l2(rd.ey, (o + k0lo) * CS, (o + k0hi) * CS + CS - 1);
            prefetch_l2(rd.hy, (o + k0lo) * CS, (o + k0hi) * CS + CS - 1);
        }
        if (ym && kmlo <= kmhi) {
            const long long o = (long long)(nx + 1 + i) * TY;
            prefetch_l2(rd.ey, (o + kmlo) * CS, (o + kmhi) * CS + CS - 1);
            prefetch_l2(rd.hy, (o + kmlo) * CS, (o + kmhi) * CS + CS - 1);
        }
    }
}

// Prefetch into L2 what the shot-lane tile at fetch position `pos` will read
// from the state of parity rp -- Ez, Hx and Hy of rows [i0-1, i1] (clamped to
// the plane), columns j0-1 .. j0+W -- and, when hist is set (adjoint), its
// Ez history rows [i0, i1) of step `it`, plus the CPML auxiliaries of a
// boundary tile.  One bulk prefetch per lane; issued a tile ahead, so the
// tile's own loads find their lines in L2.
template <int W>
__device__ __forceinline__ void prefetch_tile_shot(const Dev& g, int pos, int rp, int lane, const float* hist, int it) {
    if (pos >= g.ntiles) return;
    const int id = __ldg(g.order + pos);
    const int band = id % g.nb, rest = id / g.nb, chunk = rest % g.nc, grp = rest / g.nc;
    const int i0 = __ldg(g.chunk_row + chunk), i1 = __ldg(g.chunk_row + chunk + 1);
    const int j0 = band * W;
    const int r0 = max(i0 - 1, 0), r1 = min(i1, g.nx), nr = r1 - r0 + 1;
    const int nh = hist && j0 < g.Ph ? i1 - i0 : 0;
    const long long go = (long long)grp * g.plane + ((long long)r0 * g.P + j0 - 1 + PADC) * 32;
    const long long rowS = (long long)g.P * 32;
    for (int k = lane; k < 3 * nr + nh; k += 32) {
        const float* p;
        uint32_t bytes;
        if (k < 3 * nr) {
            const int f = k / nr, r = k - f * nr;
            const float* base = f == 0 ? g.ez[rp] : (f == 1 ? g.hx[rp] : g.hy[rp]);
            p = base + go + r * rowS;
            bytes = (W + 2) * 128;
        } else {
            const int i = i0 + (k - 3 * nr);
            p = hist + ((((long long)(it - g.hist_t0) * g.ngroups + grp) * g.nx + i) * g.Ph + j0) * 32;
            bytes = (uint32_t)min(W, g.Ph - j0) * 128;
        }
        if (!FG_OK_PTR(g, p, (int)bytes)) continue;
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
    }
    if (lane == 0 && g.th > 0) prefetch_tile_psi<32>(g, grp, rp, r0, r1, j0 - 1, j0 + W);
}

// ---------------------------------------------------------------------------
// Tiles
// ---------------------------------------------------------------------------
template <bool SHOT>
struct LaneTile {
    int id, grp, i0, i1, b0, j0, l, s;
    bool live;
};

template <int W, bool SHOT>
__device__ __forceinline__ LaneTile<SHOT> decode_tile(const Dev& g, int id, int lane) {
    LaneTile<SHOT> T;
    T.id = id;
    const int band = id % g.nb;
    const int rest = id / g.nb;
    const int chunk = rest % g.nc;
    T.grp = rest / g.nc;
    T.i0 = __ldg(g.chunk_row + chunk);
    T.i1 = __ldg(g.chunk_row + chunk + 1);
    if (SHOT) {
        T.l = lane;
        T.b0 = band * W;
        T.j0 = T.b0;
        T.s = T.grp * 32 + lane;
        T.live = true;   // padded slots (s >= S) exist in memory and stay zero
    } else {
        T.l = 0;
        T.b0 = band * 32 * W;
        T.j0 = T.b0 + lane * W;
        T.s = T.grp;
        T.live = T.j0 < g.ny;
    }
    return T;
}

// Programmatic dependent launch: a kernel launched behind this one with the
// programmatic-serialization attribute may start once every block of this
// one has executed launch_dependents; it calls griddep_wait before it
// completes, so it never completes before this one.  Both are no-ops for
// launches without a dependent / a prerequisite.
__device__ __forceinline__ void griddep_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Next tile position of this warp (lane 0 takes it, all lanes see it).
__device__ __forceinline__ int fetch_tile(int* ctr, int lane) {
    int p = 0;
    if (lane == 0) p = atomicAdd(ctr, 1);
    return __shfl_sync(FULL, p, 0);
}

// A tile as the ring producer sees it: rows [i0, i1) and the element
// offsets of its row-0 segments, decoded once when the tile is fetched.
struct TileQ {
    int i0 = 0, i1 = 0;   // i1 <= i0: no tile
    long long sbase = 0;  // state segment of row 0 within the field buffers
    long long cbase = 0;  // coefficient segment of row 0
    long long hbase = 0;  // history segment of row 0 (adjoint)
    uint32_t hs = 0;      // bytes of a history segment (adjoint)
};

template <int W, bool SHOT>
__device__ __forceinline__ TileQ tile_q(const Dev& g, int pos, int it) {
    TileQ q;
    if (pos >= g.ntiles) return q;
    constexpr int CS = SHOT ? 32 : 1;
    const LaneTile<SHOT> T = decode_tile<W, SHOT>(g, __ldg(g.order + pos), 0);
    q.i0 = T.i0;
    q.i1 = T.i1;
    const int c0s = SHOT ? T.b0 - 1 : T.b0 - 4;   // 16-byte aligned segment starts
    q.sbase = (long long)T.grp * g.plane + (long long)(c0s + PADC) * CS;
    q.cbase = T.b0 - 4 + PADC;
    const long long hrow = (long long)g.Ph * CS;
    q.hbase = ((long long)(it - g.hist_t0) * g.ngroups + T.grp) * g.nx * hrow + (long long)T.b0 * CS;
    // history cells of the band that exist in a history row
    const int hcells = SHOT ? W : max(0, min(32 * W, g.Ph - T.b0));
    q.hs = (uint32_t)hcells * CS * 4;
    return q;
}

// Producer of a warp's ring: streams the rows of the current and the next
// tile.  Only lane 0 runs it.  Invariant: (ptile, prow) names the next row to
// issue, ptile = 0 for the current tile and 1 for the next one.
struct RingProducer {
    int ptile = 0, prow = 0;
    uint32_t qi = 0;   // stages issued
    int slot = 0;      // qi % D
    TileQ q[2];        // current and next tile
};

// ---------------------------------------------------------------------------
// Forward step
// ---------------------------------------------------------------------------
template <int W>
struct FwdIn {                 // operands of row i
    float en[W + 2];           // Ez_old(i+1, j0-1 .. j0+W)
    float hxo[W + 1];          // Hx_old(i, j0-1 .. j0+W-1)
    float hyo[W];              // Hy_old(i, j0 .. j0+W-1)
    float ca[W], cb[W];        // uE0, uE1 (i, j0 ..)
    float ch[W + 1];           // uH1 (i, j0-1 ..)
};

// Interior forward row (every cell of H at columns j0-1 .. j0+W-1 and of E
// at j0 .. j0+W-1 away from the CPML and the frame): the leapfrog of
// fields_updates_gpu.cu:47-78 then :8-33.
template <int W>
__device__ __forceinline__ void fwd_core(const FwdIn<W>& B, const float (&ezc)[W + 2], const float (&hyu)[W],
                                         float (&hxn)[W + 1], float (&hyn)[W], float (&ezn)[W]) {
#pragma unroll
    for (int k = 0; k <= W; ++k) hxn[k] = __fsub_rn(B.hxo[k], __fmul_rn(B.ch[k], __fsub_rn(ezc[k + 1], ezc[k])));
#pragma unroll
    for (int w = 0; w < W; ++w)
        hyn[w] = __fadd_rn(B.hyo[w], __fmul_rn(B.ch[w + 1], __fsub_rn(B.en[w + 1], ezc[w + 1])));
#pragma unroll
    for (int w = 0; w < W; ++w)
        ezn[w] = __fmaf_rn(-B.cb[w], __fsub_rn(hxn[w + 1], hxn[w]),
                           madd2(B.ca[w], ezc[w + 1], B.cb[w], __fsub_rn(hyn[w], hyu[w])));
}

// Hertzian dipole (sourcereceiver.cu:84) on the new Ez of row i, in list
// order: the tile's source events of the row from sc on.
template <int W>
__device__ __forceinline__ void fwd_sources(const Dev& g, int i, int t, int j0, int slot, float (&ezn)[W], int& sc,
                                            int se) {
    for (; sc < se; ++sc) {
        const Ev e = __ldg(g.src_ev + sc);
        if (e.x != i) break;
        if (e.y != slot) continue;
#pragma unroll
        for (int w = 0; w < W; ++w)
            if (j0 + w == e.z) {
                const float cd = ldro(g, g.cd + coef_at(g, i, e.z));
                ezn[w] = __fmaf_rn(-cd, __ldg(g.srcw + (long long)e.w * g.nt + t), ezn[w]);
            }
    }
}

// Receiver samples of row i (store_outputs, sourcereceiver.cu:11-56, reads
// Ez at the start of step t+1 = after step t).
template <int W>
__device__ __forceinline__ void fwd_receivers(const Dev& g, int i, int t, int j0, int slot, int s, const float (&ezn)[W],
                                              int& rc, int re) {
    for (; rc < re; ++rc) {
        const Ev e = __ldg(g.rx_ev + rc);
        if (e.x != i) break;
        if (e.y != slot || t + 1 >= g.nt) continue;
#pragma unroll
        for (int w = 0; w < W; ++w)
            if (j0 + w == e.z && g.traces) g.traces[((long long)s * g.nt + t + 1) * g.nrx + e.w] = ezn[w];
    }
}

// Row i of the forward step from its operands; carries ezc (Ez_old of row i,
// columns j0-1 .. j0+W) and hyu (Hy_new of row i-1) to the next row.
template <int W, int CS, bool LEAN = false>
__device__ __forceinline__ void fwd_row(const Dev& g, const float* R, const BandY& by, const FwdIn<W>& B,
                                        float (&ezc)[W + 2], float (&hyu)[W], int i, int t, int j0, int l, int slot,
                                        int s, bool bcore,
                                        float* ezW, float* hxW, float* hyW, float* hist, long long hrow,
                                        const PsiG& rd, const PsiG& wr, int& sc, int se, int& rc, int re) {
    const int nx = g.nx, ny = g.ny, th = g.th;
    float hxn[W + 1], hyn[W], ezn[W];
    if (bcore && i >= th + 1 && i <= nx - th - 1) {
        fwd_core<W>(B, ezc, hyu, hxn, hyn, ezn);
    } else if (CS == 32 && (LEAN || by.lean)) {
        if constexpr (CS == 32)
            fwd_row_shot<W>(g, R, by, i, j0, l, B.hxo, B.hyo, B.en, ezc, hyu, B.ca, B.cb, B.ch, rd, wr, hxn, hyn, ezn);
    } else if (g.fast_cpml) {
        float dzx[W + 1], dzy[W], dhy[W], dhx[W];
#pragma unroll
        for (int k = 0; k <= W; ++k) {
            hxn[k] = B.hxo[k];
            dzx[k] = __fsub_rn(ezc[k + 1], ezc[k]);
        }
        hx_cells<W + 1, CS>(g, R, i, j0 - 1, l, hxn, dzx, B.ch, 1, rd, wr);
#pragma unroll
        for (int w = 0; w < W; ++w) {
            hyn[w] = B.hyo[w];
            dzy[w] = __fsub_rn(B.en[w + 1], ezc[w + 1]);
        }
        hy_cells<W, CS, true>(g, R, i, j0, l, hyn, dzy, B.ch + 1, rd, wr);
#pragma unroll
        for (int w = 0; w < W; ++w) {
            ezn[w] = ezc[w + 1];
            dhy[w] = __fsub_rn(hyn[w], hyu[w]);
            dhx[w] = __fsub_rn(hxn[w + 1], hxn[w]);
        }
        e_cells<W, CS>(g, R, i, j0, l, ezn, dhy, dhx, B.ca, B.cb, W, true, rd, wr);
    } else {
#pragma unroll
        for (int k = 0; k <= W; ++k) {
            const int j = j0 - 1 + k;
            hxn[k] = B.hxo[k];
            if (j >= 0 && j < ny) {
                const float dz = __fsub_rn(ezc[k + 1], ezc[k]);
                if (k == 0) hxn[k] = hx_cell<CS, false>(g, R, i, j, l, B.hxo[k], dz, B.ch[k], rd, rd);
                else hxn[k] = hx_cell<CS, true>(g, R, i, j, l, B.hxo[k], dz, B.ch[k], rd, wr);
            }
        }
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const int j = j0 + w;
            hyn[w] = B.hyo[w];
            if (j < ny)
                hyn[w] = hy_cell<CS, true>(g, R, i, j, l, B.hyo[w], __fsub_rn(B.en[w + 1], ezc[w + 1]), B.ch[w + 1],
                                           rd, wr);
        }
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const int j = j0 + w;
            ezn[w] = ezc[w + 1];
            if (j < ny)
                ezn[w] = e_cell<CS, true>(g, R, i, j, l, ezc[w + 1], __fsub_rn(hyn[w], hyu[w]),
                                          __fsub_rn(hxn[w + 1], hxn[w]), B.ca[w], B.cb[w], rd, wr);
        }
    }
    fwd_sources<W>(g, i, t, j0, slot, ezn, sc, se);
    const long long o = ((long long)i * g.P + j0 + PADC) * CS + l;
    st_cells<W, CS>(g, ezW + o, ezn);
    st_cells<W, CS>(g, hxW + o, hxn + 1);
    st_cells<W, CS>(g, hyW + o, hyn);
    if (hist && j0 < g.Ph) st_cells<W, CS, true>(g, hist + (long long)i * hrow, ezn);
    fwd_receivers<W>(g, i, t, j0, slot, s, ezn, rc, re);
#pragma unroll
    for (int k = 0; k < W + 2; ++k) ezc[k] = B.en[k];
#pragma unroll
    for (int w = 0; w < W; ++w) hyu[w] = hyn[w];
}

// Stage of forward row i of tile Q: Ez_old of row i+1, Hx_old and Hy_old of
// row i, and the uE0 / uE1 / uH1 coefficient rows.
template <int W, bool SHOT>
__device__ __forceinline__ void issue_fwd(const Dev& g, uint64_t* bar, float* st, const TileQ& Q, int i, int rp) {
    using RG = RingGeom<W, SHOT>;
    constexpr int CS = RG::CS;
    constexpr uint32_t zs = (uint32_t)(SHOT ? (W + 2) : RG::NS) * CS * 4;
    constexpr uint32_t xs = (uint32_t)(SHOT ? (W + 1) : RG::NS) * CS * 4;
    constexpr uint32_t ys = (uint32_t)(SHOT ? W : RG::NS) * CS * 4;
    constexpr uint32_t cs = (uint32_t)RG::NCF * 4;
    constexpr int yo = SHOT ? CS : 0;   // Hy starts one cell later in shot-lane stages
    const long long rowS = (long long)g.P * CS;
    const long long so = Q.sbase + (long long)i * rowS;
    const long long co = Q.cbase + (long long)i * g.P;
    float* cst = st + 3 * RG::NS * CS;
    issue_stage(g, bar, [&](auto&& f) {
        f(st, g.ez[rp] + so + rowS, zs);
        f(st + RG::NS * CS, g.hx[rp] + so, xs);
        f(st + 2 * RG::NS * CS + yo, g.hy[rp] + so + yo, ys);
        f(cst, g.ca + co, cs);
        f(cst + RG::NCF, g.cb + co, cs);
        f(cst + 2 * RG::NCF, g.ch + co, cs);
    });
}

// Forward step t of one solve by the warps of this block: tiles from the
// step's counter until none is left.  R: the CPML profile (shared or global
// memory); smem: the block's dynamic shared memory (RING stages after the
// profile).
// LEAN: every band of the plan takes the shot-lane CPML rows (the host checks
// it: fast_cpml and no band with cells in both y slabs), so the generic
// per-cell CPML paths are compiled out.
template <int W, bool SHOT, bool RING, bool LEAN = false>
__device__ __forceinline__ void fwd_step(const Dev& g, const float* R, unsigned char* smem, const int t, const int D) {
    constexpr int CS = SHOT ? 32 : 1;
    using RG = RingGeom<W, SHOT>;
    if (blockIdx.x == 0 && threadIdx.x == 0) g.tile_ctr[(t + 1) & 1] = 0;   // the next launch's counter
    int* ctr = g.tile_ctr + (t & 1);
    const int lane = threadIdx.x & 31;
    const int P = g.P, ny = g.ny, th = g.th, nt_ = g.ntiles;
    const int rp = t & 1, wp = rp ^ 1;
    const long long hrow = (long long)g.Ph * CS;

    uint64_t* bars = nullptr;
    float* ring = nullptr;
    if (RING) {
        const int wib = threadIdx.x >> 5;
        unsigned char* base = smem + prof_bytes(th);
        bars = reinterpret_cast<uint64_t*>(base) + (size_t)wib * D;
        ring = reinterpret_cast<float*>(base + ring_bar_bytes(blockDim.x >> 5, D)) + (size_t)wib * D * RG::FWD;
        if (lane == 0) {
            for (int d = 0; d < D; ++d) mbar_init(bars + d, 1);
            fence_mbar_init();
        }
        __syncwarp();
    }
    int cur = fetch_tile(ctr, lane);
    int nxt = cur < nt_ ? fetch_tile(ctr, lane) : nt_;
    RingProducer pr;
    uint32_t qc = 0;   // stages consumed
    int cslot = 0;     // qc % D
    uint32_t cpar = 0; // (qc / D) & 1
    if (RING && lane == 0) {
        pr.q[0] = tile_q<W, SHOT>(g, cur, 0);
        pr.q[1] = tile_q<W, SHOT>(g, nxt, 0);
    }
    auto produce = [&]() {
        while ((int)(pr.qi - qc) < D && pr.ptile <= 1) {
            const TileQ& Q = pr.q[pr.ptile];
            if (Q.i1 <= Q.i0) break;
            issue_fwd<W, SHOT>(g, bars + pr.slot, ring + (size_t)pr.slot * RG::FWD, Q, Q.i0 + pr.prow, rp);
            ++pr.qi;
            if (++pr.slot == D) pr.slot = 0;
            if (++pr.prow >= Q.i1 - Q.i0) {
                ++pr.ptile;
                pr.prow = 0;
            }
        }
    };
#define FG_CELL(i, j) (((long long)(i) * P + (j) + PADC) * CS + l)

    while (cur < nt_) {
        const LaneTile<SHOT> T = decode_tile<W, SHOT>(g, __ldg(g.order + cur), lane);
        if (RING && lane == 0) produce();
        if (SHOT && !RING && g.pf == 1) prefetch_tile_shot<W>(g, nxt, rp, lane, nullptr, 0);
        const int l = T.l, j0 = T.j0, slot = SHOT ? l : 0;
        const long long go = (long long)T.grp * g.plane;
        const float* ezR = g.ez[rp] + go;
        const float* hyR = g.hy[rp] + go;
        const float* hxR = g.hx[rp] + go;
        float* ezW = g.ez[wp] + go;
        float* hxW = g.hx[wp] + go;
        float* hyW = g.hy[wp] + go;
        const PsiG rd = psi_group(g, rp, T.grp), wr = psi_group(g, wp, T.grp);
        // H at columns j0-1 .. j0+W-1 and E at j0 .. j0+W-1 are all interior cells
        const bool bcore = j0 >= th + 1 && j0 + W <= ny - th;
        BandY by{};
        if constexpr (SHOT) by = band_fwd<W>(g, j0);
        int sc = __ldg(g.src_off + T.id);
        const int se = __ldg(g.src_off + T.id + 1);
        int rc = __ldg(g.rx_off + T.id);
        const int re = __ldg(g.rx_off + T.id + 1);
        float* hist = g.hist ? g.hist + (((long long)(t - g.hist_t0) * g.ngroups + T.grp) * g.nx) * hrow + (long long)j0 * CS + l
                             : nullptr;
        // Ez_old of row i0, columns j0-1 .. j0+W, and the new Hy of the row
        // above the chunk (its auxiliaries are only read)
        float ezc[W + 2], hyu[W];
        // operands of row i (direct loads)
        FwdIn<W> B;
        auto load_row = [&](int i) {
            const long long crow = coef_at(g, i, j0);
            B.en[0] = ldro(g, ezR + FG_CELL(i + 1, j0 - 1));
            ld_cells<W, CS>(g, B.en + 1, ezR + FG_CELL(i + 1, j0));
            B.en[W + 1] = ldro(g, ezR + FG_CELL(i + 1, j0 + W));
            B.hxo[0] = ldro(g, hxR + FG_CELL(i, j0 - 1));
            ld_cells<W, CS>(g, B.hxo + 1, hxR + FG_CELL(i, j0));
            ld_cells<W, CS>(g, B.hyo, hyR + FG_CELL(i, j0));
            ld_coef<W, CALIGN<W>>(g, B.ca, g.ca + crow);
            ld_coef<W, CALIGN<W>>(g, B.cb, g.cb + crow);
            B.ch[0] = ldro(g, g.ch + crow - 1);
            ld_coef<W, CALIGN<W>>(g, B.ch + 1, g.ch + crow);
        };
#pragma unroll
        for (int w = 0; w < W; ++w) hyu[w] = 0.f;
        if (T.live) {
            ezc[0] = ldro(g, ezR + FG_CELL(T.i0, j0 - 1));
            ld_cells<W, CS>(g, ezc + 1, ezR + FG_CELL(T.i0, j0));
            ezc[W + 1] = ldro(g, ezR + FG_CELL(T.i0, j0 + W));
            // the first row's operands go out with the halo row's, so the tile
            // start costs one memory round trip
            if (!RING) load_row(T.i0);
            if (T.i0 >= 1) {
                const int ih = T.i0 - 1;
                float ea[W], ha[W], ca[W], dz[W];
                ld_cells<W, CS>(g, ea, ezR + FG_CELL(ih, j0));
                ld_cells<W, CS>(g, ha, hyR + FG_CELL(ih, j0));
                ld_coef<W, CALIGN<W>>(g, ca, g.ch + coef_at(g, ih, j0));
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    hyu[w] = ha[w];
                    dz[w] = __fsub_rn(ezc[w + 1], ea[w]);
                }
                if (SHOT && (LEAN || by.lean)) {
                    if constexpr (SHOT) fwd_hy_halo_shot<W>(g, R, by, ih, j0, l, hyu, dz, ca, rd);
                } else if (g.fast_cpml) {
                    hy_cells<W, CS, false>(g, R, ih, j0, l, hyu, dz, ca, rd, rd);
                } else {
#pragma unroll
                    for (int w = 0; w < W; ++w)
                        if (j0 + w < ny) hyu[w] = hy_cell<CS, false>(g, R, ih, j0 + w, l, ha[w], dz[w], ca[w], rd, rd);
                }
            }
        }
        const int nrow = T.i1 - T.i0;
        for (int n = 0; n < nrow; ++n) {
            const int i = T.i0 + n;
            if (SHOT && !RING && g.pf == 2 && n == nrow / 2) prefetch_tile_shot<W>(g, nxt, rp, lane, nullptr, 0);
            if (RING) {
                const bool ok = wait_stage(bars + cslot, cpar);
                if (!__all_sync(FULL, ok)) {
                    // a stage never landed: record it, wait (bounded) for this
                    // warp's copies still in flight, and leave
                    if (lane == 0) {
                        atomicCAS(g.err, 0, ERR_WAIT_STAGE);
                        for (uint32_t m = qc; m < pr.qi; ++m) wait_stage(bars + m % D, (m / D) & 1u);
                    }
                    __syncwarp();
                    return;
                }
                const float* st = ring + (size_t)cslot * RG::FWD;
                const float* cst = st + 3 * RG::NS * CS;
                // this lane's first cell (column j0-1) within the stage segments
                const int cz = SHOT ? l : (lane * W + 3);
                const int cc = SHOT ? 3 : (lane * W + 3);
#pragma unroll
                for (int k = 0; k < W + 2; ++k) B.en[k] = st[cz + k * CS];
#pragma unroll
                for (int k = 0; k <= W; ++k) B.hxo[k] = st[RG::NS * CS + cz + k * CS];
#pragma unroll
                for (int w = 0; w < W; ++w) B.hyo[w] = st[2 * RG::NS * CS + cz + (w + 1) * CS];
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    B.ca[w] = cst[cc + 1 + w];
                    B.cb[w] = cst[RG::NCF + cc + 1 + w];
                }
#pragma unroll
                for (int k = 0; k <= W; ++k) B.ch[k] = cst[2 * RG::NCF + cc + k];
                __syncwarp();
                ++qc;
                if (++cslot == D) {
                    cslot = 0;
                    cpar ^= 1u;
                }
                if (lane == 0) {
                    fence_proxy_async();
                    produce();
                }
            } else if (T.live && n > 0) {
                load_row(i);
            }
            if (T.live)
                fwd_row<W, CS, LEAN>(g, R, by, B, ezc, hyu, i, t, j0, l, slot, T.s, bcore, ezW, hxW, hyW, hist, hrow, rd, wr,
                               sc, se, rc, re);
        }
        cur = nxt;
        nxt = cur < nt_ ? fetch_tile(ctr, lane) : nt_;
        if (RING && lane == 0) {
            --pr.ptile;
            pr.q[0] = pr.q[1];
            pr.q[1] = tile_q<W, SHOT>(g, nxt, 0);
        }
    }
#undef FG_CELL
}

// Step kernels are launched with programmatic stream serialisation behind the
// kernel before them (the last launch of the previous step, or any other
// kernel), so their blocks take the SMs as that kernel's blocks leave: each
// waits for it to complete (griddep_wait) before it touches anything the step
// reads or writes, then lets the slab and interior kernels behind it start
// (they read none of this launch's results; see fdtd_core.cuh).
template <int W, bool SHOT, bool RING, bool LEAN = false>
__global__ void __launch_bounds__(128, 4) k_fwd(const Dev g, const int t, const int D) {
    extern __shared__ __align__(128) unsigned char smem[];
    const float* R = stage_profile(g, smem);   // the profile is fixed for the solve
    griddep_wait();
    griddep_launch_dependents();
    // a stage of an earlier launch never landed: leave at once
    if (RING && *(volatile int*)g.err != 0) return;
    fwd_step<W, SHOT, RING, LEAN>(g, R, smem, t, D);
}

// ---------------------------------------------------------------------------
// Reference-mode adjoint step
// ---------------------------------------------------------------------------
template <int W>
struct AdjEIn {                // operands of the E update of row r
    float ez[W + 1];           // Ez_old(r, j0 .. j0+W)
    float hxo[W + 2];          // Hx_old(r, j0-1 .. j0+W)
    float hyo[W + 1];          // Hy_old(r, j0 .. j0+W)
    float ca[W + 1], cb[W + 1];
};

template <int W, int CS>
__device__ __forceinline__ void adj_e_load(const Dev& g, AdjEIn<W>& A, int r, int j0, int l, const float* ezR,
                                           const float* hxR, const float* hyR) {
    const long long rb = (long long)r * g.P + j0 + PADC;
    ld_cells<W, CS>(g, A.ez, ezR + rb * CS + l);
    A.ez[W] = ldro(g, ezR + (rb + W) * CS + l);
    A.hxo[0] = ldro(g, hxR + (rb - 1) * CS + l);
    ld_cells<W, CS>(g, A.hxo + 1, hxR + rb * CS + l);
    A.hxo[W + 1] = ldro(g, hxR + (rb + W) * CS + l);
    ld_cells<W, CS>(g, A.hyo, hyR + rb * CS + l);
    A.hyo[W] = ldro(g, hyR + (rb + W) * CS + l);
    ld_coef<W + 1, CALIGN<W>>(g, A.ca, g.ca + rb);
    ld_coef<W + 1, CALIGN<W>>(g, A.cb, g.cb + rb);
}

// back_source (back.cu:34): Ez -= residual at the receivers of row r, no
// scaling, in list order: the tile's injection events of the row from ic on.
template <int W>
__device__ __forceinline__ void adj_inject(const Dev& g, float (&ez)[W + 1], int r, int j0, int slot, long long resid_o,
                                           int& ic, int ie) {
    for (; ic < ie; ++ic) {
        const Ev e = __ldg(g.inj_ev + ic);
        if (e.x != r) break;
        if (e.y != slot) continue;
#pragma unroll
        for (int k = 0; k <= W; ++k)
            if (j0 + k == e.z) ez[k] = __fsub_rn(ez[k], inj_value(g, resid_o + e.w));
    }
}

// Interior E of row r, columns j0 .. j0+W, from the old state (hyu = old Hy
// of row r-1): the E leapfrog of fields_updates_gpu.cu:8-33 with Ucgeta's uE0.
template <int W>
__device__ __forceinline__ void adj_e_core(const AdjEIn<W>& A, const float (&hyu)[W + 1], float (&out)[W + 1]) {
#pragma unroll
    for (int k = 0; k <= W; ++k)
        out[k] = __fmaf_rn(-A.cb[k], __fsub_rn(A.hxo[k + 1], A.hxo[k]),
                           madd2(A.ca[k], A.ez[k], A.cb[k], __fsub_rn(A.hyo[k], hyu[k])));
}

// New E of row r, columns j0 .. j0+W (column j0+W is the halo), from the old
// state: residuals injected first (list order), then the E update with the
// old H (hyu = Hy_old of row r-1).  Auxiliaries are stored for the thread's
// own cells when `own` (row r inside the chunk); the halo column and the halo
// row below the chunk only read theirs.
template <int W, int CS, bool LEAN = false>
__device__ __forceinline__ void adj_e_row(const Dev& g, const float* R, const BandY& by, AdjEIn<W>& A, int r, int j0,
                                          int l, int slot, bool core, bool own, const float (&hyu)[W + 1], float (&out)[W + 1],
                                          long long resid_o, int& ic, int ie, const PsiG& rd, const PsiG& wr) {
    adj_inject<W>(g, A.ez, r, j0, slot, resid_o, ic, ie);
    if (core) {
        adj_e_core<W>(A, hyu, out);
    } else if (CS == 32 && (LEAN || by.lean)) {
        if constexpr (CS == 32)
            adj_e_row_shot<W>(g, R, by, r, j0, l, own, A.ez, A.hxo, A.hyo, hyu, A.ca, A.cb, rd, wr, out);
    } else if (g.fast_cpml) {
        float dhy[W + 1], dhx[W + 1];
#pragma unroll
        for (int k = 0; k <= W; ++k) {
            out[k] = A.ez[k];
            dhy[k] = __fsub_rn(A.hyo[k], hyu[k]);
            dhx[k] = __fsub_rn(A.hxo[k + 1], A.hxo[k]);
        }
        e_cells<W + 1, CS>(g, R, r, j0, l, out, dhy, dhx, A.ca, A.cb, W, own, rd, wr);
    } else {
        const int ny = g.ny;
#pragma unroll
        for (int k = 0; k <= W; ++k) {
            const int j = j0 + k;
            out[k] = A.ez[k];
            if (j < ny) {
                const float dhy = __fsub_rn(A.hyo[k], hyu[k]);
                const float dhx = __fsub_rn(A.hxo[k + 1], A.hxo[k]);
                if (k < W && own)
                    out[k] = e_cell<CS, true>(g, R, r, j, l, A.ez[k], dhy, dhx, A.ca[k], A.cb[k], rd, wr);
                else out[k] = e_cell<CS, false>(g, R, r, j, l, A.ez[k], dhy, dhx, A.ca[k], A.cb[k], rd, rd);
            }
        }
    }
}

// Sum v[0..M) over the 32 lanes of a warp by recursive halving.  Returns, in
// every lane, the sum of element (lane >> s) & (M-1) with s = 5 - log2(M);
// lanes whose low s bits are zero hold the M distinct sums.  Fixed
// association order (deterministic).
template <int M>
__device__ __forceinline__ float lane_reduce_scatter(float (&v)[M], int lane) {
    static_assert(M == 4 || M == 8 || M == 16, "2W elements");
#pragma unroll
    for (int len = M, m = 16; len > 1; len >>= 1, m >>= 1) {
        const bool upper = (lane & m) != 0;
#pragma unroll
        for (int k = 0; k < len / 2; ++k) {
            const float send = upper ? v[k] : v[k + len / 2];
            const float keep = upper ? v[k + len / 2] : v[k];
            v[k] = __fadd_rn(keep, __shfl_xor_sync(FULL, send, m));
        }
    }
    constexpr int s = M == 4 ? 3 : (M == 8 ? 2 : 1);
    float x = v[0];
#pragma unroll
    for (int m = (1 << s) >> 1; m >= 1; m >>= 1) x = __fadd_rn(x, __shfl_xor_sync(FULL, x, m));
    return x;
}

// Interior H of row i from the new E (ezc: row i, columns j0 .. j0+W; ezr:
// row i+1) and the old H (hxc from column j0-1, hyc from j0).
template <int W>
__device__ __forceinline__ void adj_h_core(const float (&ch)[W], const float (&ezc)[W + 1], const float (&ezr)[W + 1],
                                           const float (&hxc)[W + 2], const float (&hyc)[W + 1], float (&hx)[W],
                                           float (&hy)[W]) {
#pragma unroll
    for (int w = 0; w < W; ++w) {
        hx[w] = __fsub_rn(hxc[w + 1], __fmul_rn(ch[w], __fsub_rn(ezc[w + 1], ezc[w])));
        hy[w] = __fadd_rn(hyc[w], __fmul_rn(ch[w], __fsub_rn(ezr[w], ezc[w])));
    }
}

// Imaging (compute.py:1167-1172) of row i, cells j0 .. j0+W-1, into the fp64
// accumulators at ge / gs (the row's cell j0).  sum_t (Ez_f[t] - Ez_f[t-1])
// lambda_t is summed by parts as sum_t Ez_f[t] (lambda_t - lambda_{t+1}) -
// Ez_f[0] lambda_1: lambda_{t+1} is this step's old Ez (eoc), so the history
// (f1) is read once per step; k_imaging_tail subtracts the last term.  The
// sigma sum is sum_t Ez_f[t] lambda_t dt.  Shot lanes sum the warp's 32 shots
// by a reduce-scatter first, so each cell gets one addition per launch.
template <int W, bool SHOT>
__device__ __forceinline__ void adj_image(const Dev& g, const float (&f1)[W], const float (&ezc)[W + 1],
                                          const float (&eoc)[W], double* ge, double* gs, int j0, int lane) {
    float v[2 * W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
        v[w] = __fmul_rn(f1[w], __fsub_rn(ezc[w], eoc[w]));
        v[W + w] = __fmul_rn(__fmul_rn(f1[w], ezc[w]), g.dt);
    }
    if (SHOT) {
        constexpr int s = (2 * W) == 4 ? 3 : ((2 * W) == 8 ? 2 : 1);
        const float x = lane_reduce_scatter<2 * W>(v, lane);
        if ((lane & ((1 << s) - 1)) == 0) {
            const int e = lane >> s;   // element index 0 .. 2W-1
            const int w = e < W ? e : e - W;
            if (j0 + w < g.ny) acc_add(g, (e < W ? ge : gs) + w, (double)x);
        }
    } else {
#pragma unroll
        for (int w = 0; w < W; ++w)
            if (j0 + w < g.ny) {
                acc_add(g, ge + w, (double)v[w]);
                acc_add(g, gs + w, (double)v[W + w]);
            }
    }
}

// One iteration of the reference-mode adjoint march for a thread's W cells:
// the new E of row r = i + 1 from its old operands A (own if r is inside the
// chunk [.., i1), else the halo row below; nothing when r is the frame row),
// H of row i from the new E, the imaging sums and the stores; then the
// carried rows (new E, old H and old Ez of row i) move on to row r.
template <int W, bool SHOT, bool LEAN = false>
__device__ __forceinline__ void adj_row(const Dev& g, const float* R, const BandY& by, AdjEIn<W>& A,
                                        const float (&ch)[W], const float (&f1)[W], float (&ezc)[W + 1],
                                        float (&hxc)[W + 2], float (&hyc)[W + 1], float (&eoc)[W], int i, int i1,
                                        int j0, int l, int slot, int lane, bool bcore, long long resid_o, int& ic,
                                        int ie, const PsiG& rd, const PsiG& wr, float* ezW, float* hxW, float* hyW,
                                        double* gae, double* gas) {
    constexpr int CS = SHOT ? 32 : 1;
    const int r = i + 1;
    const int P = g.P, nx = g.nx, ny = g.ny, th = g.th;
    // new E of row r (own if inside the chunk, else the halo row below)
    float ezr[W + 1], eor[W];
    if (r < nx) {
#pragma unroll
        for (int w = 0; w < W; ++w) eor[w] = A.ez[w];
        adj_e_row<W, CS, LEAN>(g, R, by, A, r, j0, l, slot, bcore && r >= th + 1 && r <= nx - th - 1, r < i1, hyc, ezr,
                         resid_o, ic, ie, rd, wr);
    } else {
#pragma unroll
        for (int w = 0; w < W; ++w) eor[w] = 0.f;
#pragma unroll
        for (int k = 0; k <= W; ++k) ezr[k] = A.hyo[k] = 0.f;
#pragma unroll
        for (int k = 0; k < W + 2; ++k) A.hxo[k] = 0.f;
    }
    // H of row i from the new E
    float hx[W], hy[W];
    if (bcore && i >= th + 1 && i <= nx - th - 1) {
        adj_h_core<W>(ch, ezc, ezr, hxc, hyc, hx, hy);
    } else if (SHOT && (LEAN || by.lean)) {
        float dzx[W], dzy[W];
#pragma unroll
        for (int w = 0; w < W; ++w) {
            hx[w] = hxc[w + 1];
            hy[w] = hyc[w];
            dzx[w] = __fsub_rn(ezc[w + 1], ezc[w]);
            dzy[w] = __fsub_rn(ezr[w], ezc[w]);
        }
        if constexpr (SHOT) adj_h_row_shot<W>(g, R, by, i, j0, l, hx, hy, dzx, dzy, ch, rd, wr);
    } else if (g.fast_cpml) {
        float dzx[W], dzy[W];
#pragma unroll
        for (int w = 0; w < W; ++w) {
            hx[w] = hxc[w + 1];
            hy[w] = hyc[w];
            dzx[w] = __fsub_rn(ezc[w + 1], ezc[w]);
            dzy[w] = __fsub_rn(ezr[w], ezc[w]);
        }
        hx_cells<W, CS>(g, R, i, j0, l, hx, dzx, ch, 0, rd, wr);
        hy_cells<W, CS, true>(g, R, i, j0, l, hy, dzy, ch, rd, wr);
    } else {
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const int j = j0 + w;
            hx[w] = hxc[w + 1];
            hy[w] = hyc[w];
            if (j < ny) {
                hx[w] = hx_cell<CS, true>(g, R, i, j, l, hxc[w + 1], __fsub_rn(ezc[w + 1], ezc[w]), ch[w], rd,
                                          wr);
                hy[w] = hy_cell<CS, true>(g, R, i, j, l, hyc[w], __fsub_rn(ezr[w], ezc[w]), ch[w], rd, wr);
            }
        }
    }
    const long long go2 = (long long)i * ny + j0;
    adj_image<W, SHOT>(g, f1, ezc, eoc, gae + go2, gas + go2, j0, lane);
    const long long o = ((long long)i * P + j0 + PADC) * CS + l;
    st_cells<W, CS>(g, ezW + o, ezc);
    st_cells<W, CS>(g, hxW + o, hx);
    st_cells<W, CS>(g, hyW + o, hy);
#pragma unroll
    for (int k = 0; k <= W; ++k) {
        ezc[k] = ezr[k];
        hyc[k] = A.hyo[k];
    }
#pragma unroll
    for (int w = 0; w < W; ++w) eoc[w] = eor[w];
#pragma unroll
    for (int k = 0; k < W + 2; ++k) hxc[k] = A.hxo[k];
}

// Stage of adjoint iteration i of tile Q: E operands of row r = i+1 (Ez_old,
// Hx_old, Hy_old, uE0, uE1; none when r is the frame row), uH1 of row i and
// the forward Ez of step it at row i.
template <int W, bool SHOT>
__device__ __forceinline__ void issue_adj(const Dev& g, uint64_t* bar, float* st, const TileQ& Q, int i, int rp) {
    using RG = RingGeom<W, SHOT>;
    constexpr int CS = RG::CS;
    // shot-lane stages hold exactly the cells used: Ez, Hy from j0, Hx from j0-1
    constexpr uint32_t zs = (uint32_t)(SHOT ? (W + 1) : RG::NS) * CS * 4;
    constexpr uint32_t xs = (uint32_t)(SHOT ? (W + 2) : RG::NS) * CS * 4;
    constexpr uint32_t cs = (uint32_t)RG::NCF * 4;
    constexpr int zo = SHOT ? CS : 0;
    const int r = i + 1;
    const bool erow = r < g.nx;
    const long long rowS = (long long)g.P * CS;
    const long long so = Q.sbase + (long long)r * rowS;
    const long long co = Q.cbase + (long long)r * g.P;
    const float* h1 = g.hist + Q.hbase + (long long)i * g.Ph * CS;
    float* hst = st + 3 * RG::NS * CS;
    float* cst = hst + RG::NH * CS;
    issue_stage(g, bar, [&](auto&& f) {
        if (erow) {
            f(st + zo, g.ez[rp] + so + zo, zs);
            f(st + RG::NS * CS, g.hx[rp] + so, xs);
            f(st + 2 * RG::NS * CS + zo, g.hy[rp] + so + zo, zs);
            f(cst, g.ca + co, cs);
            f(cst + RG::NCF, g.cb + co, cs);
        }
        f(cst + 2 * RG::NCF, g.ch + Q.cbase + (long long)i * g.P, cs);
        f(hst, h1, Q.hs);
    });
}

// Reference-mode adjoint iteration it (reading parity rp) of one solve by the
// warps of this block; R and smem as for fwd_step.
template <int W, bool SHOT, bool RING, bool LEAN = false>
__device__ __forceinline__ void adj_step(const Dev& g, const float* R, unsigned char* smem, const int it, const int rp,
                                         const int D) {
    constexpr int CS = SHOT ? 32 : 1;
    using RG = RingGeom<W, SHOT>;
    if (blockIdx.x == 0 && threadIdx.x == 0) g.tile_ctr[rp ^ 1] = 0;   // the next launch's counter
    int* ctr = g.tile_ctr + rp;
    const int lane = threadIdx.x & 31;
    const int P = g.P, nx = g.nx, ny = g.ny, th = g.th, nt_ = g.ntiles;
    const int wp = rp ^ 1;
    const long long hrow = (long long)g.Ph * CS;

    uint64_t* bars = nullptr;
    float* ring = nullptr;
    if (RING) {
        const int wib = threadIdx.x >> 5;
        unsigned char* base = smem + prof_bytes(th);
        bars = reinterpret_cast<uint64_t*>(base) + (size_t)wib * D;
        ring = reinterpret_cast<float*>(base + ring_bar_bytes(blockDim.x >> 5, D)) + (size_t)wib * D * RG::ADJ;
        if (lane == 0) {
            for (int d = 0; d < D; ++d) mbar_init(bars + d, 1);
            fence_mbar_init();
        }
        __syncwarp();
    }
    int cur = fetch_tile(ctr, lane);
    int nxt = cur < nt_ ? fetch_tile(ctr, lane) : nt_;
    RingProducer pr;
    uint32_t qc = 0;
    int cslot = 0;
    uint32_t cpar = 0;
    if (RING && lane == 0) {
        pr.q[0] = tile_q<W, SHOT>(g, cur, it);
        pr.q[1] = tile_q<W, SHOT>(g, nxt, it);
    }
    auto produce = [&]() {
        while ((int)(pr.qi - qc) < D && pr.ptile <= 1) {
            const TileQ& Q = pr.q[pr.ptile];
            if (Q.i1 <= Q.i0) break;
            issue_adj<W, SHOT>(g, bars + pr.slot, ring + (size_t)pr.slot * RG::ADJ, Q, Q.i0 + pr.prow, rp);
            ++pr.qi;
            if (++pr.slot == D) pr.slot = 0;
            if (++pr.prow >= Q.i1 - Q.i0) {
                ++pr.ptile;
                pr.prow = 0;
            }
        }
    };

    while (cur < nt_) {
        const LaneTile<SHOT> T = decode_tile<W, SHOT>(g, __ldg(g.order + cur), lane);
        if (RING && lane == 0) produce();
        if (SHOT && !RING && g.pf == 1) prefetch_tile_shot<W>(g, nxt, rp, lane, g.hist, it);
        const int l = T.l, j0 = T.j0, slot = SHOT ? l : 0;
        // column lanes without cells only take part in the warp's stage protocol
        const bool work = SHOT || T.live;
        const long long go = (long long)T.grp * g.plane;
        const float* ezR = g.ez[rp] + go;
        const float* hxR = g.hx[rp] + go;
        const float* hyR = g.hy[rp] + go;
        float* ezW = g.ez[wp] + go;
        float* hxW = g.hx[wp] + go;
        float* hyW = g.hy[wp] + go;
        const PsiG rd = psi_group(g, rp, T.grp), wr = psi_group(g, wp, T.grp);
        // E at columns j0 .. j0+W (incl. the halo) and H at j0 .. j0+W-1 are interior cells
        const bool bcore = j0 >= th + 1 && j0 + W <= ny - th - 1;
        BandY by{};
        if constexpr (SHOT) by = band_adj<W>(g, j0);
        int ic = __ldg(g.inj_off + T.id);
        const int ie = __ldg(g.inj_off + T.id + 1);
        const long long resid_o = ((long long)T.s * g.nt + it) * g.nrx;
        const float* f1g = g.hist + ((long long)(it - g.hist_t0) * g.ngroups + T.grp) * nx * hrow + (long long)j0 * CS + l;
        double* gae = g.gacc + (long long)T.grp * 2 * ((long long)nx * ny);
        double* gas = gae + (long long)nx * ny;
        const bool hist_ok = j0 < g.Ph;

        // new E of row i0 (own), with the old H of rows i0-1 and i0; eoc keeps
        // the old Ez of the row (before the residual injection)
        float ezc[W + 1], hxc[W + 2], hyc[W + 1], eoc[W];
        if (work) {
            float hyu[W + 1];
#pragma unroll
            for (int k = 0; k <= W; ++k) hyu[k] = 0.f;
            if (T.i0 >= 1) {
                const long long rb = (long long)(T.i0 - 1) * P + j0 + PADC;
                ld_cells<W, CS>(g, hyu, hyR + rb * CS + l);
                hyu[W] = ldro(g, hyR + (rb + W) * CS + l);
            }
            AdjEIn<W> A;
            adj_e_load<W, CS>(g, A, T.i0, j0, l, ezR, hxR, hyR);
#pragma unroll
            for (int w = 0; w < W; ++w) eoc[w] = A.ez[w];
            adj_e_row<W, CS, LEAN>(g, R, by, A, T.i0, j0, l, slot, bcore && T.i0 >= th + 1 && T.i0 <= nx - th - 1, true, hyu,
                             ezc, resid_o, ic, ie, rd, wr);
#pragma unroll
            for (int k = 0; k < W + 2; ++k) hxc[k] = A.hxo[k];
#pragma unroll
            for (int k = 0; k <= W; ++k) hyc[k] = A.hyo[k];
        }

        const int nrow = T.i1 - T.i0;
        for (int n = 0; n < nrow; ++n) {
            const int i = T.i0 + n, r = i + 1;
            if (SHOT && !RING && g.pf == 2 && n == nrow / 2) prefetch_tile_shot<W>(g, nxt, rp, lane, g.hist, it);
            AdjEIn<W> A;
            float ch[W], f1[W];
            if (RING) {
                const bool ok = wait_stage(bars + cslot, cpar);
                if (!__all_sync(FULL, ok)) {
                    if (lane == 0) {
                        atomicCAS(g.err, 0, ERR_WAIT_STAGE);
                        for (uint32_t m = qc; m < pr.qi; ++m) wait_stage(bars + m % D, (m / D) & 1u);
                    }
                    __syncwarp();
                    return;
                }
                const float* st = ring + (size_t)cslot * RG::ADJ;
                const float* hst = st + 3 * RG::NS * CS;
                const float* cst = hst + RG::NH * CS;
                const int cz = SHOT ? l : (lane * W + 3);   // column j0-1
                const int cc = SHOT ? 3 : (lane * W + 3);
                if (r < nx) {
#pragma unroll
                    for (int k = 0; k <= W; ++k) {
                        A.ez[k] = st[cz + (k + 1) * CS];
                        A.hyo[k] = st[2 * RG::NS * CS + cz + (k + 1) * CS];
                        A.ca[k] = cst[cc + 1 + k];
                        A.cb[k] = cst[RG::NCF + cc + 1 + k];
                    }
#pragma unroll
                    for (int k = 0; k < W + 2; ++k) A.hxo[k] = st[RG::NS * CS + cz + k * CS];
                }
                const int hz = SHOT ? l : lane * W;   // column j0 within the history segment
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    ch[w] = cst[2 * RG::NCF + cc + 1 + w];
                    f1[w] = hist_ok ? hst[hz + w * CS] : 0.f;
                }
                __syncwarp();
                ++qc;
                if (++cslot == D) {
                    cslot = 0;
                    cpar ^= 1u;
                }
                if (lane == 0) {
                    fence_proxy_async();
                    produce();
                }
                if (!work) continue;
            } else {
                if (!work) continue;
                if (r < nx) adj_e_load<W, CS>(g, A, r, j0, l, ezR, hxR, hyR);
                ld_coef<W, CALIGN<W>>(g, ch, g.ch + coef_at(g, i, j0));
                if (hist_ok) {
                    ld_cells<W, CS>(g, f1, f1g + (long long)i * hrow);
                } else {
#pragma unroll
                    for (int w = 0; w < W; ++w) f1[w] = 0.f;
                }
            }
            adj_row<W, SHOT, LEAN>(g, R, by, A, ch, f1, ezc, hxc, hyc, eoc, i, T.i1, j0, l, slot, lane, bcore, resid_o, ic, ie, rd,
                             wr, ezW, hxW, hyW, gae, gas);
        }
        cur = nxt;
        nxt = cur < nt_ ? fetch_tile(ctr, lane) : nt_;
        if (RING && lane == 0) {
            --pr.ptile;
            pr.q[0] = pr.q[1];
            pr.q[1] = tile_q<W, SHOT>(g, nxt, it);
        }
    }
}

template <int W, bool SHOT, bool RING, bool LEAN = false>
__global__ void __launch_bounds__(128, 3) k_adj(const Dev g, const int it, const int rp, const int D) {
    extern __shared__ __align__(128) unsigned char smem[];
    const float* R = stage_profile(g, smem);
    griddep_wait();   // as k_fwd
    griddep_launch_dependents();
    if (RING && *(volatile int*)g.err != 0) return;
    adj_step<W, SHOT, RING, LEAN>(g, R, smem, it, rp, D);
}

// The last term of the summation by parts: g_eps -= sum_s Ez_f[0] lambda_1,
// with lambda_1 the adjoint Ez after the last step (it = 1).  One thread per
// (group, cell); the products are those of the per-step imaging (float32),
// summed over the group's shots in slot order.
template <int CS>
__global__ void k_imaging_tail(const Dev g, const float* __restrict__ ez_final) {
    const long long n = (long long)g.nx * g.ny;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)g.ngroups * n) return;
    const int grp = (int)(idx / n);
    const long long c = idx % n;
    const int i = (int)(c / g.ny), j = (int)(c % g.ny);
    const float* f0 = g.hist + ((((long long)(0 - g.hist_t0) * g.ngroups + grp) * g.nx + i) * g.Ph + j) * CS;
    const float* lam = ez_final + (long long)grp * g.plane + ((long long)i * g.P + j + PADC) * CS;
    float acc = 0.f;
#pragma unroll 8
    for (int l = 0; l < CS; ++l) acc = __fadd_rn(acc, __fmul_rn(__ldg(f0 + l), __ldg(lam + l)));
    double* a = g.gacc + (long long)grp * 2 * n + c;
    *a -= (double)acc;
}

}  // namespace fg
