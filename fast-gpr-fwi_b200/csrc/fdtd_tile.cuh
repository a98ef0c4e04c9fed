// Tensor-map tile pipelines: one launch per time step; persistent CTAs, each
// with R consumer warps and one producer warp.
//
// Tile = (column band, row chunk [i0, i0+R), shot group).  The producer's lane
// 0 fetches every operand of a tile -- the old Ez/Hx/Hy rows with a one-cell
// halo, the coefficient rows, and in the adjoint the stored forward Ez rows --
// with one cp.async.bulk.tensor copy per field (a box of 32 shots x cells x
// rows, or cells x rows for one shot) into one of S shared-memory stages,
// completing on the stage's "full" mbarrier; it runs up to S tiles ahead of
// the consumers and reuses a stage once its "empty" mbarrier has one arrival
// per consumer warp.  Rows and columns outside the field arrays are filled
// with zeros by the copy engine, which is the reference's zero frame.  Each
// consumer warp computes one row of the tile from the stage and writes the
// new state (and new CPML auxiliaries) straight to global memory.  Everything
// a CTA reads comes from the previous step's buffers (ping-pong), so CTAs
// never wait on each other.  A CTA takes tiles blockIdx.x, blockIdx.x +
// gridDim.x, ... of the tile table (CPML-heavy tiles first).  Every wait is
// bounded (2 s): a stage that never lands sets the device error word, the
// consumers agree to stop (one barrier with an AND reduction), wait (bounded)
// for the stages that may still be landing, and leave; later launches of the
// solve return at once.
//
//   shot lanes   (SHOT = true):  lane l is shot slot l of the group (CS = 32);
//                all lanes of a warp touch the same cells, coefficients are
//                warp-uniform and every boundary branch is uniform.
//   column lanes (SHOT = false): one shot per group (CS = 1); lane l owns
//                columns b0 + l*W .. b0 + l*W + W-1.
//
// Forward step t (src/compute.py:574-712), per row i: Hy of row i-1 (the halo
// row, recomputed), Hx (columns j0-1 .. j0+W-1) and Hy of row i, then Ez, the
// CPML corrections of each, the source injection, the stores, the Ez history
// and the receiver samples (trace[t+1] = Ez after step t, which is what the
// reference's store_outputs reads at the start of step t+1).
//
// Reference-mode adjoint step (src/compute.py:1048-1172): residual injection
// at the receivers and the E update (Ucgeta's uE0) of rows i0 .. i0+R (the
// last one is the halo row below) from the old H into shared memory, one CTA
// barrier, then H of each row from the new E and the imaging sums with the
// stored forward Ez; the products of a warp's 32 shots are summed by a
// reduce-scatter over the lanes and added to the group's fp64 accumulator.
#pragma once

#include <cuda.h>

#include "fdtd_common.cuh"
#include "fdtd_lanes.cuh"

namespace fg {

// Box geometry of a tile, in cells (SHOT: per shot slot row of 32 floats).
template <int W, bool SHOT>
struct TileGeom {
    static constexpr int CS = SHOT ? 32 : 1;
    static constexpr int BW = SHOT ? W : 32 * W;   // columns of a band
    // column windows (first column relative to j0 - 1 in shot lanes, b0 - 4 in column lanes)
    static constexpr int NWIN = SHOT ? 0 : BW + 8;
    // forward boxes: Ez rows i0-1 .. i0+R, cols j0-1 .. j0+W; Hx rows i0 .. i0+R-1, cols j0-1 ..
    // j0+W-1; Hy rows i0-1 .. i0+R-1, cols j0 .. j0+W-1
    static constexpr int FEZ = SHOT ? W + 2 : NWIN;
    static constexpr int FHX = SHOT ? W + 1 : NWIN;
    static constexpr int FHY = SHOT ? W : NWIN;
    // adjoint boxes: Ez rows i0 .. i0+R, cols j0 .. j0+W; Hx rows i0 .. i0+R, cols j0-1 .. j0+W;
    // Hy rows i0-1 .. i0+R, cols j0 .. j0+W; forward Ez rows i0 .. i0+R-1, cols j0 .. j0+W-1
    static constexpr int AEZ = SHOT ? W + 1 : NWIN;
    static constexpr int AHX = SHOT ? W + 2 : NWIN;
    static constexpr int AHY = SHOT ? W + 1 : NWIN;
    static constexpr int AH = BW;
    static constexpr int NCF = BW + 8;   // coefficient columns b0-4 .. b0+BW+3
};

__host__ __device__ inline size_t align128(size_t x) { return (x + 127) / 128 * 128; }

// Shared-memory layout of one stage (bytes), R rows; the CTA holds S stages.
template <int W, bool SHOT>
struct TileSmem {
    using G = TileGeom<W, SHOT>;
    size_t ez, hx, hy, co, hs, en, total;
    __host__ __device__ TileSmem(int R, bool adjoint) {
        const size_t cs = G::CS * sizeof(float);
        size_t o = 128;   // header: tile (b0, i0, group, id) and its event-list offsets
        ez = o;
        o = align128(o + (adjoint ? (size_t)G::AEZ * (R + 1) : (size_t)G::FEZ * (R + 2)) * cs);
        hx = o;
        o = align128(o + (adjoint ? (size_t)G::AHX * (R + 1) : (size_t)G::FHX * R) * cs);
        hy = o;
        o = align128(o + (adjoint ? (size_t)G::AHY * (R + 2) : (size_t)G::FHY * (R + 1)) * cs);
        co = o;
        o = align128(o + (size_t)G::NCF * (R + 1) * 5 * sizeof(float));
        hs = o;
        if (adjoint) o = align128(o + (size_t)G::AH * R * cs);
        en = o;
        if (adjoint) o = align128(o + (size_t)(SHOT ? W + 1 : G::NWIN) * (R + 1) * cs);
        total = o;
    }
    // bytes the copies of one stage deliver
    __host__ __device__ static uint32_t tx_bytes(int R, bool adjoint) {
        const size_t cs = G::CS * sizeof(float);
        size_t b = (size_t)G::NCF * (R + 1) * 5 * sizeof(float);
        if (adjoint)
            b += ((size_t)G::AEZ * (R + 1) + (size_t)G::AHX * (R + 1) + (size_t)G::AHY * (R + 2) + (size_t)G::AH * R) *
                 cs;
        else b += ((size_t)G::FEZ * (R + 2) + (size_t)G::FHX * R + (size_t)G::FHY * (R + 1)) * cs;
        return (uint32_t)b;
    }
};

// Stage header written by the producer (generic stores before it arms the
// stage's barrier, so they are visible to the consumers after their wait).
struct StageHead {
    int4 tile;   // b0, i0, group, id
    int4 ev;     // forward: source and receiver event ranges; adjoint: injection range
};

// Whole-CTA layout: barriers and flags, CPML profile, S stages.
constexpr int MAX_STAGES = 4;
struct PipeSmem {
    size_t full, empty, flag, prof, stages, stage_bytes, total;
    __host__ __device__ PipeSmem(int th, int S, size_t stage) {
        full = 0;
        empty = 8 * MAX_STAGES;
        flag = 16 * MAX_STAGES;   // [0] launch-abort copy of the error word, [1] this CTA gave up
        prof = 128;
        stages = align128(prof + (size_t)8 * th * sizeof(float));
        stage_bytes = stage;
        total = stages + (size_t)S * stage;
    }
};

// cp.async.bulk.tensor loads (tile mode, no multicast) of a box at the given
// coordinates, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* tm, int c0, int c1, int c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(tm), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* tm, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(tm), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* tm, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5, %6}], [%7];" ::"r"(smem_u32(dst)),
        "l"(tm), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}

// A state box: field f (0 Ez, 1 Hx, 2 Hy) of parity par, first column `col`
// (plane column, pad included) and first row `row` of group grp.
template <bool SHOT>
__device__ __forceinline__ void tma_state(void* dst, const CUtensorMap* tm, int col, int row, int grp, int f, int par,
                                          uint64_t* bar) {
    if (SHOT) tma_load_5d(dst, tm, 0, col, row, grp, 2 * f + par, bar);
    else tma_load_4d(dst, tm, col, row, grp, 2 * f + par, bar);
}

// Whether an earlier launch recorded a stage that never landed; read by
// thread 0 and shared through shared memory, so the whole CTA takes the same
// branch.
__device__ __forceinline__ bool abort_launch(const Dev& g, volatile int* flag) {
    if (threadIdx.x == 0) *flag = *(volatile int*)g.err;
    __syncthreads();
    return *flag != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void consumers_sync(int nthreads) {
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

// Bounded wait that gives up at once when the CTA has given up (`stop`); a
// wait that runs out sets `stop` and the device error word.
__device__ __forceinline__ bool wait_or_stop(const Dev& g, uint64_t* bar, uint32_t parity, volatile int* stop) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    while (!mbar_try_wait(bar, parity)) {
        if (*stop) return false;
        if (globaltimer() - t0 > WAIT_LIMIT_NS) {
            *stop = 1;
            atomicCAS(g.err, 0, ERR_WAIT_STAGE);
            return false;
        }
        __nanosleep(20);
    }
    return true;
}

// Producer loop (lane 0 of warp R): for the CTA's k-th tile, wait until stage
// k % S is free, write its header, arm its full barrier and issue the tile's
// copies.  Before leaving it waits (bounded) for the stages it issued, so no
// copy is still landing when the CTA retires.
template <class Issue>
__device__ __forceinline__ void produce_tiles(const Dev& g, uint64_t* full, uint64_t* empty, int S, volatile int* stop,
                                              Issue&& issue) {
    int s = 0;
    int k = 0;
    for (int p = blockIdx.x; p < g.ntiles; p += gridDim.x, ++k) {
        // the u-th reuse of a stage (u = k / S >= 1) waits for completion u-1
        // of its empty barrier
        if (k >= S && !wait_or_stop(g, empty + s, (uint32_t)(k / S + 1) & 1u, stop)) break;
        issue(p, s, full + s);
        if (++s == S) s = 0;
    }
    // the last min(k, S) issued stages: tiles k-S .. k-1
    for (int m = k - S < 0 ? 0 : k - S; m < k; ++m) wait_stage(full + (m % S), (uint32_t)(m / S) & 1u);
}

// ---------------------------------------------------------------------------
// Forward step
// ---------------------------------------------------------------------------
template <int W, bool SHOT>
__device__ __forceinline__ void fwd_tile_issue(const Dev& g, const CUtensorMap* tm_ez, const CUtensorMap* tm_hx,
                                               const CUtensorMap* tm_hy, const CUtensorMap* tm_co, unsigned char* st,
                                               const TileSmem<W, SHOT>& L, int R, int p, int rp, uint64_t* bar) {
    const int4 T = __ldg(g.tiles + p);
    const int b0 = T.x, i0 = T.y, grp = T.z;
    StageHead* h = reinterpret_cast<StageHead*>(st);
    h->tile = T;
    h->ev = make_int4(__ldg(g.src_off + T.w), __ldg(g.src_off + T.w + 1), __ldg(g.rx_off + T.w),
                      __ldg(g.rx_off + T.w + 1));
    mbar_expect_tx(bar, TileSmem<W, SHOT>::tx_bytes(R, false));
    const int cs = (SHOT ? b0 - 1 : b0 - 4) + PADC;   // first state column
    tma_state<SHOT>(st + L.ez, tm_ez, cs, i0 - 1, grp, 0, rp, bar);
    tma_state<SHOT>(st + L.hx, tm_hx, cs, i0, grp, 1, rp, bar);
    tma_state<SHOT>(st + L.hy, tm_hy, SHOT ? cs + 1 : cs, i0 - 1, grp, 2, rp, bar);
    tma_load_3d(st + L.co, tm_co, b0 - 4 + PADC, i0 - 1, 0, bar);
    prefetch_tile_psi<TileGeom<W, SHOT>::CS>(g, grp, rp, i0 - 1, i0 + R - 1, b0 - 1, b0 + TileGeom<W, SHOT>::BW - 1);
}

// Rows i0 + w*M .. i0 + w*M + M-1 of the stage's tile (R rows).
template <int W, bool SHOT>
__device__ __forceinline__ void fwd_tile_rows(const Dev& g, const float* Rp, const unsigned char* st,
                                              const TileSmem<W, SHOT>& L, int R, int w, int M, int t) {
    const StageHead* hd = reinterpret_cast<const StageHead*>(st);
    const int4 T = hd->tile;
    const int4 E = hd->ev;
    using G = TileGeom<W, SHOT>;
    constexpr int CS = G::CS;
    const float* sEZ = reinterpret_cast<const float*>(st + L.ez);
    const float* sHX = reinterpret_cast<const float*>(st + L.hx);
    const float* sHY = reinterpret_cast<const float*>(st + L.hy);
    const float* sCO = reinterpret_cast<const float*>(st + L.co);
    const int b0 = T.x, i0 = T.y, grp = T.z;
    const int rp = t & 1, wp = rp ^ 1;
    const int lane = threadIdx.x & 31;
    const int rr0 = w * M;
    const int ifirst = i0 + rr0;
    const int nx = g.nx, ny = g.ny, th = g.th;
    const int l = SHOT ? lane : 0;
    const int j0 = SHOT ? b0 : b0 + lane * W;
    if (ifirst >= nx || (!SHOT && j0 >= ny)) return;
    const int slot = SHOT ? lane : 0;
    const int s = SHOT ? grp * 32 + lane : grp;
    const long long go = (long long)grp * g.plane;
    const PsiG rd = psi_group(g, rp, grp), wr = psi_group(g, wp, grp);
    BandY by{};
    if constexpr (SHOT) by = band_fwd<W>(g, j0);
    // column index of j0-1 within the boxes: Ez and Hx start at j0-1 (shot
    // lanes) or b0-4 (column lanes); Hy one column later in shot lanes
    const int cz = SHOT ? 0 : lane * W + 3;
    const int cy = SHOT ? -1 : lane * W + 3;
    const int cc = SHOT ? 3 : lane * W + 3;   // coefficient column of j0-1
#define EZS(r, k) sEZ[((r) * G::FEZ + cz + (k)) * CS + l]
#define HXS(r, k) sHX[((r) * G::FHX + cz + (k)) * CS + l]
#define HYS(r, k) sHY[((r) * G::FHY + cy + (k)) * CS + l]
#define COS(p, r, k) sCO[((p) * (R + 1) + (r)) * G::NCF + cc + (k)]
    // box rows: Ez, Hy, coefficients start at i0-1 (index rr+1 = row i0+rr); Hx at i0
    float ezc[W + 2], hyu[W];
#pragma unroll
    for (int k = 0; k < W + 2; ++k) ezc[k] = EZS(rr0 + 1, k);
    // new Hy of row ifirst-1 (its auxiliaries are only read)
#pragma unroll
    for (int q = 0; q < W; ++q) hyu[q] = 0.f;
    if (ifirst >= 1) {
        float ha[W], dz[W], chu[W];
#pragma unroll
        for (int q = 0; q < W; ++q) {
            ha[q] = HYS(rr0, q + 1);
            chu[q] = COS(3, rr0, q + 1);
            dz[q] = __fsub_rn(ezc[q + 1], EZS(rr0, q + 1));
            hyu[q] = ha[q];
        }
        const int iu = ifirst - 1;
        const bool xcore = iu >= th && iu <= nx - th - 1;
        if (xcore && j0 >= 1 && j0 + W <= ny) {
#pragma unroll
            for (int q = 0; q < W; ++q) hyu[q] = __fadd_rn(ha[q], __fmul_rn(chu[q], dz[q]));
        } else if (SHOT && by.lean) {
            if constexpr (SHOT) fwd_hy_halo_shot<W>(g, Rp, by, iu, j0, l, hyu, dz, chu, rd);
        } else if (g.fast_cpml) {
            hy_cells<W, CS, false>(g, Rp, iu, j0, l, hyu, dz, chu, rd, rd);
        } else {
#pragma unroll
            for (int q = 0; q < W; ++q)
                if (j0 + q < ny) hyu[q] = hy_cell<CS, false>(g, Rp, iu, j0 + q, l, ha[q], dz[q], chu[q], rd, rd);
        }
    }
    const bool bcore = j0 >= th + 1 && j0 + W <= ny - th;
    int sc = E.x;
    const int se = E.y;
    int rc = E.z;
    const int re = E.w;
    // skip the events of the rows above this warp's rows
    while (sc < se && __ldg(g.src_ev + sc).x < ifirst) ++sc;
    while (rc < re && __ldg(g.rx_ev + rc).x < ifirst) ++rc;
    const long long hrow = (long long)g.Ph * CS;
    float* hist = g.hist ? g.hist + (((long long)(t - g.hist_t0) * g.ngroups + grp) * nx) * hrow + (long long)j0 * CS + l
                             : nullptr;
    float* ezW = g.ez[wp] + go;
    float* hxW = g.hx[wp] + go;
    float* hyW = g.hy[wp] + go;
    for (int m = 0; m < M; ++m) {
        const int rr = rr0 + m, i = i0 + rr;
        if (i >= nx) break;
        FwdIn<W> B;
#pragma unroll
        for (int k = 0; k < W + 2; ++k) B.en[k] = EZS(rr + 2, k);
#pragma unroll
        for (int k = 0; k <= W; ++k) {
            B.hxo[k] = HXS(rr, k);
            B.ch[k] = COS(3, rr + 1, k);
        }
#pragma unroll
        for (int q = 0; q < W; ++q) {
            B.hyo[q] = HYS(rr + 1, q + 1);
            B.ca[q] = COS(0, rr + 1, q + 1);
            B.cb[q] = COS(1, rr + 1, q + 1);
        }
        fwd_row<W, CS>(g, Rp, by, B, ezc, hyu, i, t, j0, l, slot, s, bcore, ezW, hxW, hyW, hist, hrow, rd, wr, sc, se, rc,
                       re);
    }
#undef EZS
#undef HXS
#undef HYS
#undef COS
}

template <int W, bool SHOT>
__global__ void __launch_bounds__(288) k_fwd_pipe(const Dev g, const __grid_constant__ CUtensorMap tm_ez,
                                                  const __grid_constant__ CUtensorMap tm_hx,
                                                  const __grid_constant__ CUtensorMap tm_hy,
                                                  const __grid_constant__ CUtensorMap tm_co, const int t,
                                                  const int S, const int R) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int NW = (blockDim.x >> 5) - 1;   // consumer warps; warp NW produces
    const int Mrows = R / NW;               // rows per consumer warp (R rows per tile)
    const TileSmem<W, SHOT> L(R, false);
    const PipeSmem M(g.th, S, L.total);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + M.full);
    uint64_t* empty = reinterpret_cast<uint64_t*>(smem + M.empty);
    float* Rp = reinterpret_cast<float*>(smem + M.prof);
    volatile int* flags = reinterpret_cast<volatile int*>(smem + M.flag);
    // launched with programmatic stream serialisation behind the previous
    // step: wait for it before anything of the solve is read, then let the
    // next step's launch place its blocks as these leave
    griddep_wait();
    griddep_launch_dependents();
    if (abort_launch(g, flags)) return;
    if (threadIdx.x == 0) {
        flags[1] = 0;
        for (int s = 0; s < S; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, NW);
        }
        fence_mbar_init();
    }
    for (int k = threadIdx.x; k < 8 * g.th; k += blockDim.x) Rp[k] = __ldg(g.pml + k);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rp = t & 1;
    if (warp == NW) {
        if (lane == 0)
            produce_tiles(g, full, empty, S, flags + 1, [&](int p, int s, uint64_t* bar) {
                fwd_tile_issue<W, SHOT>(g, &tm_ez, &tm_hx, &tm_hy, &tm_co, smem + M.stages + (size_t)s * L.total, L, R,
                                        p, rp, bar);
            });
        return;
    }
    int s = 0;
    uint32_t par = 0;
    for (int p = blockIdx.x; p < g.ntiles; p += gridDim.x) {
        // after a stage that never landed every wait returns at once and the
        // tiles are skipped; the error word reports it
        if (wait_or_stop(g, full + s, par, flags + 1))
            fwd_tile_rows<W, SHOT>(g, Rp, smem + M.stages + (size_t)s * L.total, L, R, warp, Mrows, t);
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + s);
        if (++s == S) {
            s = 0;
            par ^= 1u;
        }
    }
}

// ---------------------------------------------------------------------------
// Reference-mode adjoint step
// ---------------------------------------------------------------------------
template <int W, bool SHOT>
__device__ __forceinline__ void adj_tile_issue(const Dev& g, const CUtensorMap* tm_ez, const CUtensorMap* tm_hx,
                                               const CUtensorMap* tm_hy, const CUtensorMap* tm_co,
                                               const CUtensorMap* tm_h, unsigned char* st,
                                               const TileSmem<W, SHOT>& L, int R, int p, int rp, int it,
                                               uint64_t* bar) {
    const int4 T = __ldg(g.tiles + p);
    const int b0 = T.x, i0 = T.y, grp = T.z;
    StageHead* h = reinterpret_cast<StageHead*>(st);
    h->tile = T;
    h->ev = make_int4(__ldg(g.inj_off + T.w), __ldg(g.inj_off + T.w + 1), 0, 0);
    mbar_expect_tx(bar, TileSmem<W, SHOT>::tx_bytes(R, true));
    const int cs = (SHOT ? b0 - 1 : b0 - 4) + PADC;
    tma_state<SHOT>(st + L.ez, tm_ez, SHOT ? cs + 1 : cs, i0, grp, 0, rp, bar);
    tma_state<SHOT>(st + L.hx, tm_hx, cs, i0, grp, 1, rp, bar);
    tma_state<SHOT>(st + L.hy, tm_hy, SHOT ? cs + 1 : cs, i0 - 1, grp, 2, rp, bar);
    tma_load_3d(st + L.co, tm_co, b0 - 4 + PADC, i0, 0, bar);
    const int hz = (it - g.hist_t0) * g.ngroups + grp;
    if (SHOT) tma_load_4d(st + L.hs, tm_h, 0, b0, i0, hz, bar);
    else tma_load_3d(st + L.hs, tm_h, b0, i0, hz, bar);
    prefetch_tile_psi<TileGeom<W, SHOT>::CS>(g, grp, rp, i0, i0 + R, b0, b0 + TileGeom<W, SHOT>::BW);
}

// Box column indices of one lane: j0 within the Ez/Hy/new-E boxes, j0-1 within
// the Hx box, j0-1 within the coefficient box.
template <int W, bool SHOT>
struct AdjCols {
    int c0, cx, cc;
    __device__ __forceinline__ AdjCols(int lane) {
        c0 = SHOT ? 0 : lane * W + 4;
        cx = SHOT ? 0 : lane * W + 3;
        cc = SHOT ? 3 : lane * W + 3;
    }
};

// Phase 1: new E of rows i0 .. i0+R (row i0+R is the halo row below) into the
// stage's new-E rows; warp w takes row i0+w, warp 0 also the halo row.
template <int W, bool SHOT>
__device__ __forceinline__ void adj_tile_e(const Dev& g, const float* Rp, unsigned char* st,
                                           const TileSmem<W, SHOT>& L, int R, int w, int M, int it, int rp) {
    const StageHead* hd = reinterpret_cast<const StageHead*>(st);
    const int4 T = hd->tile;
    const int4 E = hd->ev;
    using G = TileGeom<W, SHOT>;
    constexpr int CS = G::CS;
    constexpr int NE = SHOT ? W + 1 : G::NWIN;
    const float* sEZ = reinterpret_cast<const float*>(st + L.ez);
    const float* sHX = reinterpret_cast<const float*>(st + L.hx);
    const float* sHY = reinterpret_cast<const float*>(st + L.hy);
    const float* sCO = reinterpret_cast<const float*>(st + L.co);
    float* sEN = reinterpret_cast<float*>(st + L.en);
    const int b0 = T.x, i0 = T.y, grp = T.z;
    const int lane = threadIdx.x & 31;
    const int nx = g.nx, ny = g.ny, th = g.th;
    const int l = SHOT ? lane : 0;
    const int j0 = SHOT ? b0 : b0 + lane * W;
    if (!SHOT && j0 >= ny) return;
    const int slot = SHOT ? lane : 0;
    const int s = SHOT ? grp * 32 + lane : grp;
    const PsiG rd = psi_group(g, rp, grp), wr = psi_group(g, rp ^ 1, grp);
    const int i1 = min(i0 + R, nx);
    const bool bcore = j0 >= th + 1 && j0 + W <= ny - th - 1;
    BandY by{};
    if constexpr (SHOT) by = band_adj<W>(g, j0);
    const long long resid_o = ((long long)s * g.nt + it) * g.nrx;
    const AdjCols<W, SHOT> C(lane);
#define EZS(r, k) sEZ[((r) * G::AEZ + C.c0 + (k)) * CS + l]
#define HXS(r, k) sHX[((r) * G::AHX + C.cx + (k)) * CS + l]
#define HYS(r, k) sHY[((r) * G::AHY + C.c0 + (k)) * CS + l]
#define ENS(r, k) sEN[((r) * NE + C.c0 + (k)) * CS + l]
#define COS(p, r, k) sCO[((p) * (R + 1) + (r)) * G::NCF + C.cc + (k)]
    // warp w: rows w*M .. w*M+M-1; warp 0 also row R (the halo row below)
    for (int m = 0; m <= M; ++m) {
        const int rr = m < M ? w * M + m : (w == 0 ? R : R + 1);
        if (rr > R) break;
        const int r = i0 + rr;
        if (r >= nx) {
#pragma unroll
            for (int k = 0; k <= W; ++k) ENS(rr, k) = 0.f;
            continue;
        }
        AdjEIn<W> A;
        float hyu[W + 1];
#pragma unroll
        for (int k = 0; k <= W; ++k) {
            A.ez[k] = EZS(rr, k);
            A.hyo[k] = HYS(rr + 1, k);
            hyu[k] = HYS(rr, k);
            A.ca[k] = COS(0, rr, k + 1);
            A.cb[k] = COS(1, rr, k + 1);
        }
#pragma unroll
        for (int k = 0; k < W + 2; ++k) A.hxo[k] = HXS(rr, k);
        int ic = E.x;
        const int ie = E.y;
        while (ic < ie && __ldg(g.inj_ev + ic).x < r) ++ic;
        float e[W + 1];
        adj_e_row<W, CS>(g, Rp, by, A, r, j0, l, slot, bcore && r >= th + 1 && r <= nx - th - 1, r < i1, hyu, e, resid_o,
                         ic, ie, rd, wr);
#pragma unroll
        for (int k = 0; k <= W; ++k) ENS(rr, k) = e[k];
    }
#undef EZS
#undef HXS
#undef HYS
#undef ENS
#undef COS
}

// Phase 2: H of row i0+w from the new E, the imaging sums, the stores.

// H of row i0 + w (w: row index within the tile) from the new E, imaging, stores.
template <int W, bool SHOT>
__device__ __forceinline__ void adj_tile_h_row(const Dev& g, const float* Rp, const unsigned char* st,
                                                    const TileSmem<W, SHOT>& L, int R, int w, int it, int rp) {
    const int4 T = reinterpret_cast<const StageHead*>(st)->tile;
    using G = TileGeom<W, SHOT>;
    constexpr int CS = G::CS;
    constexpr int NE = SHOT ? W + 1 : G::NWIN;
    const float* sEZ = reinterpret_cast<const float*>(st + L.ez);
    const float* sHX = reinterpret_cast<const float*>(st + L.hx);
    const float* sHY = reinterpret_cast<const float*>(st + L.hy);
    const float* sCO = reinterpret_cast<const float*>(st + L.co);
    const float* sH = reinterpret_cast<const float*>(st + L.hs);
    const float* sEN = reinterpret_cast<const float*>(st + L.en);
    const int b0 = T.x, i0 = T.y, grp = T.z;
    const int lane = threadIdx.x & 31;
    const int nx = g.nx, ny = g.ny, th = g.th;
    const int i = i0 + w;
    if (i >= nx) return;
    const int l = SHOT ? lane : 0;
    const int j0 = SHOT ? b0 : b0 + lane * W;
    const bool live = SHOT || j0 < ny;
    const int wp = rp ^ 1;
    const long long go = (long long)grp * g.plane;
    const PsiG rd = psi_group(g, rp, grp), wr = psi_group(g, wp, grp);
    const bool bcore = j0 >= th + 1 && j0 + W <= ny - th - 1;
    const AdjCols<W, SHOT> C(lane);
#define EZS(r, k) sEZ[((r) * G::AEZ + C.c0 + (k)) * CS + l]
#define HXS(r, k) sHX[((r) * G::AHX + C.cx + (k)) * CS + l]
#define HYS(r, k) sHY[((r) * G::AHY + C.c0 + (k)) * CS + l]
#define ENS(r, k) sEN[((r) * NE + C.c0 + (k)) * CS + l]
#define COS(p, r, k) sCO[((p) * (R + 1) + (r)) * G::NCF + C.cc + (k)]
    float ezc[W + 1], ezr[W], hx[W], hy[W], ch[W], f1[W], eo[W];
#pragma unroll
    for (int k = 0; k <= W; ++k) ezc[k] = live ? ENS(w, k) : 0.f;
#pragma unroll
    for (int q = 0; q < W; ++q) {
        ezr[q] = live ? ENS(w + 1, q) : 0.f;
        hx[q] = live ? HXS(w, q + 1) : 0.f;
        hy[q] = live ? HYS(w + 1, q) : 0.f;
        ch[q] = live ? COS(3, w, q + 1) : 0.f;
        eo[q] = live ? EZS(w, q) : 0.f;
        f1[q] = live ? sH[((size_t)w * G::AH + (SHOT ? 0 : lane * W) + q) * CS + l] : 0.f;
    }
#undef EZS
#undef HXS
#undef HYS
#undef ENS
#undef COS
    if (live) {
        if (bcore && i >= th + 1 && i <= nx - th - 1) {
#pragma unroll
            for (int q = 0; q < W; ++q) {
                hx[q] = __fsub_rn(hx[q], __fmul_rn(ch[q], __fsub_rn(ezc[q + 1], ezc[q])));
                hy[q] = __fadd_rn(hy[q], __fmul_rn(ch[q], __fsub_rn(ezr[q], ezc[q])));
            }
        } else if (SHOT && g.fast_cpml) {
            float dzx[W], dzy[W];
#pragma unroll
            for (int q = 0; q < W; ++q) {
                dzx[q] = __fsub_rn(ezc[q + 1], ezc[q]);
                dzy[q] = __fsub_rn(ezr[q], ezc[q]);
            }
            if constexpr (SHOT) {
                const BandY by = band_adj<W>(g, j0);
                if (by.lean) adj_h_row_shot<W>(g, Rp, by, i, j0, l, hx, hy, dzx, dzy, ch, rd, wr);
                else {
                    hx_cells<W, CS>(g, Rp, i, j0, l, hx, dzx, ch, 0, rd, wr);
                    hy_cells<W, CS, true>(g, Rp, i, j0, l, hy, dzy, ch, rd, wr);
                }
            }
        } else if (g.fast_cpml) {
            float dzx[W], dzy[W];
#pragma unroll
            for (int q = 0; q < W; ++q) {
                dzx[q] = __fsub_rn(ezc[q + 1], ezc[q]);
                dzy[q] = __fsub_rn(ezr[q], ezc[q]);
            }
            hx_cells<W, CS>(g, Rp, i, j0, l, hx, dzx, ch, 0, rd, wr);
            hy_cells<W, CS, true>(g, Rp, i, j0, l, hy, dzy, ch, rd, wr);
        } else {
#pragma unroll
            for (int q = 0; q < W; ++q) {
                const int j = j0 + q;
                if (j < ny) {
                    hx[q] = hx_cell<CS, true>(g, Rp, i, j, l, hx[q], __fsub_rn(ezc[q + 1], ezc[q]), ch[q], rd, wr);
                    hy[q] = hy_cell<CS, true>(g, Rp, i, j, l, hy[q], __fsub_rn(ezr[q], ezc[q]), ch[q], rd, wr);
                }
            }
        }
    }
    // imaging (compute.py:1167-1172), summed by parts: sum_t Ez_f[t] (lambda_t -
    // lambda_{t+1}) with lambda_{t+1} the old Ez of this step (k_imaging_tail
    // subtracts Ez_f[0] lambda_1); sigma: sum_t Ez_f[t] lambda_t dt
    float v[2 * W];
#pragma unroll
    for (int q = 0; q < W; ++q) {
        v[q] = __fmul_rn(f1[q], __fsub_rn(ezc[q], eo[q]));
        v[W + q] = __fmul_rn(__fmul_rn(f1[q], ezc[q]), g.dt);
    }
    double* gae = g.gacc + (long long)grp * 2 * ((long long)nx * ny);
    double* gas = gae + (long long)nx * ny;
    const long long go2 = (long long)i * ny + j0;
    if (SHOT) {
        constexpr int sh = (2 * W) == 4 ? 3 : ((2 * W) == 8 ? 2 : 1);
        const float x = lane_reduce_scatter<2 * W>(v, lane);
        if ((lane & ((1 << sh) - 1)) == 0) {
            const int e = lane >> sh;
            const int q = e < W ? e : e - W;
            if (j0 + q < ny) {
                double* a = (e < W ? gae : gas) + go2 + q;
                acc_add(g, a, (double)x);
            }
        }
    } else if (live) {
#pragma unroll
        for (int q = 0; q < W; ++q)
            if (j0 + q < ny) {
                acc_add(g, gae + go2 + q, (double)v[q]);
                acc_add(g, gas + go2 + q, (double)v[W + q]);
            }
    }
    if (!live) return;
    const long long o = ((long long)i * g.P + j0 + PADC) * CS + l;
    st_cells<W, CS>(g, g.ez[wp] + go + o, ezc);
    st_cells<W, CS>(g, g.hx[wp] + go + o, hx);
    st_cells<W, CS>(g, g.hy[wp] + go + o, hy);
}

// Rows w*M .. w*M+M-1 of the tile, phase 2.
template <int W, bool SHOT>
__device__ __forceinline__ void adj_tile_h(const Dev& g, const float* Rp, const unsigned char* st,
                                           const TileSmem<W, SHOT>& L, int R, int w, int M, int it, int rp) {
    for (int m = 0; m < M; ++m) adj_tile_h_row<W, SHOT>(g, Rp, st, L, R, w * M + m, it, rp);
}

template <int W, bool SHOT>
__global__ void __launch_bounds__(288) k_adj_pipe(const Dev g, const __grid_constant__ CUtensorMap tm_ez,
                                                  const __grid_constant__ CUtensorMap tm_hx,
                                                  const __grid_constant__ CUtensorMap tm_hy,
                                                  const __grid_constant__ CUtensorMap tm_co,
                                                  const __grid_constant__ CUtensorMap tm_h, const int it,
                                                  const int rp, const int S, const int R) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int NW = (blockDim.x >> 5) - 1;   // consumer warps; warp NW produces
    const int Mrows = R / NW;               // rows per consumer warp (R rows per tile)
    const TileSmem<W, SHOT> L(R, true);
    const PipeSmem M(g.th, S, L.total);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + M.full);
    uint64_t* empty = reinterpret_cast<uint64_t*>(smem + M.empty);
    float* Rp = reinterpret_cast<float*>(smem + M.prof);
    volatile int* flags = reinterpret_cast<volatile int*>(smem + M.flag);
    // launched with programmatic stream serialisation behind the previous
    // step: wait for it before anything of the solve is read, then let the
    // next step's launch place its blocks as these leave
    griddep_wait();
    griddep_launch_dependents();
    if (abort_launch(g, flags)) return;
    if (threadIdx.x == 0) {
        flags[1] = 0;
        for (int s = 0; s < S; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, NW);
        }
        fence_mbar_init();
    }
    for (int k = threadIdx.x; k < 8 * g.th; k += blockDim.x) Rp[k] = __ldg(g.pml + k);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == NW) {
        if (lane == 0)
            produce_tiles(g, full, empty, S, flags + 1, [&](int p, int s, uint64_t* bar) {
                adj_tile_issue<W, SHOT>(g, &tm_ez, &tm_hx, &tm_hy, &tm_co, &tm_h,
                                        smem + M.stages + (size_t)s * L.total, L, R, p, rp, it, bar);
            });
        return;
    }
    int s = 0;
    uint32_t par = 0;
    for (int p = blockIdx.x; p < g.ntiles; p += gridDim.x) {
        const bool ok = wait_or_stop(g, full + s, par, flags + 1);
        unsigned char* st = smem + M.stages + (size_t)s * L.total;
        if (ok) adj_tile_e<W, SHOT>(g, Rp, st, L, R, warp, Mrows, it, rp);
        consumers_sync(32 * NW);
        if (ok) adj_tile_h<W, SHOT>(g, Rp, st, L, R, warp, Mrows, it, rp);
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + s);
        if (++s == S) {
            s = 0;
            par ^= 1u;
        }
    }
}

}  // namespace fg
