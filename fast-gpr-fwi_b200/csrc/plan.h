// Internal interface of libfastgpr between its translation units: the plan
// (host tables, launch shape, workspace layout) and the launchers of the
// step-kernel families, each compiled in a file of its own:
//   steps_lanes_fwd.cu  lane-march forward   (fdtd_lanes.cuh)
//   steps_lanes_adj.cu  lane-march adjoint   (fdtd_lanes.cuh)
//   steps_tiles.cu      tensor-map tile pipelines (fdtd_tile.cuh)
//   steps_pairs.cu      shot-pair lane march (fdtd_pairs.cuh)
//   steps_band.cu       band pipelines       (fdtd_band.cuh)
//   steps_exact.cu      exact adjoint        (fdtd_exact.cuh)
//   steps_core.cu       interior tiles       (fdtd_core.cuh)
//   steps_multi.cu      persistent multi-step solves of one or more models (fdtd_multi.cuh)
// Not part of the C ABI (include/fastgpr.h).
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/fastgpr.h"
#include "fdtd_common.cuh"
#include "fdtd_lanes.cuh"
#include "fdtd_tile.cuh"
#include "fdtd_multi.cuh"

using fg::Dev;
using fg::Ev;

struct fg_plan {
    // problem
    int nx, ny, S, nt, th, nsrc, nrx;
    float dx, dt;
    std::vector<int32_t> src, rx;
    std::vector<float> srcw, pml;
    // launch shape
    int kernel;         // 0 = tensor-map tiles, 1 = lane march, 2 = band pipeline
    bool shot;          // shot lanes (CS = 32 or, with pair, 64) or column lanes (CS = 1)
    bool pair = false;  // two shots per lane (CS = 64, lane march only)
    int W, TI, WPB, D;  // cells per thread, rows per tile, warps per block, ring stages (0 = direct loads)
    int pf = 0;         // next-tile L2 prefetch of the lane march (Dev::pf)
    bool split = false; // interior tiles (positions >= core0) run in the lean interior kernels
    int core0 = 0;      // first fetch position of an interior tile (== ntiles when none)
    int slab0 = 0;      // first fetch position of a slab tile: x tiles [slab0, yslab0), y tiles [yslab0, core0)
    int yslab0 = 0;
    int fwd_slab_blocks = 0, adj_slab_blocks = 0;
    bool slab_on = false; // slab tiles in the slab kernel (else in the general kernel)
    int slab_bpsm = 0;    // slab kernel blocks per SM at most (0 = as many as fit)
    int split_bpsm = 2; // blocks per SM of the general kernel's launch beside the interior kernel
    bool persist = false;   // whole solves in one persistent cooperative launch (small grids)
    // tensor maps of the tile kernels (encoded when a workspace is bound)
    CUtensorMap tm_fez, tm_fhx, tm_fhy, tm_aez, tm_ahx, tm_ahy, tm_co;
    int CS, SL;         // floats per cell in a group plane, shots per group
    int P, TY, Ph, BW, nb, nc, ngroups, ntiles;
    std::vector<int> chunk_row, order;
    std::vector<int4> tiles;   // (b0, i0, group, id) per position of `order`
    std::vector<Ev> src_ev, rx_ev, inj_ev;
    std::vector<int> src_off, rx_off, inj_off;
    // workspace layout (byte offsets)
    size_t o_coef, o_state, o_psi, o_chunk, o_order, o_tiles, o_ctr, o_srcev, o_rxev, o_injev, o_offs, o_srcw, o_pml, o_gacc,
        o_sums, o_partial, o_norms, o_err, o_rxpos, o_bar, total;
    // blocks of a persistent launch (0 = not yet measured) for the forward and adjoint kernels
    int fwd_blocks = 0, adj_blocks = 0, fwd_core_blocks = 0, adj_core_blocks = 0;
    // RN(1/dx) when the reciprocal division step is enabled (checked at bind), else 0
    float dinv = 0.f;
    int div_scaled = 0;   // the scaled step matches __fdiv_rn for every |x| < 2^31 (checked at bind)
    uint64_t id = 0;    // unique per plan in the process (which plan last filled the static scratch)
    // the adjoint's own plan (own state, coefficients, accumulators and launch
    // shape); its workspace follows this plan's in the caller's workspace
    fg_plan* adj = nullptr;
    ~fg_plan() { delete adj; }
    long long plane, pxs, pys;
    size_t state_bytes, psi_bytes;
    char* ws = nullptr;
    int64_t ws_bytes = 0;
    Dev g;
};


namespace fgk {

using FwdFn = cudaError_t (*)(const Dev&, int, int, int, int*, cudaStream_t);
using AdjFn = cudaError_t (*)(const Dev&, int, int, int, int, int*, cudaStream_t);

template <int W, bool SHOT>
inline size_t ring_smem(int wpb, int D, bool adjoint) {
    using RG = fg::RingGeom<W, SHOT>;
    return fg::ring_bar_bytes(wpb, D) + (size_t)wpb * D * (adjoint ? RG::ADJ : RG::FWD) * sizeof(float);
}

template <class K>
inline cudaError_t allow_smem(K kernel, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Launch `kernel` on `st` with programmatic stream serialisation behind the
// kernel before it (the kernel waits for that one with griddepcontrol.wait
// before it reads or writes any state).
template <class K, class... A>
inline cudaError_t launch_pdl(K kernel, int blocks, int threads, size_t smem, cudaStream_t st, A... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Blocks of a persistent launch: as many as are resident on the device at
// once, at most one warp per tile.
template <class K>
inline cudaError_t persistent_blocks(K kernel, int wpb, size_t smem, int ntiles, int* blocks) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 32 * wpb, smem);
    if (e != cudaSuccess) return e;
    const int need = (ntiles + wpb - 1) / wpb;
    *blocks = std::max(1, std::min(need, std::max(per_sm, 1) * sms));
    return cudaSuccess;
}

// Persistent pipeline launches: WPB consumer warps (TI / WPB rows each) + 1
// producer warp per CTA,
// as many CTAs as are resident on the device (at most one per tile).
template <class K>
inline cudaError_t pipe_blocks(K kernel, int threads, size_t smem, int ntiles, int* blocks) {
    if (*blocks) return cudaSuccess;
    cudaError_t e = allow_smem(kernel, smem);
    int dev = 0, sms = 0, per_sm = 0;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (e != cudaSuccess) return e;
    *blocks = std::max(1, std::min(ntiles, std::max(per_sm, 1) * sms));
    return cudaSuccess;
}
using FwdTileFn = cudaError_t (*)(fg_plan*, const Dev&, int, cudaStream_t);
using AdjTileFn = cudaError_t (*)(fg_plan*, const Dev&, const CUtensorMap&, int, int, cudaStream_t);

// Launchers of one step of a kernel family for a launch shape (cells per
// thread W), or nullptr when the family has no kernel of that shape.
FwdFn pick_fwd(bool shot, int W);        // lane march, forward
AdjFn pick_adj(bool shot, int W);        // lane march, adjoint
FwdFn pick_fwd2(int W);                  // shot pairs, forward
AdjFn pick_adj2(int W);                  // shot pairs, adjoint
FwdTileFn pick_fwd_tile(bool shot, int W);
AdjTileFn pick_adj_tile(bool shot, int W);
FwdFn pick_fwd_core(int W);              // interior tiles of the lane march, forward
AdjFn pick_adj_core(int W);              // interior tiles of the lane march, adjoint
FwdFn pick_fwd_slab(int W);              // slab tiles of the lane march, forward
AdjFn pick_adj_slab(int W);              // slab tiles of the lane march, adjoint
FwdFn pick_fwd_band(int W, int C);       // band pipeline (C consumer warps), forward
AdjFn pick_adj_band(int W, int C);       // band pipeline, adjoint
// Shared memory of a band-pipeline CTA (0: no kernel of that shape).
size_t band_smem(int W, int C, int th, int D, bool adjoint);
// Persistent multi-step solves (steps_multi.cu): every step of the models in
// M in one cooperative launch of at most `want` blocks.
cudaError_t launch_fwd_persist(const fg::Dev& g, bool shot, int W, unsigned* bar, int want, int t0, int t1,
                               cudaStream_t st);
cudaError_t launch_adj_persist(const fg::Dev& g, bool shot, int W, unsigned* bar, int want, int k0, int k1,
                               cudaStream_t st);
cudaError_t launch_fwd_multi(const fg::MultiDevs& M, bool shot, int W, int want, int t0, int t1, cudaStream_t st);
cudaError_t launch_adj_multi(const fg::MultiDevs& M, bool shot, int W, int want, int k0, int k1, cudaStream_t st);
// Exact adjoint (steps_exact.cu): one transposed step of every cell and its
// imaging sums; the receiver injection; the gradient from the sums.
cudaError_t launch_adj_exact(const Dev& g, int it, int rp, int CS, int proj, cudaStream_t st);
cudaError_t launch_inject_exact(const Dev& g, const int2* rxpos, const float* w, int t, int par, int CS,
                                cudaStream_t st);
cudaError_t launch_grad_exact(const double* sums, const float* er, const float* se, int nx, int ny, double a,
                              float* ge, float* gs, cudaStream_t st);
// Shared memory of the larger (adjoint) ring of a lane-march plan, or 0 for
// direct loads; of the larger (adjoint) CTA of a tile-pipeline plan.
size_t plan_ring_smem(const fg_plan* p);
size_t plan_tile_smem(const fg_plan* p);

}  // namespace fgk
