// Launchers of the persistent multi-step kernels (fdtd_multi.cuh).  Their
// state loads must see other blocks' stores of earlier steps of the launch.
#define FG_MULTI_STEP 1
#include "plan.h"
#include "fdtd_multi.cuh"

namespace fgk {

namespace {

// Cooperative launch of `kernel` with at most `want` blocks of 128 threads
// (fewer when fewer are resident at once).
template <class K, class... A>
cudaError_t launch_coop(K kernel, int want, cudaStream_t st, A... args) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorLaunchOutOfResources;
    const int blocks = std::max(1, std::min(want, per_sm * sms));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <int W, bool SHOT>
cudaError_t fwd_persist(const fg::Dev& g, unsigned* bar, int want, int t0, int t1, cudaStream_t st) {
    return launch_coop(fg::k_fwd_persist<W, SHOT>, want, st, g, bar, t0, t1);
}
template <int W, bool SHOT>
cudaError_t adj_persist(const fg::Dev& g, unsigned* bar, int want, int k0, int k1, cudaStream_t st) {
    return launch_coop(fg::k_adj_persist<W, SHOT>, want, st, g, bar, k0, k1);
}
template <int W, bool SHOT>
cudaError_t fwd_multi(const fg::MultiDevs& M, int want, int t0, int t1, cudaStream_t st) {
    return launch_coop(fg::k_fwd_multi<W, SHOT>, want, st, M, t0, t1);
}
template <int W, bool SHOT>
cudaError_t adj_multi(const fg::MultiDevs& M, int want, int k0, int k1, cudaStream_t st) {
    return launch_coop(fg::k_adj_multi<W, SHOT>, want, st, M, k0, k1);
}

}  // namespace

// want: blocks the largest model's tiles can keep busy (one warp per tile).
cudaError_t launch_fwd_multi(const fg::MultiDevs& M, bool shot, int W, int want, int t0, int t1, cudaStream_t st) {
    switch ((shot ? 10 : 0) + W) {
        case 12: return fwd_multi<2, true>(M, want, t0, t1, st);
        case 14: return fwd_multi<4, true>(M, want, t0, t1, st);
        case 18: return fwd_multi<8, true>(M, want, t0, t1, st);
        case 2: return fwd_multi<2, false>(M, want, t0, t1, st);
        case 4: return fwd_multi<4, false>(M, want, t0, t1, st);
        case 8: return fwd_multi<8, false>(M, want, t0, t1, st);
    }
    return cudaErrorInvalidValue;
}
cudaError_t launch_adj_multi(const fg::MultiDevs& M, bool shot, int W, int want, int k0, int k1, cudaStream_t st) {
    switch ((shot ? 10 : 0) + W) {
        case 12: return adj_multi<2, true>(M, want, k0, k1, st);
        case 14: return adj_multi<4, true>(M, want, k0, k1, st);
        case 18: return adj_multi<8, true>(M, want, k0, k1, st);
        case 2: return adj_multi<2, false>(M, want, k0, k1, st);
        case 4: return adj_multi<4, false>(M, want, k0, k1, st);
        case 8: return adj_multi<8, false>(M, want, k0, k1, st);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_fwd_persist(const fg::Dev& g, bool shot, int W, unsigned* bar, int want, int t0, int t1,
                               cudaStream_t st) {
    switch ((shot ? 10 : 0) + W) {
        case 12: return fwd_persist<2, true>(g, bar, want, t0, t1, st);
        case 14: return fwd_persist<4, true>(g, bar, want, t0, t1, st);
        case 18: return fwd_persist<8, true>(g, bar, want, t0, t1, st);
        case 2: return fwd_persist<2, false>(g, bar, want, t0, t1, st);
        case 4: return fwd_persist<4, false>(g, bar, want, t0, t1, st);
        case 8: return fwd_persist<8, false>(g, bar, want, t0, t1, st);
    }
    return cudaErrorInvalidValue;
}
cudaError_t launch_adj_persist(const fg::Dev& g, bool shot, int W, unsigned* bar, int want, int k0, int k1,
                               cudaStream_t st) {
    switch ((shot ? 10 : 0) + W) {
        case 12: return adj_persist<2, true>(g, bar, want, k0, k1, st);
        case 14: return adj_persist<4, true>(g, bar, want, k0, k1, st);
        case 18: return adj_persist<8, true>(g, bar, want, k0, k1, st);
        case 2: return adj_persist<2, false>(g, bar, want, k0, k1, st);
        case 4: return adj_persist<4, false>(g, bar, want, k0, k1, st);
        case 8: return adj_persist<8, false>(g, bar, want, k0, k1, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace fgk
