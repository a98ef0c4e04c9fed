// Launchers of the interior-tile step kernels (fdtd_core.cuh).
#include "plan.h"
#include "fdtd_core.cuh"

namespace fgk {

// Launch `kernel` on `st`; with pdl, behind the general kernel of the same
// step with programmatic stream serialisation (see fdtd_core.cuh).
template <class K, class... A>
cudaError_t launch_core(K kernel, int blocks, bool pdl, cudaStream_t st, A... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// `pdl` (the D argument of the launcher signature): launched behind a general
// kernel of the same step.
template <int W>
cudaError_t launch_fwd_core(const Dev& g, int t, int, int pdl, int* blocks, cudaStream_t st) {
    auto kernel = fg::k_fwd_core<W>;
    if (*blocks == 0) {
        const cudaError_t e = persistent_blocks(kernel, 4, 0, g.ntiles - g.core0, blocks);
        if (e != cudaSuccess) return e;
    }
    return launch_core(kernel, *blocks, pdl != 0, st, g, t);
}
template <int W>
cudaError_t launch_adj_core(const Dev& g, int it, int rp, int, int pdl, int* blocks, cudaStream_t st) {
    auto kernel = fg::k_adj_core<W>;
    if (*blocks == 0) {
        const cudaError_t e = persistent_blocks(kernel, 4, 0, g.ntiles - g.core0, blocks);
        if (e != cudaSuccess) return e;
        // Without a slab kernel, the general kernel on every boundary tile
        // sets the step's length; interior warps beyond 2 blocks per SM only
        // take its issue slots (measured, us per adjoint step with at most 2
        // blocks per SM / as many as fit: 440 x 340, 64 shots 89.3 / 90.5;
        // 440 x 340, 32 shots 57.5 / 59.6; beside a slab kernel, 296 x 296,
        // 32 shots 40.5 / 38.9, so the cap applies only without one)
        if (g.core0 == g.slab0) {
            int dev = 0, sms = 0;
            cudaError_t e2 = cudaGetDevice(&dev);
            if (e2 == cudaSuccess) e2 = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e2 != cudaSuccess) return e2;
            *blocks = std::max(1, std::min(*blocks, 2 * sms));
        }
    }
    return launch_core(kernel, *blocks, pdl != 0, st, g, it, rp);
}

FwdFn pick_fwd_core(int W) {
    switch (W) {
        case 2: return launch_fwd_core<2>;
        case 4: return launch_fwd_core<4>;
        case 8: return launch_fwd_core<8>;
    }
    return nullptr;
}
AdjFn pick_adj_core(int W) {
    switch (W) {
        case 2: return launch_adj_core<2>;
        case 4: return launch_adj_core<4>;
        case 8: return launch_adj_core<8>;
    }
    return nullptr;
}

}  // namespace fgk
