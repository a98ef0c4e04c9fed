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
