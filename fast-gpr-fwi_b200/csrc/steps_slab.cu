// Launchers of the slab-tile step kernels (fdtd_slab.cuh).
#include "plan.h"
#include "fdtd_slab.cuh"

namespace fgk {

namespace {

// Launch `kernel` with the CPML profile in dynamic shared memory; with pdl,
// behind the general kernel of the same step with programmatic stream
// serialisation.
template <class K, class... A>
cudaError_t launch_slab(K kernel, int blocks, size_t smem, bool pdl, cudaStream_t st, A... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Blocks of a slab launch: as many as are resident, at most `cap` per SM
// (cap 0: no cap), at most one warp per tile.
template <class K>
cudaError_t slab_blocks(K kernel, size_t smem, int ntiles, int cap, int* blocks) {
    cudaError_t e = persistent_blocks(kernel, 4, smem, ntiles, blocks);
    if (e != cudaSuccess || cap <= 0) return e;
    int dev = 0, sms = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) *blocks = std::max(1, std::min(*blocks, cap * sms));
    return e;
}

template <int W>
cudaError_t launch_fwd_slab(const Dev& g, int t, int cap, int pdl, int* blocks, cudaStream_t st) {
    auto kernel = fg::k_fwd_slab<W>;
    const size_t smem = fg::prof_bytes(g.th);
    if (*blocks == 0) {
        const cudaError_t e = slab_blocks(kernel, smem, g.core0 - g.slab0, cap, blocks);
        if (e != cudaSuccess) return e;
    }
    return launch_slab(kernel, *blocks, smem, pdl != 0, st, g, t);
}
template <int W>
cudaError_t launch_adj_slab(const Dev& g, int it, int rp, int cap, int pdl, int* blocks, cudaStream_t st) {
    auto kernel = fg::k_adj_slab<W>;
    const size_t smem = fg::prof_bytes(g.th);
    if (*blocks == 0) {
        const cudaError_t e = slab_blocks(kernel, smem, g.core0 - g.slab0, cap, blocks);
        if (e != cudaSuccess) return e;
    }
    return launch_slab(kernel, *blocks, smem, pdl != 0, st, g, it, rp);
}

}  // namespace

FwdFn pick_fwd_slab(int W) {
    switch (W) {
        case 2: return launch_fwd_slab<2>;
        case 4: return launch_fwd_slab<4>;
        case 8: return launch_fwd_slab<8>;
    }
    return nullptr;
}
AdjFn pick_adj_slab(int W) {
    switch (W) {
        case 2: return launch_adj_slab<2>;
        case 4: return launch_adj_slab<4>;
        case 8: return launch_adj_slab<8>;
    }
    return nullptr;
}

}  // namespace fgk
