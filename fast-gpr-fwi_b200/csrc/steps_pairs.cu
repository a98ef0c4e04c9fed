// Launchers of the shot-pair lane-march step kernels (fdtd_pairs.cuh).
#include "plan.h"
#include "fdtd_pairs.cuh"

namespace fgk {

template <int W>
cudaError_t launch_fwd2(const Dev& g, int t, int, int, int* blocks, cudaStream_t st) {
    const size_t smem = fg::prof_bytes(g.th);
    auto kernel = fg::k_fwd2<W>;
    if (*blocks == 0) {
        cudaError_t e = allow_smem(kernel, smem);
        if (e == cudaSuccess) e = persistent_blocks(kernel, 4, smem, g.ntiles, blocks);
        if (e != cudaSuccess) return e;
    }
    kernel<<<*blocks, 128, smem, st>>>(g, t);
    return cudaSuccess;
}
template <int W>
cudaError_t launch_adj2(const Dev& g, int it, int rp, int, int, int* blocks, cudaStream_t st) {
    const size_t smem = fg::prof_bytes(g.th);
    auto kernel = fg::k_adj2<W>;
    if (*blocks == 0) {
        cudaError_t e = allow_smem(kernel, smem);
        if (e == cudaSuccess) e = persistent_blocks(kernel, 4, smem, g.ntiles, blocks);
        if (e != cudaSuccess) return e;
    }
    kernel<<<*blocks, 128, smem, st>>>(g, it, rp);
    return cudaSuccess;
}
FwdFn pick_fwd2(int W) { return W == 2 ? launch_fwd2<2> : W == 4 ? launch_fwd2<4> : nullptr; }
AdjFn pick_adj2(int W) { return W == 2 ? launch_adj2<2> : W == 4 ? launch_adj2<4> : nullptr; }

}  // namespace fgk
