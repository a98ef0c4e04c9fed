// Launchers of the lane-march adjoint step kernels (fdtd_lanes.cuh).
#include "plan.h"

namespace fgk {

template <int W, bool SHOT, bool RING, bool LEAN = false>
cudaError_t launch_adj_k(const Dev& g, int it, int rp, int wpb, int D, int* blocks, cudaStream_t st) {
    const size_t smem = fg::prof_bytes(g.th) + (RING ? ring_smem<W, SHOT>(wpb, D, true) : 0);
    auto kernel = fg::k_adj<W, SHOT, RING, LEAN>;
    if (*blocks == 0) {
        cudaError_t e = allow_smem(kernel, smem);
        if (e == cudaSuccess) e = persistent_blocks(kernel, wpb, smem, g.ntiles, blocks);
        if (e != cudaSuccess) return e;
    }
    return launch_pdl(kernel, *blocks, 32 * wpb, smem, st, g, it, rp, D);
}
template <int W, bool SHOT>
cudaError_t launch_adj(const Dev& g, int it, int rp, int wpb, int D, int* blocks, cudaStream_t st) {
    if (D != 0) return launch_adj_k<W, SHOT, true>(g, it, rp, wpb, D, blocks, st);
    if constexpr (SHOT)
        if (g.lean) return launch_adj_k<W, SHOT, false, true>(g, it, rp, wpb, D, blocks, st);
    return launch_adj_k<W, SHOT, false>(g, it, rp, wpb, D, blocks, st);
}

template <bool SHOT>
AdjFn pick_adj_w(int W) {
    switch (W) {
        case 2: return launch_adj<2, SHOT>;
        case 4: return launch_adj<4, SHOT>;
        case 8: return launch_adj<8, SHOT>;
    }
    return nullptr;
}
AdjFn pick_adj(bool shot, int W) { return shot ? pick_adj_w<true>(W) : pick_adj_w<false>(W); }

}  // namespace fgk
