// Launchers of the lane-march forward step kernels (fdtd_lanes.cuh).
#include "plan.h"

namespace fgk {

template <int W, bool SHOT, bool RING, bool LEAN = false>
cudaError_t launch_fwd_k(const Dev& g, int t, int wpb, int D, int* blocks, cudaStream_t st) {
    const size_t smem = fg::prof_bytes(g.th) + (RING ? ring_smem<W, SHOT>(wpb, D, false) : 0);
    auto kernel = fg::k_fwd<W, SHOT, RING, LEAN>;
    if (*blocks == 0) {
        cudaError_t e = allow_smem(kernel, smem);
        if (e == cudaSuccess) e = persistent_blocks(kernel, wpb, smem, g.ntiles, blocks);
        if (e != cudaSuccess) return e;
    }
    return launch_pdl(kernel, *blocks, 32 * wpb, smem, st, g, t, D);
}
template <int W, bool SHOT>
cudaError_t launch_fwd(const Dev& g, int t, int wpb, int D, int* blocks, cudaStream_t st) {
    if (D != 0) return launch_fwd_k<W, SHOT, true>(g, t, wpb, D, blocks, st);
    if constexpr (SHOT)
        if (g.lean) return launch_fwd_k<W, SHOT, false, true>(g, t, wpb, D, blocks, st);
    return launch_fwd_k<W, SHOT, false>(g, t, wpb, D, blocks, st);
}
template <bool SHOT>
FwdFn pick_fwd_w(int W) {
    switch (W) {
        case 2: return launch_fwd<2, SHOT>;
        case 4: return launch_fwd<4, SHOT>;
        case 8: return launch_fwd<8, SHOT>;
    }
    return nullptr;
}
FwdFn pick_fwd(bool shot, int W) { return shot ? pick_fwd_w<true>(W) : pick_fwd_w<false>(W); }
// Shared memory of the larger (adjoint) ring, or 0 for direct loads.
size_t plan_ring_smem(const fg_plan* p) {
    if (p->D == 0) return 0;
    switch ((p->shot ? 10 : 0) + p->W) {
        case 12: return ring_smem<2, true>(p->WPB, p->D, true);
        case 14: return ring_smem<4, true>(p->WPB, p->D, true);
        case 18: return ring_smem<8, true>(p->WPB, p->D, true);
        case 2: return ring_smem<2, false>(p->WPB, p->D, true);
        case 4: return ring_smem<4, false>(p->WPB, p->D, true);
        case 8: return ring_smem<8, false>(p->WPB, p->D, true);
    }
    return 0;
}

}  // namespace fgk
