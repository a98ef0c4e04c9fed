// Launchers of the tensor-map tile-pipeline step kernels (fdtd_tile.cuh).
#include "plan.h"

namespace fgk {

template <int W, bool SHOT>
cudaError_t launch_fwd_tile(fg_plan* p, const Dev& g, int t, cudaStream_t st) {
    const fg::TileSmem<W, SHOT> L(p->TI, false);
    const fg::PipeSmem M(p->th, p->D, L.total);
    auto kernel = fg::k_fwd_pipe<W, SHOT>;
    const int threads = 32 * (p->WPB + 1);
    const cudaError_t e = pipe_blocks(kernel, threads, M.total, p->ntiles, &p->fwd_blocks);
    if (e != cudaSuccess) return e;
    return launch_pdl(kernel, p->fwd_blocks, threads, M.total, st, g, p->tm_fez, p->tm_fhx, p->tm_fhy, p->tm_co, t,
                      p->D, p->TI);
}
template <int W, bool SHOT>
cudaError_t launch_adj_tile(fg_plan* p, const Dev& g, const CUtensorMap& tmh, int it, int rp, cudaStream_t st) {
    const fg::TileSmem<W, SHOT> L(p->TI, true);
    const fg::PipeSmem M(p->th, p->D, L.total);
    auto kernel = fg::k_adj_pipe<W, SHOT>;
    const int threads = 32 * (p->WPB + 1);
    const cudaError_t e = pipe_blocks(kernel, threads, M.total, p->ntiles, &p->adj_blocks);
    if (e != cudaSuccess) return e;
    return launch_pdl(kernel, p->adj_blocks, threads, M.total, st, g, p->tm_aez, p->tm_ahx, p->tm_ahy, p->tm_co, tmh,
                      it, rp, p->D, p->TI);
}
FwdTileFn pick_fwd_tile(bool shot, int W) {
    if (shot) return W == 4 ? launch_fwd_tile<4, true> : W == 8 ? launch_fwd_tile<8, true> : nullptr;
    return W == 2 ? launch_fwd_tile<2, false> : W == 4 ? launch_fwd_tile<4, false> : nullptr;
}
AdjTileFn pick_adj_tile(bool shot, int W) {
    if (shot) return W == 4 ? launch_adj_tile<4, true> : W == 8 ? launch_adj_tile<8, true> : nullptr;
    return W == 2 ? launch_adj_tile<2, false> : W == 4 ? launch_adj_tile<4, false> : nullptr;
}
// Shared memory of the larger (adjoint) pipeline CTA.
size_t plan_tile_smem(const fg_plan* p) {
    size_t stage = 0;
    switch ((p->shot ? 10 : 0) + p->W) {
        case 14: stage = fg::TileSmem<4, true>(p->TI, true).total; break;
        case 18: stage = fg::TileSmem<8, true>(p->TI, true).total; break;
        case 2: stage = fg::TileSmem<2, false>(p->TI, true).total; break;
        case 4: stage = fg::TileSmem<4, false>(p->TI, true).total; break;
    }
    return fg::PipeSmem(p->th, p->D, stage).total;
}

}  // namespace fgk
