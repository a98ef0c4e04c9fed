// Launchers of the band-pipeline step kernels (fdtd_band.cuh).
#include "plan.h"
#include "fdtd_band.cuh"

namespace fgk {

template <int W, int C>
cudaError_t launch_fwd_band(const Dev& g, int t, int, int D, int* blocks, cudaStream_t st) {
    const fg::BandSmem L(g.th, D, fg::BandGeom<W, C>::FWD);
    auto kernel = fg::k_fwd_band<W, C>;
    const cudaError_t e = pipe_blocks(kernel, 32 * (C + 1), L.total, g.ntiles, blocks);
    if (e != cudaSuccess) return e;
    kernel<<<*blocks, 32 * (C + 1), L.total, st>>>(g, t, D);
    return cudaSuccess;
}
template <int W, int C>
cudaError_t launch_adj_band(const Dev& g, int it, int rp, int, int D, int* blocks, cudaStream_t st) {
    const fg::BandSmem L(g.th, D, fg::BandGeom<W, C>::ADJ);
    auto kernel = fg::k_adj_band<W, C>;
    const cudaError_t e = pipe_blocks(kernel, 32 * (C + 1), L.total, g.ntiles, blocks);
    if (e != cudaSuccess) return e;
    kernel<<<*blocks, 32 * (C + 1), L.total, st>>>(g, it, rp, D);
    return cudaSuccess;
}

// (cells per thread, consumer warps) pairs with a kernel
#define FG_BAND_SHAPES(X) X(2, 4) X(2, 8) X(4, 2) X(4, 4)

FwdFn pick_fwd_band(int W, int C) {
#define X(w, c) \
    if (W == w && C == c) return launch_fwd_band<w, c>;
    FG_BAND_SHAPES(X)
#undef X
    return nullptr;
}
AdjFn pick_adj_band(int W, int C) {
#define X(w, c) \
    if (W == w && C == c) return launch_adj_band<w, c>;
    FG_BAND_SHAPES(X)
#undef X
    return nullptr;
}
size_t band_smem(int W, int C, int th, int D, bool adjoint) {
#define X(w, c)                                                                                            \
    if (W == w && C == c)                                                                                  \
        return fg::BandSmem(th, D, adjoint ? fg::BandGeom<w, c>::ADJ : fg::BandGeom<w, c>::FWD).total;
    FG_BAND_SHAPES(X)
#undef X
    return 0;
}

}  // namespace fgk
