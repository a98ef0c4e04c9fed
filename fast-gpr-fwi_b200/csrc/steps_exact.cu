// Launchers of the exact-adjoint kernels (fdtd_exact.cuh).
#include "plan.h"
#include "fdtd_exact.cuh"

namespace fgk {

cudaError_t launch_adj_exact(const Dev& g, int it, int rp, int CS, int proj, cudaStream_t st) {
    const long long n = (long long)g.ngroups * g.nx * g.ny * CS;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    const size_t smem = (size_t)8 * g.th * sizeof(float);
    if (CS == 32) fg::k_adj_exact<32><<<blocks, 256, smem, st>>>(g, it, rp, proj);
    else if (CS == 1) fg::k_adj_exact<1><<<blocks, 256, smem, st>>>(g, it, rp, proj);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_inject_exact(const Dev& g, const int2* rxpos, const float* w, int t, int par, int CS,
                                cudaStream_t st) {
    const unsigned blocks = (unsigned)((g.S + 127) / 128);
    if (CS == 32) fg::k_inject_exact<32><<<blocks, 128, 0, st>>>(g, rxpos, w, t, par);
    else if (CS == 1) fg::k_inject_exact<1><<<blocks, 128, 0, st>>>(g, rxpos, w, t, par);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_grad_exact(const double* sums, const float* er, const float* se, int nx, int ny, double a,
                              float* ge, float* gs, cudaStream_t st) {
    const long long n = (long long)nx * ny;
    fg::k_grad_exact<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(sums, er, se, nx, ny, a, ge, gs);
    return cudaGetLastError();
}

}  // namespace fgk
