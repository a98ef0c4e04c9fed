// Causal FIR low-pass of receiver traces (reference src/multiscale.py:19-53):
// each series is reflect-padded by k-1 samples on the left and
// cross-correlated with the k taps,
//   out[t] = sum_{m=0}^{k-1} taps[m] * x[refl(t + m - (k-1))],  refl(q) = |q|,
// along the time axis of a (batch, T, R) array (R innermost), so the traces
// the solver returns, (shots, steps, receivers), are filtered in place of
// the reference's permute / reshape / conv1d / permute.  One thread per
// output sample, threads of a warp on consecutive receivers (coalesced); the
// taps sit in shared memory; the k reads of a sample hit L1 (neighbouring
// samples share them).  The sum runs over m in order with fused
// multiply-adds in float32.
#pragma once

#include <cstdint>

namespace fg {

constexpr int FIR_THREADS = 256;
constexpr int FIR_MAX_TAPS = 8192;   // shared-memory taps (32 KB)

__global__ void __launch_bounds__(FIR_THREADS) k_fir_causal(const float* __restrict__ x, long long batch, int T, int R,
                                                           const float* __restrict__ taps, int k,
                                                           float* __restrict__ out) {
    __shared__ float h[FIR_MAX_TAPS];
    for (int m = threadIdx.x; m < k; m += blockDim.x) h[m] = taps[m];
    __syncthreads();
    const long long n = batch * T * R;
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
        const long long s = o / ((long long)T * R);
        const int rem = (int)(o - s * (long long)T * R);
        const int t = rem / R, r = rem % R;
        const float* xs = x + s * (long long)T * R + r;
        float acc = 0.f;
        const int q0 = t - (k - 1);
        for (int m = 0; m < k; ++m) {
            int q = q0 + m;
            q = q < 0 ? -q : q;
            acc = __fmaf_rn(h[m], __ldg(xs + (long long)q * R), acc);
        }
        out[o] = acc;
    }
}

}  // namespace fg
