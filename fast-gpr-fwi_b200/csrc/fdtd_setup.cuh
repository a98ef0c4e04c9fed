// Kernels launched once per solve or per plan bind, outside the time loop:
// the update coefficients, the division checks and the gradient reductions.
// Included by fastgpr.cu only.
#pragma once

#include "fdtd_common.cuh"

namespace fg {

// ---------------------------------------------------------------------------
// Update coefficients: the reference's ucget / ucgeta (src/lib/uc.cu:11-45,
// :60-91) on the (nx, ny) model, written into pitched planes: cell (i, j) at
// i * P + j + col0, everything else (the i == nx row, columns j >= ny and the
// col0 leading pad columns) zero.
// ---------------------------------------------------------------------------
__global__ void k_coefficients(const float* __restrict__ er, const float* __restrict__ se,
                               const float* __restrict__ mr, int nx, int ny, float dt, float dx, int adjoint,
                               float* __restrict__ out, int P, int col0) {
    const long long plane = (long long)(nx + 1) * P;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= plane) return;
    const int i = (int)(idx / P), j = (int)(idx % P) - col0;
    float uE0 = 0.f, uE1 = 0.f, uE4 = 0.f, uH1 = 0.f, uH4 = 0.f;
    if (i < nx && j >= 0 && j < ny) {
        const float e0 = 8.8541878128e-12f;   // __constant__ float e0, uc.cu:8
        const float m0 = 1.25663706212e-06f;  // __constant__ float m0, uc.cu:9
        const long long c = (long long)i * ny + j;
        const float erv = er[c], sev = se[c], mrv = mr[c];
        const float HA = __fdiv_rn(__fmul_rn(m0, mrv), dt);
        const float inv_dx = __fdiv_rn(1.0f, dx);
        uH1 = __fdiv_rn(inv_dx, HA);
        uH4 = __fdiv_rn(1.0f, HA);
        if (!(sev > 100.0f)) {
            // EA/EB: float e0*er/dt plus the double literal 0.5*se, rounded to float
            const float q = __fdiv_rn(__fmul_rn(e0, erv), dt);
            const double hs = __dmul_rn(0.5, (double)sev);
            const float EA = __double2float_rn(__dadd_rn((double)q, hs));
            uE1 = __fdiv_rn(inv_dx, EA);
            uE4 = __fdiv_rn(1.0f, EA);
            if (adjoint) {
                const float num = __fmul_rn(__fmul_rn(2.0f, e0), erv);
                uE0 = __fdiv_rn(num, __fmaf_rn(sev, dt, num));
            } else {
                const float EB = __double2float_rn(__dsub_rn((double)q, hs));
                uE0 = __fdiv_rn(EB, EA);
            }
        }
    }
    out[idx] = uE0;
    out[plane + idx] = uE1;
    out[2 * plane + idx] = uE4;
    out[3 * plane + idx] = uH1;
    out[4 * plane + idx] = uH4;
}

// ---------------------------------------------------------------------------
// Check of div_d's correction step against __fdiv_rn for every significand
// of [1, 2): bad[0] counts the mismatches (bit patterns).
// ---------------------------------------------------------------------------
__global__ void k_div_check(float d, float dinv, int* bad) {
    int n = 0;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < (1 << 23); m += gridDim.x * blockDim.x) {
        const float x = __int_as_float(0x3f800000 | m);
        n += __float_as_int(div_d_step(x, d, dinv)) != __float_as_int(__fdiv_rn(x, d));
    }
    if (n) atomicAdd(bad, n);
}

// Check of div_d_scaled against __fdiv_rn for every x with |x| < 2^31 (bit
// patterns 0 .. 0x4effffff and their negatives): bad[0] counts the
// mismatches.
__global__ void k_div_check_scaled(float d, float dinv, int* bad) {
    int n = 0;
    const long long total = 0x4f000000ll;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < total;
         m += (long long)gridDim.x * blockDim.x) {
        const float x = __int_as_float((int)m);
        n += __float_as_int(div_d_scaled(x, d, dinv)) != __float_as_int(__fdiv_rn(x, d));
        n += __float_as_int(div_d_scaled(-x, d, dinv)) != __float_as_int(__fdiv_rn(-x, d));
    }
    if (n) atomicAdd(bad, n);
}

// ---------------------------------------------------------------------------
// Gradient reduction: sum the shot-group planes (fixed order), then the two
// L2 norms by a deterministic two-level reduction, then scale.
// ---------------------------------------------------------------------------
__global__ void k_grad_sum(const double* __restrict__ gacc, int ngroups, long long n, double* __restrict__ sums,
                           double* __restrict__ partial) {
    __shared__ double red[2][256];
    double a = 0.0, b = 0.0;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        double se = 0.0, ss = 0.0;
        for (int k = 0; k < ngroups; ++k) {
            se += gacc[(long long)k * 2 * n + c];
            ss += gacc[(long long)k * 2 * n + n + c];
        }
        sums[c] = se;
        sums[n + c] = ss;
        a += se * se;
        b += ss * ss;
    }
    red[0][threadIdx.x] = a;
    red[1][threadIdx.x] = b;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            red[0][threadIdx.x] += red[0][threadIdx.x + w];
            red[1][threadIdx.x] += red[1][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = red[0][0];
        partial[2 * blockIdx.x + 1] = red[1][0];
    }
}

__global__ void k_grad_norm(const double* __restrict__ partial, int nblocks, double* __restrict__ norms) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double a = 0.0, b = 0.0;
    for (int k = 0; k < nblocks; ++k) {
        a += partial[2 * k];
        b += partial[2 * k + 1];
    }
    norms[0] = sqrt(a);
    norms[1] = sqrt(b);
}

__global__ void k_grad_scale(const double* __restrict__ sums, const double* __restrict__ norms, long long n,
                             int normalize, float* __restrict__ ge, float* __restrict__ gs) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double ne = normalize ? norms[0] : 1.0;
    const double ns = normalize ? norms[1] : 1.0;
    if (ge) ge[c] = (float)(sums[c] / ne);
    if (gs) gs[c] = (float)(sums[n + c] / ns);
}

}  // namespace fg
