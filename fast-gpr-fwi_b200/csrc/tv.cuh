// ADMM total-variation denoising of a 2-D model (reference src/tv.py:135-217),
// the regulariser of the reference's default gradient (src/compute.py:916-933).
//
// The reference runs up to 500 ADMM iterations as ~25 tensor operations each
// plus a host-side convergence test per iteration.  Here the whole solve is
// one persistent kernel, launched cooperatively so every CTA is resident:
//
//   setup    m = max(data) (NaN-propagating), X = Y = [0 | data/(m + 1e-6) | 0]
//            on a one-cell zero border, Z = U = 0
//   per iteration, two phases separated by grid barriers:
//     A  interior cells:  X' = (N4(X) * lam * rho + rhs) / (1 + 4 lam rho)
//                         rhs = Y + lr (Dt Zx + Dt Zy) - lam (Dt Ux + Dt Uy)
//     B  every cell:      D X' (periodic backward differences), t = (U + rho D X') / rho,
//                         Z = sign(t) max(|t| - 1/rho, 0), U += rho (D X' - Z),
//                         and the block sums of (X' - X)^2 in float64
//     stop when ||X' - X|| < tol (every CTA sums the block sums in the same order)
//   out = X[1:-1, 1:-1] * m
//
// Every elementwise step rounds as float32 tensor operations do (each
// operation separately, scalars rounded to float32, no contraction: the
// library is built with -fmad=false); the four-neighbour sum is taken as
// ((up + left) + right) + down.  The convergence norm is summed in float64;
// it can stop one iteration apart from a float32 norm only when ||X' - X||
// lies within float32 rounding of tol.
//
// Grid barriers are bounded: a CTA that waits more than 2 s sets the error
// word and every CTA leaves (the output is then not written).
#pragma once

#include <cstdint>

#include "fdtd_common.cuh"

namespace fg {

struct TvArgs {
    const float* data;   // (M, N)
    float* out;          // (M, N)
    int M, N;            // model; the ADMM arrays are (M+2) x (N+2)
    float lam, lr, rho, inv_rho, den;   // lamda, lamda*rho, rho, 1/rho, 1 + 4 lamda rho (float32)
    int num_iter;
    double tol;
    float *x0, *x1, *y, *zx, *zy, *ux, *uy;   // (M+2) x (N+2) each
    double* partial;     // [2][gridDim.x] block sums of the convergence norm
    float* pmax;         // [gridDim.x] block maxima of the data
    unsigned* bar;       // [0] arrivals, [1] generation
    int* err;            // error word
    int* iters;          // iterations run
};

constexpr int ERR_TV_BARRIER = 301;
constexpr int TV_THREADS = 256;

__device__ __forceinline__ float nan_max(float a, float b) { return (a > b || a != a) ? a : b; }
// torch.sign on float: (0 < x) - (x < 0), so sign(+-0) = +0 and sign(NaN) = 0
__device__ __forceinline__ float torch_sign(float x) { return (float)((0.f < x) - (x < 0.f)); }
// torch.clamp(x, min=0): -0 and NaN pass through
__device__ __forceinline__ float clamp_min0(float x) { return x < 0.f ? 0.f : x; }

// Grid barrier (all CTAs resident: cooperative launch), by generation
// counter; the wait gives up after 2 s and reports it.
__device__ __forceinline__ bool tv_barrier(const TvArgs& a, volatile int* stop) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = a.bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(a.bar, 1u) == gridDim.x - 1) {
            a.bar[0] = 0;
            __threadfence();
            atomicAdd((unsigned*)gen, 1u);
        } else {
            uint64_t t0;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
            while (*gen == g) {
                if (*(volatile int*)a.err != 0) {
                    *stop = 1;
                    break;
                }
                uint64_t t;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                if (t - t0 > 2000000000ull) {
                    atomicCAS(a.err, 0, ERR_TV_BARRIER);
                    *stop = 1;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *stop == 0;
}

// Reduce v over the block with `op` (identity `id`); the result is valid in warp 0.
template <class T, class Op>
__device__ __forceinline__ T block_reduce(T v, T* sh, T id, Op op) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v = op(v, __shfl_xor_sync(FULL, v, m));
    if (lane == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sh[lane] : id;
#pragma unroll
        for (int m = 16; m >= 1; m >>= 1) v = op(v, __shfl_xor_sync(FULL, v, m));
    }
    __syncthreads();
    return v;
}

__global__ void __launch_bounds__(TV_THREADS) k_total_variation(const TvArgs a) {
    __shared__ double shd[TV_THREADS / 32];
    __shared__ float shf[TV_THREADS / 32];
    __shared__ float sh_val;
    __shared__ int stop;
    if (threadIdx.x == 0) stop = 0;
    __syncthreads();
    const int M = a.M, N = a.N, M2 = M + 2, N2 = N + 2;
    const long long cells = (long long)M2 * N2;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const float ninf = __int_as_float(0xff800000);

    // setup: data maximum, then the scaled model on a zero border
    float m = ninf;
    for (long long c = t0; c < (long long)M * N; c += stride) m = nan_max(m, a.data[c]);
    m = block_reduce(m, shf, ninf, nan_max);
    if (threadIdx.x == 0) a.pmax[blockIdx.x] = m;
    if (!tv_barrier(a, &stop)) return;
    if (threadIdx.x == 0) {
        float mm = a.pmax[0];
        for (unsigned b = 1; b < gridDim.x; ++b) mm = nan_max(mm, a.pmax[b]);
        sh_val = mm;
    }
    __syncthreads();
    const float dmax = sh_val;
    const float scale = __fadd_rn(dmax, 1e-6f);
    for (long long c = t0; c < cells; c += stride) {
        const int i = (int)(c / N2), j = (int)(c % N2);
        float v = 0.f;
        if (i >= 1 && i <= M && j >= 1 && j <= N) v = __fdiv_rn(a.data[(long long)(i - 1) * N + (j - 1)], scale);
        a.x0[c] = v;
        a.x1[c] = 0.f;
        a.y[c] = v;
        a.zx[c] = a.zy[c] = a.ux[c] = a.uy[c] = 0.f;
    }
    if (!tv_barrier(a, &stop)) return;

    float* X = a.x0;
    float* Xn = a.x1;
    int it = 0;
    while (it < a.num_iter) {
        // phase A: interior X update from the old X, Z, U
        for (long long c = t0; c < cells; c += stride) {
            const int i = (int)(c / N2), j = (int)(c % N2);
            if (i < 1 || i > M || j < 1 || j > N) {
                Xn[c] = 0.f;
                continue;
            }
            const float dzx = __fsub_rn(a.zx[c], a.zx[c + 1]);
            const float dzy = __fsub_rn(a.zy[c], a.zy[c + N2]);
            const float dux = __fsub_rn(a.ux[c], a.ux[c + 1]);
            const float duy = __fsub_rn(a.uy[c], a.uy[c + N2]);
            const float rhs = __fsub_rn(__fadd_rn(a.y[c], __fmul_rn(a.lr, __fadd_rn(dzx, dzy))),
                                        __fmul_rn(a.lam, __fadd_rn(dux, duy)));
            const float ns = __fadd_rn(__fadd_rn(__fadd_rn(X[c - N2], X[c - 1]), X[c + 1]), X[c + N2]);
            Xn[c] = __fdiv_rn(__fadd_rn(__fmul_rn(__fmul_rn(ns, a.lam), a.rho), rhs), a.den);
        }
        if (!tv_barrier(a, &stop)) return;
        // phase B: Z, U from the new X (periodic differences) and the norm
        double acc = 0.0;
        for (long long c = t0; c < cells; c += stride) {
            const int i = (int)(c / N2), j = (int)(c % N2);
            const float xc = Xn[c];
            const float dx = __fsub_rn(xc, Xn[c + (j == 0 ? N2 - 1 : -1)]);
            const float dy = __fsub_rn(xc, Xn[c + (i == 0 ? (long long)(M2 - 1) * N2 : -(long long)N2)]);
            float u = a.ux[c];
            float t = __fdiv_rn(__fadd_rn(u, __fmul_rn(a.rho, dx)), a.rho);
            float z = __fmul_rn(torch_sign(t), clamp_min0(__fsub_rn(fabsf(t), a.inv_rho)));
            a.zx[c] = z;
            a.ux[c] = __fadd_rn(u, __fmul_rn(a.rho, __fsub_rn(dx, z)));
            u = a.uy[c];
            t = __fdiv_rn(__fadd_rn(u, __fmul_rn(a.rho, dy)), a.rho);
            z = __fmul_rn(torch_sign(t), clamp_min0(__fsub_rn(fabsf(t), a.inv_rho)));
            a.zy[c] = z;
            a.uy[c] = __fadd_rn(u, __fmul_rn(a.rho, __fsub_rn(dy, z)));
            const double d = (double)__fsub_rn(xc, X[c]);
            acc += d * d;
        }
        acc = block_reduce(acc, shd, 0.0, [](double p, double q) { return p + q; });
        if (threadIdx.x == 0) a.partial[(it & 1) * gridDim.x + blockIdx.x] = acc;
        if (!tv_barrier(a, &stop)) return;
        ++it;
        // every CTA sums the block sums in the same order and takes the same branch
        if (threadIdx.x == 0) {
            double s = 0.0;
            const double* p = a.partial + ((it - 1) & 1) * gridDim.x;
            for (unsigned b = 0; b < gridDim.x; ++b) s += p[b];
            sh_val = sqrt(s) < a.tol ? 1.f : 0.f;
        }
        __syncthreads();
        float* tmp = X;
        X = Xn;
        Xn = tmp;
        if (sh_val != 0.f) break;
    }
    for (long long c = t0; c < (long long)M * N; c += stride) {
        const int i = (int)(c / N) + 1, j = (int)(c % N) + 1;
        a.out[c] = __fmul_rn(X[(long long)i * N2 + j], dmax);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.iters = it;
}

}  // namespace fg
