// Persistent multi-step solves: every time step of one or more models in one
// cooperative launch.
//
// On a small grid a step is a few microseconds of work, and launching one
// kernel per step (2 nt launches per forward + gradient) makes the launch
// latency the cost.  Here one launch runs the whole time loop: in step t
// the warps of the grid take the tiles of model 0, then of model 1, ... (each
// model's own tile counter, the lane march of fdtd_lanes.cuh: fwd_step /
// adj_step), and a grid barrier separates the steps.  Models of different
// grids, shot counts and step counts share the launch (a model whose steps
// are done sits out); each keeps its own plan, workspace and buffers.
//
// No descriptor field is read through a computed address into parameter
// space: a single model's Dev is an ordinary kernel parameter (k_fwd_persist,
// k_adj_persist), and a batch's descriptors are copied into shared memory at
// the start of the launch (stage_devs), where the model index may vary.
//
// The grid barrier is a generation counter in global memory; every block is
// resident (cooperative launch).  Waits are bounded: a barrier not reached
// within 2 s sets the error word (ERR_WAIT_GRID) and every block leaves at the
// next barrier; fg_plan_check reports it.
#pragma once

#include "fdtd_common.cuh"
#include "fdtd_lanes.cuh"

namespace fg {

constexpr int MULTI_MAX = 8;                 // models per launch
constexpr int ERR_WAIT_GRID = 202;           // device error word: a grid barrier gave up

// The models of one launch, passed by value (kernel parameter space).
struct MultiDevs {
    Dev d[MULTI_MAX];
    int n;
    unsigned* bar;   // [0] arrivals, [1] generation (arrivals zero at launch)
    int* err;        // error word of the launch (the first model's)
};

// Grid barrier with a bounded wait; false when this or another block gave up.
// bar[0] counts arrivals (zero at launch), bar[1] is the generation.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* err, volatile int* stop) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = bar + 1;
        const unsigned g0 = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            bar[0] = 0;
            __threadfence();
            atomicAdd((unsigned*)gen, 1u);
        } else {
            const uint64_t t0 = globaltimer();
            while (*gen == g0) {
                if (*(volatile int*)err != 0) {
                    *stop = 1;
                    break;
                }
                if (globaltimer() - t0 > WAIT_LIMIT_NS) {
                    atomicCAS(err, 0, ERR_WAIT_GRID);
                    *stop = 1;
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *stop == 0;
}

// Copy the batch's descriptors into shared memory (4-byte words).
__device__ __forceinline__ const Dev* stage_devs(const MultiDevs& M, unsigned char* buf) {
    static_assert(sizeof(Dev) % 4 == 0, "Dev is copied as 4-byte words");
    const int words = M.n * (int)(sizeof(Dev) / 4);
    const int* src = reinterpret_cast<const int*>(M.d);
    int* dst = reinterpret_cast<int*>(buf);
    for (int k = threadIdx.x; k < words; k += blockDim.x) dst[k] = src[k];
    __syncthreads();
    return reinterpret_cast<const Dev*>(buf);
}

// ---------------------------------------------------------------------------
// One model
// ---------------------------------------------------------------------------
// Forward steps [t0, t1).
template <int W, bool SHOT>
__global__ void __launch_bounds__(128, 4) k_fwd_persist(const Dev g, unsigned* bar, const int t0, const int t1) {
    __shared__ int stop;
    if (threadIdx.x == 0) stop = 0;
    __syncthreads();
    for (int t = t0; t < t1; ++t) {
        fwd_step<W, SHOT, false>(g, g.pml, nullptr, t, 0);
        if (!grid_barrier(bar, g.err, &stop)) return;
    }
}

// Reference-mode adjoint rounds [k0, k1): iteration it = nt - 1 - k, parity k & 1.
template <int W, bool SHOT>
__global__ void __launch_bounds__(128, 3) k_adj_persist(const Dev g, unsigned* bar, const int k0, const int k1) {
    __shared__ int stop;
    if (threadIdx.x == 0) stop = 0;
    __syncthreads();
    for (int k = k0; k < k1; ++k) {
        adj_step<W, SHOT, false>(g, g.pml, nullptr, g.nt - 1 - k, k & 1, 0);
        if (!grid_barrier(bar, g.err, &stop)) return;
    }
}

// ---------------------------------------------------------------------------
// Several models
// ---------------------------------------------------------------------------
// Forward steps [t0, t1) of every model (a model runs its steps t < its nt).
template <int W, bool SHOT>
__global__ void __launch_bounds__(128, 2) k_fwd_multi(const __grid_constant__ MultiDevs M, const int t0,
                                                     const int t1) {
    __shared__ __align__(16) unsigned char buf[MULTI_MAX * sizeof(Dev)];
    __shared__ int stop;
    if (threadIdx.x == 0) stop = 0;
    const Dev* D = stage_devs(M, buf);
    const int n = M.n;
    for (int t = t0; t < t1; ++t) {
        for (int m = 0; m < n; ++m) {
            const Dev& g = D[m];
            if (t < g.nt) fwd_step<W, SHOT, false>(g, g.pml, nullptr, t, 0);
        }
        if (!grid_barrier(M.bar, M.err, &stop)) return;
    }
}

// Reference-mode adjoint rounds: in round k model m runs its iteration
// it = nt_m - 1 - k (reading parity k & 1) while it >= 1.
template <int W, bool SHOT>
__global__ void __launch_bounds__(128, 2) k_adj_multi(const __grid_constant__ MultiDevs M, const int k0,
                                                     const int k1) {
    __shared__ __align__(16) unsigned char buf[MULTI_MAX * sizeof(Dev)];
    __shared__ int stop;
    if (threadIdx.x == 0) stop = 0;
    const Dev* D = stage_devs(M, buf);
    const int n = M.n;
    for (int k = k0; k < k1; ++k) {
        for (int m = 0; m < n; ++m) {
            const Dev& g = D[m];
            const int it = g.nt - 1 - k;
            if (it >= 1) adj_step<W, SHOT, false>(g, g.pml, nullptr, it, k & 1, 0);
        }
        if (!grid_barrier(M.bar, M.err, &stop)) return;
    }
}

}  // namespace fg
