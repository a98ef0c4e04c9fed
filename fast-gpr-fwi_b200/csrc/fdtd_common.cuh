// Device-side pieces shared by the solver kernels: the per-solve descriptor,
// guarded global accesses, the per-cell update arithmetic, the coefficient
// kernel and the gradient reductions.
//
// Memory layout.  Shots are processed in groups.  A group's field plane is
// (nx+1) rows x P columns x CS shot slots, shot slot fastest, with one
// leading zero column so that column -1 exists:
//   cell (i, j) of slot l  ->  (i * P + j + 1) * CS + l
// Shot-lane solves use CS = 32 (a warp's 32 lanes are 32 shots of the same
// cells, so one warp access is one 128-byte line); column-lane solves use
// CS = 1 (one shot per group, the classic row-major plane, lanes own
// consecutive columns).  Row nx and columns >= ny are the reference's zero
// frame.  Coefficient planes are (nx+1) x P with the same leading column,
// shared by all shots.  CPML auxiliaries and the Ez history have no pad.
//
// Per-cell arithmetic follows the reference kernels (paths relative to the
// reference project):
//   interior E  src/lib/fields_updates_gpu.cu:8-33
//   interior H  src/lib/fields_updates_gpu.cu:47-78
//   CPML E      src/lib/pml_updates_e.cu:58-76 (x), 267-285 (y) and the plus sides
//   CPML H      src/lib/pml_updates_h.cu:37-54 (x), 273-290 (y) and the plus sides
// The library is compiled with -fmad=false, so every fused multiply-add below
// is an explicit __fmaf_rn and nothing else is contracted; the result of each
// cell is the reference's bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fg {

constexpr unsigned FULL = 0xffffffffu;
constexpr int PADC = 4;   // leading zero columns of field and coefficient planes

// Event: something that happens to one cell of one shot at one row of a tile
// (a receiver sample, a source injection, an adjoint residual injection).
// x = row i, y = shot slot within the group, z = column j, w = index
// (receiver r or source n).  A tile's events are sorted by (x, y, z, w).
using Ev = int4;

struct Dev {
    // geometry
    int nx, ny;          // compute grid; row nx and columns >= ny are the zero frame
    int P;               // row pitch of field / coefficient planes (cells)
    int th;              // CPML thickness
    int TY;              // row pitch of y-slab CPML auxiliaries (>= th)
    int S, nt, nrx;      // shots, time steps, receivers per shot
    int Ph;              // row pitch of the Ez history (cells, >= ny)
    int ngroups;         // shot groups
    float d;             // cell size (CPML derivative divisor)
    float dinv;          // RN(1/d) when div_d may use it (checked at bind), else 0
    int div_scaled;      // div_d_scaled is __fdiv_rn for every |x| < 2^31 (checked at bind)
    float dt;            // time step (sigma imaging factor)
    long long plane;     // floats of one group's plane of one field
    long long pxs, pys;  // floats of one group's x-slab / y-slab auxiliaries
    // coefficient planes: uE0 (or Ucgeta's uE0), uE1, uE4, uH1, uH4
    const float *ca, *cb, *cd, *ch, *ci;
    const float* pml;    // (8, th): ERA ERB ERE ERF HRA HRB HRE HRF
    // state, ping-pong pairs; index = parity
    float *ez[2], *hx[2], *hy[2];
    float *pex[2], *pey[2], *phx[2], *phy[2];
    // tiling: tile = (group, row chunk, column band); warps fetch tiles in the
    // order of `order` (CPML-heavy tiles first) from a launch counter
    int nb, nc, ntiles;
    const int* order;                       // (ntiles) tile ids
    const int4* tiles;                      // (ntiles) (b0, i0, group, id) in fetch order
    int* tile_ctr;                          // 8 counters: general, interior, slab kernels x 2 launch parities
    int fast_cpml;                          // 2 th < nx and 2 th < ny: no cell in two slabs of one axis
    int core0;                              // first fetch position of the interior tiles (lean kernels)
    int slab0, yslab0;                      // x-slab tiles [slab0, yslab0), y-slab tiles [yslab0, core0)
    int lean;                               // every band takes the shot-lane CPML rows (see fwd_step)
    int pf;                                 // lane march, shot lanes: prefetch a warp's next tile into L2
                                            // (0 no, 1 when the current tile starts, 2 at its middle row)
    const int* chunk_row;                   // (nc+1) row boundaries
    const Ev* src_ev; const int* src_off;   // forward sources per tile
    const Ev* rx_ev;  const int* rx_off;    // forward receivers per tile
    const Ev* inj_ev; const int* inj_off;   // adjoint injections, rows [i0, i1], columns [b0, b0+BW]
    const float* srcw;   // (nsrc, nt)
    // solve I/O
    float* traces;       // (S, nt, nrx)
    float* hist;         // (steps, ngroups, nx, Ph, CS): step t at index t - hist_t0
    int hist_t0;         // first step the history buffer holds (0 = the whole run)
    const float* resid;  // (S, nt, nrx): residual, or the synthetic traces when obs is set
    const float* obs;    // (S, nt, nrx) observed traces: inject obs_scale * sign(resid - obs), else NULL
    float obs_scale;
    double* gacc;        // (ngroups, 2, nx, ny)
    // bounds of every buffer the kernels touch (checked builds)
    const char* ws_lo; const char* ws_hi;
    const char* out_lo; const char* out_hi;   // the history buffer
    int* err;            // device error word
};

#ifdef FG_CHECKED
// Checked build: every workspace / history access is tested against the
// buffer it belongs to; a violation records a code and the access is
// skipped (loads return 0), so a logic error never becomes a memory fault.
__device__ __forceinline__ bool in_bounds(const Dev& g, const void* p, int bytes) {
    const char* c = (const char*)p;
    if (c >= g.ws_lo && c + bytes <= g.ws_hi) return true;
    if (g.out_lo && c >= g.out_lo && c + bytes <= g.out_hi) return true;
    atomicCAS(g.err, 0, 100);
    return false;
}
#define FG_OK_PTR(g, p, bytes) in_bounds((g), (p), (bytes))
#else
#define FG_OK_PTR(g, p, bytes) true
#endif

// Loads of values that no thread writes during the step (old state of the
// read parity, coefficients, CPML vectors, history) take the read-only cache
// path.  A launch that runs several steps reads state that other blocks wrote
// earlier in the same launch, which that path is not guaranteed to see: the
// translation unit of such kernels defines FG_MULTI_STEP, and the loads then
// go to L2 (ld.global.cg), which every block's stores reach.
#ifdef FG_MULTI_STEP
#define FG_LDRO(p) __ldcg(p)
#else
#define FG_LDRO(p) __ldg(p)
#endif
__device__ __forceinline__ float ldro(const Dev& g, const float* p) {
    if (!FG_OK_PTR(g, p, 4)) return 0.f;
    return FG_LDRO(p);
}
__device__ __forceinline__ void st1(const Dev& g, float* p, float x) {
    if (!FG_OK_PTR(g, p, 4)) return;
    __stcg(p, x);
}

// N cells of one shot starting at p, consecutive cells CS floats apart.
template <int N, int CS>
__device__ __forceinline__ void ld_cells(const Dev& g, float* x, const float* p) {
    if constexpr (CS == 1 && N % 4 == 0) {
#pragma unroll
        for (int k = 0; k < N; k += 4) {
            if (!FG_OK_PTR(g, p + k, 16)) {
                x[k] = x[k + 1] = x[k + 2] = x[k + 3] = 0.f;
                continue;
            }
            const float4 q = FG_LDRO(reinterpret_cast<const float4*>(p + k));
            x[k] = q.x; x[k + 1] = q.y; x[k + 2] = q.z; x[k + 3] = q.w;
        }
    } else if constexpr (CS == 1 && N == 2) {
        if (!FG_OK_PTR(g, p, 8)) {
            x[0] = x[1] = 0.f;
            return;
        }
        const float2 q = FG_LDRO(reinterpret_cast<const float2*>(p));
        x[0] = q.x; x[1] = q.y;
    } else {
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = ldro(g, p + k * CS);
    }
}

// Store N cells; STREAM marks data not read again soon (the history).
template <int N, int CS, bool STREAM = false>
__device__ __forceinline__ void st_cells(const Dev& g, float* p, const float* x) {
    if constexpr (CS == 1 && N % 4 == 0) {
#pragma unroll
        for (int k = 0; k < N; k += 4) {
            if (!FG_OK_PTR(g, p + k, 16)) continue;
            const float4 q = make_float4(x[k], x[k + 1], x[k + 2], x[k + 3]);
            if (STREAM) __stcs(reinterpret_cast<float4*>(p + k), q);
            else __stcg(reinterpret_cast<float4*>(p + k), q);
        }
    } else if constexpr (CS == 1 && N == 2) {
        if (!FG_OK_PTR(g, p, 8)) return;
        const float2 q = make_float2(x[0], x[1]);
        if (STREAM) __stcs(reinterpret_cast<float2*>(p), q);
        else __stcg(reinterpret_cast<float2*>(p), q);
    } else {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            if (!FG_OK_PTR(g, p + k * CS, 4)) continue;
            if (STREAM) __stcs(p + k * CS, x[k]);
            else __stcg(p + k * CS, x[k]);
        }
    }
}

// Value injected at a receiver by the adjoint (back.cu:34 subtracts it from
// Ez): the residual resid[o]; or, with observed traces, the derivative of
// the L1 misfit sum |syn - obs| * scale formed on the fly from the synthetic
// traces (in resid) and the observed ones, scale * sign(syn - obs), as
// torch's L1 loss backward forms it (sign(0) = 0).
__device__ __forceinline__ float inj_value(const Dev& g, long long o) {
    const float syn = __ldg(g.resid + o);
    if (!g.obs) return syn;
    const float d = __fsub_rn(syn, __ldg(g.obs + o));
    return __fmul_rn((float)((0.f < d) - (d < 0.f)), g.obs_scale);
}

// a += x on a float64 imaging accumulator: a reduction applied by the memory
// system (red.global.add.f64, round to nearest), so the warp does not wait
// for the old value.  Every address has one adder per launch, so the result
// is the plain a + x.
__device__ __forceinline__ void acc_add(const Dev& g, double* a, double x) {
    if (!FG_OK_PTR(g, a, 8)) return;
    asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;" ::"l"(a), "d"(x) : "memory");
}

// N consecutive coefficients of one row (planes are not per shot); p is
// aligned to A floats (4: 16 bytes, 2: 8 bytes), so the run is read with
// vector loads.
template <int N, int A = 1>
__device__ __forceinline__ void ld_coef(const Dev& g, float* x, const float* p) {
    constexpr int V = A >= 4 ? 4 : (A >= 2 ? 2 : 1);
    constexpr int NV = V > 1 ? N / V * V : 0;
#pragma unroll
    for (int k = 0; k < NV; k += V) {
        if (!FG_OK_PTR(g, p + k, 4 * V)) {
#pragma unroll
            for (int q = 0; q < V; ++q) x[k + q] = 0.f;
            continue;
        }
        if constexpr (V == 4) {
            const float4 v = __ldg(reinterpret_cast<const float4*>(p + k));
            x[k] = v.x; x[k + 1] = v.y; x[k + 2] = v.z; x[k + 3] = v.w;
        } else if constexpr (V == 2) {
            const float2 v = __ldg(reinterpret_cast<const float2*>(p + k));
            x[k] = v.x; x[k + 1] = v.y;
        }
    }
#pragma unroll
    for (int k = NV; k < N; ++k) x[k] = ldro(g, p + k);
}

__device__ __forceinline__ long long coef_at(const Dev& g, int i, int j) { return (long long)i * g.P + j + PADC; }
// Alignment (floats) of coef_at(i, j0) for a thread's first column j0: the
// row pitch P and the pad are multiples of 4 and j0 is a multiple of W.
template <int W>
constexpr int CALIGN = W % 4 == 0 ? 4 : (W % 2 == 0 ? 2 : 1);

// a*b + c*d with the first product fused, a*b - c*d likewise.
__device__ __forceinline__ float madd2(float a, float b, float c, float d) {
    return __fmaf_rn(a, b, __fmul_rn(c, d));
}
__device__ __forceinline__ float msub2(float a, float b, float c, float d) {
    return __fmaf_rn(a, b, -__fmul_rn(c, d));
}

// x / d rounded to nearest, as __fdiv_rn(x, d).  With dinv = RN(1/d) the
// quotient is q = RN(x * dinv), then one correction step q' = RN(q + r * dinv)
// with the exact remainder r = x - q d from an FMA (Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990; Muller et al., Handbook of Floating-Point Arithmetic,
// ch. 5).  The step returns RN(x/d) when q is within one ulp of x/d, which
// holds when |d * dinv - 1| < 2^-25.  The quotient of x and of x * 2^e round
// alike, so one binade of x decides every x whose exponent keeps q and r
// normal: the library enables dinv only after checking all 2^23 significands
// of [1, 2) against __fdiv_rn on the device, and only for d in [2^-30, 2^30];
// other x (|x| outside [2^-90, 2^90), NaN, infinity) take __fdiv_rn.
__device__ __forceinline__ float div_d_step(float x, float d, float dinv) {
    const float q = __fmul_rn(x, dinv);
    const float r = __fmaf_rn(-q, d, x);
    return __fmaf_rn(r, dinv, q);
}
// The step on x * 2^59, scaled back by 2^-59.  For |x| < 2^31 the scaled
// argument is zero or lies in [2^-90, 2^90), where the step is the correctly
// rounded quotient, so no test of x is needed below 2^31; scaling back is
// exact unless the quotient is subnormal, where the two roundings may differ
// from one (the bind-time check, k_div_check_scaled, decides per divisor).
// For x = -0 the step gives +0: the sign of x goes back on (a no-op for every
// other x, as d > 0).
__device__ __forceinline__ float div_d_scaled(float x, float d, float dinv) {
    return copysignf(__fmul_rn(div_d_step(__fmul_rn(x, 0x1p59f), d, dinv), 0x1p-59f), x);
}
__device__ __forceinline__ float div_d(const Dev& g, float x) {
    if (g.dinv != 0.f) {
        const float ax = fabsf(x);
        if (ax >= 0x1p-90f && ax < 0x1p90f) return div_d_step(x, g.d, g.dinv);
        if (ax == 0.f) return __fmul_rn(x, g.dinv);   // +-0 / d keeps the sign of x (d > 0)
    }
    return __fdiv_rn(x, g.d);
}

// One HORIPML order-1 correction: F +-= u4*((RA-1)*D + RB*psi); psi = RE*psi - RF*D.
// R points at the 4 coefficient vectors (RA, RB, RE, RF) of length th, in
// shared memory (the solver kernels stage the profile there at launch).
template <bool PLUS>
__device__ __forceinline__ float cpml(const Dev& g, float f, float deriv, float u4, float& psi, const float* R,
                                      int k) {
    const int th = g.th;
    const float ra1 = __fsub_rn(R[k], 1.0f);
    const float rb = R[th + k];
    const float re = R[2 * th + k];
    const float rf = R[3 * th + k];
    const float t = madd2(ra1, deriv, rb, psi);
    const float out = __fmaf_rn(PLUS ? u4 : -u4, t, f);
    psi = msub2(re, psi, rf, deriv);
    return out;
}

// One group's CPML auxiliaries for one parity.
//   ex, hx: x slabs, [2 th][P][CS]: E rows k = th-i (i in 1..th) and th+(i-(nx-th));
//           H rows k = th-1-i (i in 0..th-1) and th+(i-(nx-th))
//   ey, hy: y slabs, [2 (nx+1)][TY][CS]: row i (y0 slab) and nx+1+i (ymax slab)
struct PsiG {
    float *ex, *ey, *hx, *hy;
};
__device__ __forceinline__ PsiG psi_group(const Dev& g, int par, int grp) {
    PsiG p;
    p.ex = g.pex[par] + (long long)grp * g.pxs;
    p.ey = g.pey[par] + (long long)grp * g.pys;
    p.hx = g.phx[par] + (long long)grp * g.pxs;
    p.hy = g.phy[par] + (long long)grp * g.pys;
    return p;
}

// E update of cell (i, j), shot slot l: interior leapfrog (i>=1, j>=1) then
// the CPML corrections in the reference's slab order x0, y0, xmax, ymax.
//   dhy = Hy[i][j] - Hy[i-1][j], dhx = Hx[i][j] - Hx[i][j-1]
// The auxiliaries are read from `rd` and, when STORE, written to `wr`.
template <int CS, bool STORE>
__device__ __forceinline__ float e_cell(const Dev& g, const float* R, int i, int j, int l, float ez, float dhy,
                                        float dhx, float ca, float cb, const PsiG& rd, const PsiG& wr) {
    if (i >= 1 && j >= 1) ez = __fmaf_rn(-cb, dhx, madd2(ca, ez, cb, dhy));
    const int th = g.th;
    if (th > 0) {
        const int P = g.P, nx = g.nx, ny = g.ny;
        const bool x0 = (i >= 1 && i <= th), xm = (i >= nx - th);
        const bool y0 = (j >= 1 && j <= th), ym = (j >= ny - th);
        if (x0 | xm | y0 | ym) {
            const float cd = ldro(g, g.cd + (long long)i * P + j + PADC);
            if (x0) {
                const int k = th - i;
                const long long o = ((long long)k * P + j) * CS + l;
                float psi = ldro(g, rd.ex + o);
                ez = cpml<true>(g, ez, div_d(g, dhy), cd, psi, R, k);
                if (STORE) st1(g, wr.ex + o, psi);
            }
            if (y0) {
                const int k = th - j;
                const long long o = ((long long)i * g.TY + k) * CS + l;
                float psi = ldro(g, rd.ey + o);
                ez = cpml<false>(g, ez, div_d(g, dhx), cd, psi, R, k);
                if (STORE) st1(g, wr.ey + o, psi);
            }
            if (xm) {
                const int k = i - (nx - th);
                const long long o = ((long long)(th + k) * P + j) * CS + l;
                float psi = ldro(g, rd.ex + o);
                ez = cpml<true>(g, ez, div_d(g, dhy), cd, psi, R, k);
                if (STORE) st1(g, wr.ex + o, psi);
            }
            if (ym) {
                const int k = j - (ny - th);
                const long long o = ((long long)(nx + 1 + i) * g.TY + k) * CS + l;
                float psi = ldro(g, rd.ey + o);
                ez = cpml<false>(g, ez, div_d(g, dhx), cd, psi, R, k);
                if (STORE) st1(g, wr.ey + o, psi);
            }
        }
    }
    return ez;
}

// Hx update of cell (i, j): interior (i >= 1) then the y-slab CPML (y0, ymax).
//   dzx = Ez[i][j+1] - Ez[i][j]
template <int CS, bool STORE>
__device__ __forceinline__ float hx_cell(const Dev& g, const float* R, int i, int j, int l, float hx, float dzx,
                                         float ch, const PsiG& rd, const PsiG& wr) {
    if (i >= 1) hx = msub2(1.0f, hx, ch, dzx);
    const int th = g.th;
    if (th > 0) {
        const int ny = g.ny;
        const bool y0 = j <= th - 1, ym = j >= ny - th;
        if (y0 | ym) {
            const float ci = ldro(g, g.ci + (long long)i * g.P + j + PADC);
            const float* HR = R + 4 * th;
            if (y0) {
                const int k = th - 1 - j;
                const long long o = ((long long)i * g.TY + k) * CS + l;
                float psi = ldro(g, rd.hy + o);
                hx = cpml<false>(g, hx, div_d(g, dzx), ci, psi, HR, k);
                if (STORE) st1(g, wr.hy + o, psi);
            }
            if (ym) {
                const int k = j - (ny - th);
                const long long o = ((long long)(g.nx + 1 + i) * g.TY + k) * CS + l;
                float psi = ldro(g, rd.hy + o);
                hx = cpml<false>(g, hx, div_d(g, dzx), ci, psi, HR, k);
                if (STORE) st1(g, wr.hy + o, psi);
            }
        }
    }
    return hx;
}

// Hy update of cell (i, j): interior (j >= 1) then the x-slab CPML (x0, xmax).
//   dzy = Ez[i+1][j] - Ez[i][j]
template <int CS, bool STORE>
__device__ __forceinline__ float hy_cell(const Dev& g, const float* R, int i, int j, int l, float hy, float dzy,
                                         float ch, const PsiG& rd, const PsiG& wr) {
    if (j >= 1) hy = madd2(1.0f, hy, ch, dzy);
    const int th = g.th;
    if (th > 0) {
        const int nx = g.nx, P = g.P;
        const bool x0 = i <= th - 1, xm = i >= nx - th;
        if (x0 | xm) {
            const float ci = ldro(g, g.ci + (long long)i * P + j + PADC);
            const float* HR = R + 4 * th;
            if (x0) {
                const int k = th - 1 - i;
                const long long o = ((long long)k * P + j) * CS + l;
                float psi = ldro(g, rd.hx + o);
                hy = cpml<true>(g, hy, div_d(g, dzy), ci, psi, HR, k);
                if (STORE) st1(g, wr.hx + o, psi);
            }
            if (xm) {
                const int k = i - (nx - th);
                const long long o = ((long long)(th + k) * P + j) * CS + l;
                float psi = ldro(g, rd.hx + o);
                hy = cpml<true>(g, hy, div_d(g, dzy), ci, psi, HR, k);
                if (STORE) st1(g, wr.hx + o, psi);
            }
        }
    }
    return hy;
}

// ---------------------------------------------------------------------------
// CPML for a run of N cells of one row, when no cell lies in two slabs of the
// same axis (2 th < nx and 2 th < ny).  All loads of the run (uE4/uH4
// coefficients and the auxiliaries) are issued before any update, so a CPML
// row costs one memory round trip instead of one per slab.  The profile
// vectors R (8 x th: ERA ERB ERE ERF HRA HRB HRE HRF) are read from shared
// memory.  The arithmetic and the slab order per cell (x0, y0, xmax, ymax)
// are those of e_cell / hx_cell / hy_cell.
// ---------------------------------------------------------------------------

// Ez of cells (i, j0 + n), n < N: interior then CPML; auxiliaries of the
// first `nown` cells are stored when `own_row`.
template <int N, int CS>
__device__ __forceinline__ void e_cells(const Dev& g, const float* R, int i, int j0, int l, float* ez,
                                        const float* dhy, const float* dhx, const float* ca, const float* cb,
                                        int nown, bool own_row, const PsiG& rd, const PsiG& wr) {
    const int th = g.th, nx = g.nx, ny = g.ny, P = g.P, TY = g.TY;
    const bool x0 = th > 0 && i >= 1 && i <= th, xm = th > 0 && i >= nx - th;
    const bool fxr = x0 || xm;
    const int kx = x0 ? th - i : i - (nx - th);
    const long long pxo = (long long)(x0 ? kx : th + kx) * P;
    float cd[N], px[N], py[N];
    bool fy0[N], fym[N];
#pragma unroll
    for (int n = 0; n < N; ++n) {
        const int j = j0 + n;
        const bool ok = j < ny;
        fy0[n] = th > 0 && ok && j >= 1 && j <= th;
        fym[n] = th > 0 && ok && j >= ny - th;
        const bool fx = fxr && ok;
        cd[n] = (fx || fy0[n] || fym[n]) ? ldro(g, g.cd + (long long)i * P + j + PADC) : 0.f;
        px[n] = fx ? ldro(g, rd.ex + (pxo + j) * CS + l) : 0.f;
        py[n] = fy0[n] ? ldro(g, rd.ey + ((long long)i * TY + (th - j)) * CS + l)
                       : (fym[n] ? ldro(g, rd.ey + ((long long)(nx + 1 + i) * TY + (j - (ny - th))) * CS + l) : 0.f);
    }
#pragma unroll
    for (int n = 0; n < N; ++n) {
        const int j = j0 + n;
        if (j >= ny) continue;
        float e = ez[n];
        if (i >= 1 && j >= 1) e = __fmaf_rn(-cb[n], dhx[n], madd2(ca[n], e, cb[n], dhy[n]));
        const bool fy = fy0[n] || fym[n];
        const int ky = fy0[n] ? th - j : j - (ny - th);
        if (fxr && !(xm && fy0[n])) e = cpml<true>(g, e, div_d(g, dhy[n]), cd[n], px[n], R, kx);
        if (fy) e = cpml<false>(g, e, div_d(g, dhx[n]), cd[n], py[n], R, ky);
        if (xm && fy0[n]) e = cpml<true>(g, e, div_d(g, dhy[n]), cd[n], px[n], R, kx);
        ez[n] = e;
    }
    if (!own_row) return;
#pragma unroll
    for (int n = 0; n < N; ++n) {
        const int j = j0 + n;
        if (n >= nown || j >= ny) continue;
        if (fxr) st1(g, wr.ex + (pxo + j) * CS + l, px[n]);
        if (fy0[n]) st1(g, wr.ey + ((long long)i * TY + (th - j)) * CS + l, py[n]);
        if (fym[n]) st1(g, wr.ey + ((long long)(nx + 1 + i) * TY + (j - (ny - th))) * CS + l, py[n]);
    }
}

// Hx of cells (i, j0 + n): interior (i >= 1) then the y slabs; auxiliaries of
// cells n >= own0 are stored.
template <int N, int CS>
__device__ __forceinline__ void hx_cells(const Dev& g, const float* R, int i, int j0, int l, float* hx,
                                         const float* dzx, const float* ch, int own0, const PsiG& rd,
                                         const PsiG& wr) {
    const int th = g.th, nx = g.nx, ny = g.ny, P = g.P, TY = g.TY;
    const float* HR = R + 4 * th;
    float ci[N], py[N];
    bool fy0[N], fym[N];
#pragma unroll
    for (int n = 0; n < N; ++n) {
        const int j = j0 + n;
        const bool ok = j >= 0 && j < ny;
        fy0[n] = th > 0 && ok && j <= th - 1;
        fym[n] = th > 0 && ok && j >= ny - th;
        ci[n] = (fy0[n] || fym[n]) ? ldro(g, g.ci + (long long)i * P + j + PADC) : 0.f;
        py[n] = fy0[n] ? ldro(g, rd.hy + ((long long)i * TY + (th - 1 - j)) * CS + l)
                       : (fym[n] ? ldro(g, rd.hy + ((long long)(nx + 1 + i) * TY + (j - (ny - th))) * CS + l) : 0.f);
    }
#pragma unroll
    for (int n = 0; n < N; ++n) {
        const int j = j0 + n;
        if (j < 0 || j >= ny) continue;
        float h = hx[n];
        if (i >= 1) h = msub2(1.0f, h, ch[n], dzx[n]);
        if (fy0[n] || fym[n]) {
            const int ky = fy0[n] ? th - 1 - j : j - (ny - th);
            h = cpml<false>(g, h, div_d(g, dzx[n]), ci[n], py[n], HR, ky);
        }
        hx[n] = h;
    }
#pragma unroll
    for (int n = 0; n < N; ++n) {
        const int j = j0 + n;
        if (n < own0 || j < 0 || j >= ny) continue;
        if (fy0[n]) st1(g, wr.hy + ((long long)i * TY + (th - 1 - j)) * CS + l, py[n]);
        if (fym[n]) st1(g, wr.hy + ((long long)(nx + 1 + i) * TY + (j - (ny - th))) * CS + l, py[n]);
    }
}

// Hy of cells (i, j0 + n): interior (j >= 1) then the x slabs (row-uniform);
// auxiliaries stored when STORE.
template <int N, int CS, bool STORE>
__device__ __forceinline__ void hy_cells(const Dev& g, const float* R, int i, int j0, int l, float* hy,
                                         const float* dzy, const float* ch, const PsiG& rd, const PsiG& wr) {
    const int th = g.th, nx = g.nx, ny = g.ny, P = g.P;
    const float* HR = R + 4 * th;
    const bool x0 = th > 0 && i <= th - 1, xm = th > 0 && i >= nx - th;
    const bool fxr = x0 || xm;
    const int kx = x0 ? th - 1 - i : i - (nx - th);
    const long long pxo = (long long)(x0 ? kx : th + kx) * P;
    float ci[N], px[N];
#pragma unroll
    for (int n = 0; n < N; ++n) {
        const int j = j0 + n;
        const bool fx = fxr && j < ny;
        ci[n] = fx ? ldro(g, g.ci + (long long)i * P + j + PADC) : 0.f;
        px[n] = fx ? ldro(g, rd.hx + (pxo + j) * CS + l) : 0.f;
    }
#pragma unroll
    for (int n = 0; n < N; ++n) {
        const int j = j0 + n;
        if (j >= ny) continue;
        float h = hy[n];
        if (j >= 1) h = madd2(1.0f, h, ch[n], dzy[n]);
        if (fxr) h = cpml<true>(g, h, div_d(g, dzy[n]), ci[n], px[n], HR, kx);
        hy[n] = h;
    }
    if constexpr (STORE) {
        if (!fxr) return;
#pragma unroll
        for (int n = 0; n < N; ++n) {
            const int j = j0 + n;
            if (j < ny) st1(g, wr.hx + (pxo + j) * CS + l, px[n]);
        }
    }
}

}  // namespace fg
