// Device-side pieces shared by the TMz FDTD kernels: the per-solve grid
// descriptor, guarded global accesses, and the per-cell update arithmetic.
//
// Per-cell arithmetic follows the reference kernels (paths relative to the
// reference project):
//   interior E  src/lib/fields_updates_gpu.cu:124-134
//   interior H  src/lib/fields_updates_gpu.cu:162-180
//   CPML E      src/lib/pml_updates_e.cu:58-76 (x), 267-285 (y) and the plus sides
//   CPML H      src/lib/pml_updates_h.cu:37-54 (x), 273-290 (y) and the plus sides
// The library is compiled with -fmad=false, so every fused multiply-add below
// is an explicit __fmaf_rn and nothing else is contracted.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fg {

constexpr unsigned FULL = 0xffffffffu;

// Event: something that happens to one cell of one shot at one row of a tile
// (a receiver sample, a source injection, an adjoint residual injection).
// x = row i, y = shot slot within the warp's shot group, z = column j, w = index
// (receiver r or source n).
using Ev = int4;

struct GridDev {
    // geometry
    int nx, ny;          // compute grid; row nx and column ny are the zero frame
    int P;               // row pitch of field / coefficient planes (floats, multiple of 32)
    int th;              // CPML thickness
    int TY;              // row pitch of y-slab CPML auxiliaries (>= th)
    int S, nt, nrx;      // shots, time steps, receivers per shot
    int Ph;              // row pitch of the Ez history (floats, multiple of 4, >= ny)
    float d;             // cell size (CPML derivative divisor)
    float dt;            // time step (sigma imaging factor)
    long long plane;     // floats in one (nx+1) x P plane
    long long pxs, pys;  // per-shot floats of x-slab / y-slab auxiliaries
    // coefficient planes: uE0 (or Ucgeta's uE0), uE1, uE4, uH1, uH4
    const float *ca, *cb, *cd, *ch, *ci;
    const float* pml;    // (8, th): ERA ERB ERE ERF HRA HRB HRE HRF
    // state, ping-pong pairs; index 0/1 = parity
    float *ez[2], *hx[2], *hy[2];
    float *pex[2], *pey[2], *phx[2], *phy[2];
    // tiling
    int nb, nc, G, ngroups, ntiles;
    const int* chunk_row;               // (nc+1) row boundaries
    const Ev* src_ev; const int* src_off;   // forward sources per tile
    const Ev* rx_ev;  const int* rx_off;    // forward receivers per tile
    const Ev* inj_ev; const int* inj_off;   // adjoint injections, rows [i0, i1]
    const Ev* injh_ev; const int* injh_off; // adjoint injections on the halo column
    const float* srcw;   // (nsrc, nt)
    // solve I/O
    float* traces;       // (S, nt, nrx)
    float* hist;         // (nt, S, nx, ny)
    const float* resid;  // (S, nt, nrx)
    double* gacc;        // (ngroups, 2, nx, ny)
    // bounds of every buffer the kernels touch (checked builds)
    const char* ws_lo; const char* ws_hi;
    const char* out_lo; const char* out_hi;   // the history buffer
    int* err;            // device error word
};

#ifdef FG_CHECKED
// Checked build: every global access is tested against the workspace or the
// caller buffer it belongs to; a violation records a code and the access is
// skipped (loads return 0), so a logic error never becomes a memory fault.
__device__ __forceinline__ bool in_ws(const GridDev& g, const void* p, int bytes) {
    const char* c = (const char*)p;
    if (c >= g.ws_lo && c + bytes <= g.ws_hi) return true;
    if (g.out_lo && c >= g.out_lo && c + bytes <= g.out_hi) return true;
    atomicCAS(g.err, 0, 100);
    return false;
}
#define FG_WS_OK(g, p, bytes) in_ws((g), (p), (bytes))
#else
#define FG_WS_OK(g, p, bytes) true
#endif

template <int V> struct VecT;
template <> struct VecT<1> { using T = float; };
template <> struct VecT<2> { using T = float2; };
template <> struct VecT<4> { using T = float4; };

// Coherent (L2) load of V floats from a state buffer.
template <int V>
__device__ __forceinline__ void ld_state(const GridDev& g, float (&x)[V], const float* p) {
    if (!FG_WS_OK(g, p, 4 * V)) {
#pragma unroll
        for (int v = 0; v < V; ++v) x[v] = 0.f;
        return;
    }
    if constexpr (V == 4) {
        const float4 q = __ldcg(reinterpret_cast<const float4*>(p));
        x[0] = q.x; x[1] = q.y; x[2] = q.z; x[3] = q.w;
    } else if constexpr (V == 2) {
        const float2 q = __ldcg(reinterpret_cast<const float2*>(p));
        x[0] = q.x; x[1] = q.y;
    } else {
        x[0] = __ldcg(p);
    }
}

// Read-only (coefficient) load of V floats.
template <int V>
__device__ __forceinline__ void ld_coef(const GridDev& g, float (&x)[V], const float* p) {
    if (!FG_WS_OK(g, p, 4 * V)) {
#pragma unroll
        for (int v = 0; v < V; ++v) x[v] = 0.f;
        return;
    }
    if constexpr (V == 4) {
        const float4 q = __ldg(reinterpret_cast<const float4*>(p));
        x[0] = q.x; x[1] = q.y; x[2] = q.z; x[3] = q.w;
    } else if constexpr (V == 2) {
        const float2 q = __ldg(reinterpret_cast<const float2*>(p));
        x[0] = q.x; x[1] = q.y;
    } else {
        x[0] = __ldg(p);
    }
}

template <int V>
__device__ __forceinline__ void st_state(const GridDev& g, float* p, const float (&x)[V]) {
    if (!FG_WS_OK(g, p, 4 * V)) return;
    if constexpr (V == 4) {
        __stcg(reinterpret_cast<float4*>(p), make_float4(x[0], x[1], x[2], x[3]));
    } else if constexpr (V == 2) {
        __stcg(reinterpret_cast<float2*>(p), make_float2(x[0], x[1]));
    } else {
        __stcg(p, x[0]);
    }
}

__device__ __forceinline__ float ld1(const GridDev& g, const float* p) {
    if (!FG_WS_OK(g, p, 4)) return 0.f;
    return __ldcg(p);
}
__device__ __forceinline__ float ldc1(const GridDev& g, const float* p) {
    if (!FG_WS_OK(g, p, 4)) return 0.f;
    return __ldg(p);
}
__device__ __forceinline__ void st1(const GridDev& g, float* p, float x) {
    if (!FG_WS_OK(g, p, 4)) return;
    __stcg(p, x);
}

// a*b + c*d with the first product fused, a*b - c*d likewise.
__device__ __forceinline__ float madd2(float a, float b, float c, float d) {
    return __fmaf_rn(a, b, __fmul_rn(c, d));
}
__device__ __forceinline__ float msub2(float a, float b, float c, float d) {
    return __fmaf_rn(a, b, -__fmul_rn(c, d));
}

// One HORIPML order-1 correction: F +-= u4*((RA-1)*D + RB*psi); psi = RE*psi - RF*D.
// R points at the 4 coefficient vectors (RA, RB, RE, RF) of length th.
template <bool PLUS>
__device__ __forceinline__ float cpml(const GridDev& g, float f, float deriv, float u4, float& psi,
                                      const float* R, int k) {
    const int th = g.th;
    const float ra1 = __fsub_rn(ldc1(g, R + k), 1.0f);
    const float rb = ldc1(g, R + th + k);
    const float re = ldc1(g, R + 2 * th + k);
    const float rf = ldc1(g, R + 3 * th + k);
    const float t = madd2(ra1, deriv, rb, psi);
    const float out = __fmaf_rn(PLUS ? u4 : -u4, t, f);
    psi = msub2(re, psi, rf, deriv);
    return out;
}

// Per-shot views of the CPML auxiliaries for one parity.
struct PsiShot {
    float *ex, *ey, *hx, *hy;  // E x-slabs, E y-slabs, H x-slabs (Hy), H y-slabs (Hx)
};
__device__ __forceinline__ PsiShot psi_shot(const GridDev& g, int par, int s) {
    PsiShot p;
    p.ex = g.pex[par] + (long long)s * g.pxs;
    p.ey = g.pey[par] + (long long)s * g.pys;
    p.hx = g.phx[par] + (long long)s * g.pxs;
    p.hy = g.phy[par] + (long long)s * g.pys;
    return p;
}

// E update of cell (i, j) of one shot: interior leapfrog (i>=1, j>=1) then the
// CPML corrections in the reference's slab order x0, y0, xmax, ymax.
//   dhy = Hy[i][j] - Hy[i-1][j], dhx = Hx[i][j] - Hx[i][j-1] (new H values)
// The auxiliaries are read from `rd` and, when STORE, written to `wr`.
template <bool STORE>
__device__ __forceinline__ float e_update(const GridDev& g, int i, int j, float ez, float dhy, float dhx,
                                          float ca, float cb, const PsiShot& rd, const PsiShot& wr) {
    if (i >= 1 && j >= 1) ez = __fmaf_rn(-cb, dhx, madd2(ca, ez, cb, dhy));
    const int th = g.th;
    if (th > 0) {
        const int P = g.P, nx = g.nx, ny = g.ny;
        const bool x0 = (i >= 1 && i <= th), xm = (i >= nx - th);
        const bool y0 = (j >= 1 && j <= th), ym = (j >= ny - th);
        if (x0 | xm | y0 | ym) {
            const float cd = ldc1(g, g.cd + (long long)i * P + j);
            if (x0) {
                const int k = th - i;
                const long long o = (long long)k * P + j;
                float psi = ld1(g, rd.ex + o);
                ez = cpml<true>(g, ez, __fdiv_rn(dhy, g.d), cd, psi, g.pml, k);
                if (STORE) st1(g, wr.ex + o, psi);
            }
            if (y0) {
                const int k = th - j;
                const long long o = (long long)i * g.TY + k;
                float psi = ld1(g, rd.ey + o);
                ez = cpml<false>(g, ez, __fdiv_rn(dhx, g.d), cd, psi, g.pml, k);
                if (STORE) st1(g, wr.ey + o, psi);
            }
            if (xm) {
                const int k = i - (nx - th);
                const long long o = (long long)(th + k) * P + j;
                float psi = ld1(g, rd.ex + o);
                ez = cpml<true>(g, ez, __fdiv_rn(dhy, g.d), cd, psi, g.pml, k);
                if (STORE) st1(g, wr.ex + o, psi);
            }
            if (ym) {
                const int k = j - (ny - th);
                const long long o = (long long)(nx + 1 + i) * g.TY + k;
                float psi = ld1(g, rd.ey + o);
                ez = cpml<false>(g, ez, __fdiv_rn(dhx, g.d), cd, psi, g.pml, k);
                if (STORE) st1(g, wr.ey + o, psi);
            }
        }
    }
    return ez;
}

// H update of cell (i, j) of one shot.
//   dzx = Ez[i][j+1] - Ez[i][j] (drives Hx), dzy = Ez[i+1][j] - Ez[i][j] (drives Hy)
template <bool STORE, bool DO_HX, bool DO_HY>
__device__ __forceinline__ void h_update(const GridDev& g, int i, int j, float& hx, float& hy, float dzx,
                                         float dzy, float ch, const PsiShot& rd, const PsiShot& wr) {
    if (DO_HX && i >= 1) hx = msub2(1.0f, hx, ch, dzx);
    if (DO_HY && j >= 1) hy = madd2(1.0f, hy, ch, dzy);
    const int th = g.th;
    if (th > 0) {
        const int P = g.P, nx = g.nx, ny = g.ny;
        const bool x0 = DO_HY && (i <= th - 1), xm = DO_HY && (i >= nx - th);
        const bool y0 = DO_HX && (j <= th - 1), ym = DO_HX && (j >= ny - th);
        if (x0 | xm | y0 | ym) {
            const float ci = ldc1(g, g.ci + (long long)i * P + j);
            const float* HR = g.pml + 4 * th;
            if (x0) {
                const int k = th - 1 - i;
                const long long o = (long long)k * P + j;
                float psi = ld1(g, rd.hx + o);
                hy = cpml<true>(g, hy, __fdiv_rn(dzy, g.d), ci, psi, HR, k);
                if (STORE) st1(g, wr.hx + o, psi);
            }
            if (y0) {
                const int k = th - 1 - j;
                const long long o = (long long)i * g.TY + k;
                float psi = ld1(g, rd.hy + o);
                hx = cpml<false>(g, hx, __fdiv_rn(dzx, g.d), ci, psi, HR, k);
                if (STORE) st1(g, wr.hy + o, psi);
            }
            if (xm) {
                const int k = i - (nx - th);
                const long long o = (long long)(th + k) * P + j;
                float psi = ld1(g, rd.hx + o);
                hy = cpml<true>(g, hy, __fdiv_rn(dzy, g.d), ci, psi, HR, k);
                if (STORE) st1(g, wr.hx + o, psi);
            }
            if (ym) {
                const int k = j - (ny - th);
                const long long o = (long long)(nx + 1 + i) * g.TY + k;
                float psi = ld1(g, rd.hy + o);
                hx = cpml<false>(g, hx, __fdiv_rn(dzx, g.d), ci, psi, HR, k);
                if (STORE) st1(g, wr.hy + o, psi);
            }
        }
    }
}

}  // namespace fg
