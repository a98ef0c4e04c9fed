// Shot-lane CPML rows.  In a shot-lane solve the 32 lanes of a warp are 32
// shots of the same cells, so every slab test of a row is warp-uniform.  The
// functions below update one row of a band outside the interior core with
// every CPML operand of the row (uE4 / uH4 coefficients and the auxiliaries
// of every slab the row touches) loaded before the first update, so a CPML
// row costs one memory round trip.  The y-slab geometry of a band (which of
// its cells lie in a y slab and where their auxiliaries sit) is computed once
// per tile.  Arithmetic, update domains and the slab order per cell (x0, y0,
// xmax, ymax) are those of e_cell / hx_cell / hy_cell and of the reference
// kernels they cite (src/lib/pml_updates_e.cu, src/lib/pml_updates_h.cu).
#pragma once

#include "fdtd_common.cuh"

namespace fg {

// Cells c0 .. c0+N-1 of a row, as one E or H update sees them.
//   in: bit n set when 0 <= c0+n < ny
//   m:  bit n set when cell n lies in a y slab of this update
// A cell n of m has slab column k0 + dk*n and slab row i + off (off = 0 for
// the y0 slab, nx+1 for the ymax slab).  one_side is false when the run has
// cells in both y slabs (a grid narrower than 2 th + 8); those bands take the
// generic per-cell path.
struct YRun {
    uint32_t in, m;
    int k0, dk, off;
    bool one_side;
};

// E: y0 slab j in [1, th] (k = th - j); H: j in [0, th-1] (k = th-1-j); both:
// ymax slab j >= ny - th (k = j - (ny - th)).
template <int N>
__device__ __forceinline__ YRun y_run(const Dev& g, int c0, bool efield) {
    const int th = g.th, ny = g.ny;
    uint32_t in = 0, lo = 0, hi = 0;
#pragma unroll
    for (int n = 0; n < N; ++n) {
        const int j = c0 + n;
        const bool ok = j >= 0 && j < ny;
        in |= (uint32_t)ok << n;
        if (th > 0 && ok) {
            lo |= (uint32_t)(efield ? (j >= 1 && j <= th) : (j <= th - 1)) << n;
            hi |= (uint32_t)(j >= ny - th) << n;
        }
    }
    YRun y;
    y.in = in;
    y.one_side = !(lo && hi);
    if (lo) {
        y.m = lo;
        y.k0 = (efield ? th : th - 1) - c0;
        y.dk = -1;
        y.off = 0;
    } else {
        y.m = hi;
        y.k0 = c0 - (ny - th);
        y.dk = 1;
        y.off = g.nx + 1;
    }
    return y;
}

// Row i as one E or H update sees it: whether it lies in an x slab, which
// one, its profile index and its row in the x-slab arrays.
//   E: x0 slab i in [1, th] (k = th - i); H: i in [0, th-1] (k = th-1-i);
//   both: xmax slab i >= nx - th (k = i - (nx - th)); slab row k (x0) or th + k.
struct XRow {
    bool on, maxside;
    int k, r;
};
__device__ __forceinline__ XRow x_row(const Dev& g, int i, bool efield) {
    const int th = g.th, nx = g.nx;
    const bool lo = th > 0 && (efield ? (i >= 1 && i <= th) : (i <= th - 1));
    const bool hi = th > 0 && i >= nx - th;
    XRow x;
    x.on = lo || hi;
    x.maxside = hi && !lo;
    x.k = lo ? (efield ? th - i : th - 1 - i) : i - (nx - th);
    x.r = lo ? x.k : th + x.k;
    return x;
}

// y-slab geometry of a band: the H run and the E run of its rows.
//   forward: Hx at j0-1 .. j0+W-1 (W+1 cells), Hy and E at j0 .. j0+W-1
//   adjoint: E at j0 .. j0+W (W+1 cells), Hx and Hy at j0 .. j0+W-1
struct BandY {
    YRun h, e;
    bool lean;   // the shot-lane CPML rows apply (fast_cpml and one-sided runs)
};
__device__ __forceinline__ uint32_t low_bits(int n) { return n >= 32 ? 0xffffffffu : ((1u << n) - 1u); }
template <int W>
__device__ __forceinline__ BandY band_fwd(const Dev& g, int j0) {
    BandY b;
    b.h = y_run<W + 1>(g, j0 - 1, false);
    b.e = y_run<W>(g, j0, true);
    b.lean = g.fast_cpml && b.h.one_side && b.e.one_side;
    return b;
}
template <int W>
__device__ __forceinline__ BandY band_adj(const Dev& g, int j0) {
    BandY b;
    b.h = y_run<W>(g, j0, false);
    b.e = y_run<W + 1>(g, j0, true);
    b.lean = g.fast_cpml && b.h.one_side && b.e.one_side;
    return b;
}

__device__ __forceinline__ bool bit(uint32_t m, int n) { return (m >> n) & 1u; }

// Auxiliaries of the cells of a y run (slab array a, row i): lane's shot slot.
template <int N>
__device__ __forceinline__ void ld_yrun(const Dev& g, const float* a, int i, const YRun& y, int lane, float (&p)[N]) {
    const float* b = a + ((long long)(i + y.off) * g.TY + y.k0) * 32 + lane;
    const int step = 32 * y.dk;
#pragma unroll
    for (int n = 0; n < N; ++n) p[n] = bit(y.m, n) ? ldro(g, b + n * step) : 0.f;
}
template <int N>
__device__ __forceinline__ void st_yrun(const Dev& g, float* a, int i, const YRun& y, uint32_t own, int lane,
                                        const float (&p)[N]) {
    float* b = a + ((long long)(i + y.off) * g.TY + y.k0) * 32 + lane;
    const int step = 32 * y.dk;
#pragma unroll
    for (int n = 0; n < N; ++n)
        if (bit(y.m & own, n)) st1(g, b + n * step, p[n]);
}
// Auxiliaries of cells c0 .. c0+N-1 (those of mask `in`) in x-slab row r.
template <int N>
__device__ __forceinline__ void ld_xrun(const Dev& g, const float* a, int r, int c0, uint32_t in, int lane,
                                        float (&p)[N]) {
    const float* b = a + ((long long)r * g.P + c0) * 32 + lane;
#pragma unroll
    for (int n = 0; n < N; ++n) p[n] = bit(in, n) ? ldro(g, b + n * 32) : 0.f;
}
template <int N>
__device__ __forceinline__ void st_xrun(const Dev& g, float* a, int r, int c0, uint32_t own, int lane,
                                        const float (&p)[N]) {
    float* b = a + ((long long)r * g.P + c0) * 32 + lane;
#pragma unroll
    for (int n = 0; n < N; ++n)
        if (bit(own, n)) st1(g, b + n * 32, p[n]);
}

// Division of a row by the cell size, decided once per row.  div_d tests the
// range of every x and branches per lane to __fdiv_rn; inside the unrolled
// CPML rows those tests and branches cost more than the arithmetic.  Where
// the plan's divisor passed k_div_check_scaled, div_d_scaled is __fdiv_rn's
// quotient for every |x| < 2^31: one warp vote per row asks whether every
// input the row divides is below that (NaN is not), and the row then runs
// straight-line with div_d_scaled, or with div_d throughout.  All 32 lanes
// are active: they are 32 shots of the same cells.
template <int N>
__device__ __forceinline__ bool div_row_fast(const Dev& g, uint32_t m, const float (&x)[N]) {
    bool bad = false;
#pragma unroll
    for (int n = 0; n < N; ++n)
        if (bit(m, n)) bad |= !(fabsf(x[n]) < 0x1p31f);
    return g.div_scaled && !__any_sync(0xffffffffu, bad);
}
template <bool FAST>
__device__ __forceinline__ float div_row(const Dev& g, float x) {
    if constexpr (FAST) return div_d_scaled(x, g.d, g.dinv);
    else return div_d(g, x);
}

// E of cells j0 .. j0+N-1 of row i from dhy / dhx (old E in ez, updated in
// place): interior (i >= 1, j >= 1), then the CPML corrections in slab order.
// cd / px / py are the row's loaded uE4 and auxiliaries (px, py updated).
template <int N, bool FAST>
__device__ __forceinline__ void e_shot_k(const Dev& g, const float* R, int i, int j0, const XRow& xe, const YRun& ye,
                                         float (&ez)[N], const float (&dhy)[N], const float (&dhx)[N], const float* ca,
                                         const float* cb, const float (&cd)[N], float (&px)[N], float (&py)[N]) {
    const int th = g.th;
    float xa = 0.f, xb = 0.f, xc = 0.f, xf = 0.f;
    if (xe.on) {
        xa = __fsub_rn(R[xe.k], 1.0f);
        xb = R[th + xe.k];
        xc = R[2 * th + xe.k];
        xf = R[3 * th + xe.k];
    }
#pragma unroll
    for (int n = 0; n < N; ++n) {
        if (!bit(ye.in, n)) continue;
        float e = ez[n];
        if (i >= 1 && j0 + n >= 1) e = __fmaf_rn(-cb[n], dhx[n], madd2(ca[n], e, cb[n], dhy[n]));
        const bool fy = bit(ye.m, n);
        // x0 and xmax come before and after y0 in the slab order; ymax is last
        const bool late_x = xe.maxside && fy && ye.off == 0;
        if (xe.on && !late_x) {
            const float dd = div_row<FAST>(g, dhy[n]);
            e = __fmaf_rn(cd[n], madd2(xa, dd, xb, px[n]), e);
            px[n] = msub2(xc, px[n], xf, dd);
        }
        if (fy) e = cpml<false>(g, e, div_row<FAST>(g, dhx[n]), cd[n], py[n], R, ye.k0 + ye.dk * n);
        if (late_x) {
            const float dd = div_row<FAST>(g, dhy[n]);
            e = __fmaf_rn(cd[n], madd2(xa, dd, xb, px[n]), e);
            px[n] = msub2(xc, px[n], xf, dd);
        }
        ez[n] = e;
    }
}
template <int N>
__device__ __forceinline__ void e_shot(const Dev& g, const float* R, int i, int j0, const XRow& xe, const YRun& ye,
                                       float (&ez)[N], const float (&dhy)[N], const float (&dhx)[N], const float* ca,
                                       const float* cb, const float (&cd)[N], float (&px)[N], float (&py)[N]) {
    if (div_row_fast<N>(g, xe.on ? ye.in : 0u, dhy) && div_row_fast<N>(g, ye.m & ye.in, dhx))
        e_shot_k<N, true>(g, R, i, j0, xe, ye, ez, dhy, dhx, ca, cb, cd, px, py);
    else
        e_shot_k<N, false>(g, R, i, j0, xe, ye, ez, dhy, dhx, ca, cb, cd, px, py);
}

// Hx of cells c0 .. c0+N-1 of row i (old Hx in h, updated in place):
// interior (i >= 1), then the y-slab correction.
template <int N, bool FAST>
__device__ __forceinline__ void hx_shot_k(const Dev& g, const float* R, int i, const YRun& yh, float (&h)[N],
                                          const float (&dz)[N], const float* ch, const float (&ci)[N], float (&py)[N]) {
    const float* HR = R + 4 * g.th;
#pragma unroll
    for (int n = 0; n < N; ++n) {
        if (!bit(yh.in, n)) continue;
        float v = h[n];
        if (i >= 1) v = msub2(1.0f, v, ch[n], dz[n]);
        if (bit(yh.m, n)) v = cpml<false>(g, v, div_row<FAST>(g, dz[n]), ci[n], py[n], HR, yh.k0 + yh.dk * n);
        h[n] = v;
    }
}
template <int N>
__device__ __forceinline__ void hx_shot(const Dev& g, const float* R, int i, const YRun& yh, float (&h)[N],
                                        const float (&dz)[N], const float* ch, const float (&ci)[N], float (&py)[N]) {
    if (div_row_fast<N>(g, yh.m & yh.in, dz))
        hx_shot_k<N, true>(g, R, i, yh, h, dz, ch, ci, py);
    else
        hx_shot_k<N, false>(g, R, i, yh, h, dz, ch, ci, py);
}

// Hy of cells j0 .. j0+N-1 of row i (validity mask `in`): interior (j >= 1),
// then the x-slab correction (row-uniform profile index).
template <int N, bool FAST>
__device__ __forceinline__ void hy_shot_k(const Dev& g, const float* R, int j0, const XRow& xh, uint32_t in,
                                          float (&h)[N], const float (&dz)[N], const float* ch, const float* ci,
                                          float (&px)[N]) {
    const int th = g.th;
    const float* HR = R + 4 * th;
    float xa = 0.f, xb = 0.f, xc = 0.f, xf = 0.f;
    if (xh.on) {
        xa = __fsub_rn(HR[xh.k], 1.0f);
        xb = HR[th + xh.k];
        xc = HR[2 * th + xh.k];
        xf = HR[3 * th + xh.k];
    }
#pragma unroll
    for (int n = 0; n < N; ++n) {
        if (!bit(in, n)) continue;
        float v = h[n];
        if (j0 + n >= 1) v = madd2(1.0f, v, ch[n], dz[n]);
        if (xh.on) {
            const float dd = div_row<FAST>(g, dz[n]);
            v = __fmaf_rn(ci[n], madd2(xa, dd, xb, px[n]), v);
            px[n] = msub2(xc, px[n], xf, dd);
        }
        h[n] = v;
    }
}
template <int N>
__device__ __forceinline__ void hy_shot(const Dev& g, const float* R, int j0, const XRow& xh, uint32_t in,
                                        float (&h)[N], const float (&dz)[N], const float* ch, const float* ci,
                                        float (&px)[N]) {
    if (div_row_fast<N>(g, xh.on ? in : 0u, dz))
        hy_shot_k<N, true>(g, R, j0, xh, in, h, dz, ch, ci, px);
    else
        hy_shot_k<N, false>(g, R, j0, xh, in, h, dz, ch, ci, px);
}

// uE4 / uH4 of cells c0 .. c0+N-1 of row i that `need` them.
template <int N>
__device__ __forceinline__ void ld_coef_mask(const Dev& g, const float* plane, int i, int c0, uint32_t need,
                                             float (&c)[N]) {
    const float* b = plane + (long long)i * g.P + c0 + PADC;
#pragma unroll
    for (int n = 0; n < N; ++n) c[n] = bit(need, n) ? ldro(g, b + n) : 0.f;
}

// ---------------------------------------------------------------------------
// Forward row i of a band (columns j0 .. j0+W-1) outside the interior core:
// Hx at j0-1 .. j0+W-1 (the first is the halo column: its auxiliary is read,
// not stored), Hy and E at j0 .. j0+W-1.
// ---------------------------------------------------------------------------
template <int W>
__device__ __forceinline__ void fwd_row_shot(const Dev& g, const float* R, const BandY& by, int i, int j0, int lane,
                                             const float (&hxo)[W + 1], const float (&hyo)[W], const float (&en)[W + 2],
                                             const float (&ezc)[W + 2], const float (&hyu)[W], const float* ca,
                                             const float* cb, const float* ch, const PsiG& rd, const PsiG& wr,
                                             float (&hxn)[W + 1], float (&hyn)[W], float (&ezn)[W]) {
    const XRow xh = x_row(g, i, false), xe = x_row(g, i, true);
    const uint32_t ein = by.e.in;
    // every CPML operand of the row
    float ci[W + 1], cd[W], pyh[W + 1], pxh[W], pxe[W], pye[W];
    ld_coef_mask<W + 1>(g, g.ci, i, j0 - 1, by.h.m | (xh.on ? (ein << 1) : 0u), ci);
    ld_coef_mask<W>(g, g.cd, i, j0, (xe.on ? ein : 0u) | by.e.m, cd);
    ld_yrun<W + 1>(g, rd.hy, i, by.h, lane, pyh);
    ld_xrun<W>(g, rd.hx, xh.r, j0, xh.on ? ein : 0u, lane, pxh);
    ld_xrun<W>(g, rd.ex, xe.r, j0, xe.on ? ein : 0u, lane, pxe);
    ld_yrun<W>(g, rd.ey, i, by.e, lane, pye);
    float dzx[W + 1], dzy[W];
#pragma unroll
    for (int n = 0; n <= W; ++n) {
        hxn[n] = hxo[n];
        dzx[n] = __fsub_rn(ezc[n + 1], ezc[n]);
    }
    hx_shot<W + 1>(g, R, i, by.h, hxn, dzx, ch, ci, pyh);
#pragma unroll
    for (int w = 0; w < W; ++w) {
        hyn[w] = hyo[w];
        dzy[w] = __fsub_rn(en[w + 1], ezc[w + 1]);
    }
    hy_shot<W>(g, R, j0, xh, ein, hyn, dzy, ch + 1, ci + 1, pxh);
    float dhy[W], dhx[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
        ezn[w] = ezc[w + 1];
        dhy[w] = __fsub_rn(hyn[w], hyu[w]);
        dhx[w] = __fsub_rn(hxn[w + 1], hxn[w]);
    }
    e_shot<W>(g, R, i, j0, xe, by.e, ezn, dhy, dhx, ca, cb, cd, pxe, pye);
    st_yrun<W + 1>(g, wr.hy, i, by.h, ~1u, lane, pyh);
    if (xh.on) st_xrun<W>(g, wr.hx, xh.r, j0, ein, lane, pxh);
    if (xe.on) st_xrun<W>(g, wr.ex, xe.r, j0, ein, lane, pxe);
    st_yrun<W>(g, wr.ey, i, by.e, ~0u, lane, pye);
}

// Hy of row i-1 above a forward chunk (cells j0 .. j0+W-1): its auxiliaries
// are only read (the tile of that row stores them).
template <int W>
__device__ __forceinline__ void fwd_hy_halo_shot(const Dev& g, const float* R, const BandY& by, int i, int j0,
                                                 int lane, float (&hy)[W], const float (&dz)[W], const float* ch,
                                                 const PsiG& rd) {
    const XRow xh = x_row(g, i, false);
    const uint32_t in = xh.on ? by.e.in : 0u;
    float ci[W], px[W];
    ld_coef_mask<W>(g, g.ci, i, j0, in, ci);
    ld_xrun<W>(g, rd.hx, xh.r, j0, in, lane, px);
    hy_shot<W>(g, R, j0, xh, by.e.in, hy, dz, ch, ci, px);
}

// ---------------------------------------------------------------------------
// Adjoint rows (reference mode: the forward operator with Ucgeta's uE0)
// ---------------------------------------------------------------------------

// New E of row r, cells j0 .. j0+W (column j0+W is the halo): auxiliaries of
// the first W cells are stored when `own_row`.
template <int W>
__device__ __forceinline__ void adj_e_row_shot(const Dev& g, const float* R, const BandY& by, int r, int j0, int lane,
                                               bool own_row, const float* ez, const float* hxo, const float* hyo,
                                               const float* hyu, const float* ca, const float* cb,
                                               const PsiG& rd, const PsiG& wr, float (&out)[W + 1]) {
    const XRow xe = x_row(g, r, true);
    const uint32_t ein = by.e.in;
    float cd[W + 1], px[W + 1], py[W + 1];
    ld_coef_mask<W + 1>(g, g.cd, r, j0, (xe.on ? ein : 0u) | by.e.m, cd);
    ld_xrun<W + 1>(g, rd.ex, xe.r, j0, xe.on ? ein : 0u, lane, px);
    ld_yrun<W + 1>(g, rd.ey, r, by.e, lane, py);
    float dhy[W + 1], dhx[W + 1];
#pragma unroll
    for (int n = 0; n <= W; ++n) {
        out[n] = ez[n];
        dhy[n] = __fsub_rn(hyo[n], hyu[n]);
        dhx[n] = __fsub_rn(hxo[n + 1], hxo[n]);
    }
    e_shot<W + 1>(g, R, r, j0, xe, by.e, out, dhy, dhx, ca, cb, cd, px, py);
    if (!own_row) return;
    const uint32_t own = low_bits(W);
    if (xe.on) st_xrun<W + 1>(g, wr.ex, xe.r, j0, ein & own, lane, px);
    st_yrun<W + 1>(g, wr.ey, r, by.e, own, lane, py);
}

// H of row i, cells j0 .. j0+W-1, from the new E (dzx = E[i][j+1] - E[i][j],
// dzy = E[i+1][j] - E[i][j]); hx / hy hold the old H and are updated.
template <int W>
__device__ __forceinline__ void adj_h_row_shot(const Dev& g, const float* R, const BandY& by, int i, int j0, int lane,
                                               float (&hx)[W], float (&hy)[W], const float (&dzx)[W],
                                               const float (&dzy)[W], const float* ch, const PsiG& rd,
                                               const PsiG& wr) {
    const XRow xh = x_row(g, i, false);
    const uint32_t in = by.h.in;
    float ci[W], py[W], px[W];
    ld_coef_mask<W>(g, g.ci, i, j0, by.h.m | (xh.on ? in : 0u), ci);
    ld_yrun<W>(g, rd.hy, i, by.h, lane, py);
    ld_xrun<W>(g, rd.hx, xh.r, j0, xh.on ? in : 0u, lane, px);
    hx_shot<W>(g, R, i, by.h, hx, dzx, ch, ci, py);
    hy_shot<W>(g, R, j0, xh, in, hy, dzy, ch, ci, px);
    st_yrun<W>(g, wr.hy, i, by.h, ~0u, lane, py);
    if (xh.on) st_xrun<W>(g, wr.hx, xh.r, j0, in, lane, px);
}

}  // namespace fg
