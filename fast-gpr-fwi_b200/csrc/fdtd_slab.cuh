// Slab step kernels (shot lanes): the lane march restricted to the tiles of
// the CPML slabs that hold no source, receiver or injection and do not lie in
// two slabs at once, launched between the general lane march and the
// interior kernel.
//
// Two kinds of tile (the plan orders them from slab0 on):
//   x tiles [slab0, yslab0): the interior's columns (no cell of the tile or
//     of its halo in a y slab), rows touching an x slab, the first and last
//     rows included.  A row inside an x slab updates Hx as in the interior
//     and Hy and E with the row's x-slab terms (row-uniform profile values);
//     the other rows are interior rows; row 0 keeps its E and Hx.
//   y tiles [yslab0, core0): the interior's rows, columns touching one y
//     slab (the band's cells in the y0 or the ymax slab, not both), the first
//     and last columns included.  Every row updates Hy as in the interior and
//     Hx and E with the y-slab terms of the cells that lie in the slab;
//     column 0 keeps its E and Hy, cells beyond the grid are kept.
// Either kind needs none of the event, ring, prefetch and per-cell
// fallback code of the general kernels, so these kernels hold the row
// updates of one slab kind each, with the loads of the interior kernels.
// Every cell is updated by the same arithmetic, in the same order, as the
// general kernels' shot-lane CPML rows (fdtd_shot.cuh: e_shot, hx_shot,
// hy_shot and their division vote), so it gets the same bits.
//
// Scheduling as for the interior kernels (fdtd_core.cuh): persistent warps
// take fetch positions from their own counter (tile_ctr[4 + parity]); the
// kernel is launched behind the general kernel of the step with
// programmatic stream serialisation, lets the interior kernel behind it start
// at once, and waits for the general kernel only before it completes.
#pragma once

#include "fdtd_common.cuh"
#include "fdtd_lanes.cuh"
#include "fdtd_core.cuh"

namespace fg {

// ---------------------------------------------------------------------------
// E rows of the slab kernels (N cells from j0; dhy / dhx the H differences)
// ---------------------------------------------------------------------------
// x-slab terms only (the E branch of e_shot_k with no y-slab cell)
template <int N, bool FAST>
__device__ __forceinline__ void e_xrow_k(const Dev& g, const float* R, bool upd, const XRow& xe, float (&ez)[N],
                                         const float (&dhy)[N], const float (&dhx)[N], const float* ca, const float* cb,
                                         const float (&cd)[N], float (&px)[N]) {
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
        float e = ez[n];
        if (upd) e = __fmaf_rn(-cb[n], dhx[n], madd2(ca[n], e, cb[n], dhy[n]));
        if (xe.on) {
            const float dd = div_row<FAST>(g, dhy[n]);
            e = __fmaf_rn(cd[n], madd2(xa, dd, xb, px[n]), e);
            px[n] = msub2(xc, px[n], xf, dd);
        }
        ez[n] = e;
    }
}
// upd: the row takes the interior update (i >= 1; row 0 keeps its E)
template <int N>
__device__ __forceinline__ void e_xrow(const Dev& g, const float* R, bool upd, const XRow& xe, float (&ez)[N],
                                       const float (&dhy)[N], const float (&dhx)[N], const float* ca, const float* cb,
                                       const float (&cd)[N], float (&px)[N]) {
    if (div_row_fast<N>(g, xe.on ? low_bits(N) : 0u, dhy))
        e_xrow_k<N, true>(g, R, upd, xe, ez, dhy, dhx, ca, cb, cd, px);
    else
        e_xrow_k<N, false>(g, R, upd, xe, ez, dhy, dhx, ca, cb, cd, px);
}

// y-slab terms only, for the cells of the run ye (the E branch of e_shot_k
// outside the x slabs)
template <int N, bool FAST>
__device__ __forceinline__ void e_yrow_k(const Dev& g, const float* R, int j0, const YRun& ye, float (&ez)[N],
                                         const float (&dhy)[N], const float (&dhx)[N], const float* ca, const float* cb,
                                         const float (&cd)[N], float (&py)[N]) {
#pragma unroll
    for (int n = 0; n < N; ++n) {
        if (!bit(ye.in, n)) continue;
        float e = ez[n];
        if (j0 + n >= 1) e = __fmaf_rn(-cb[n], dhx[n], madd2(ca[n], e, cb[n], dhy[n]));
        if (bit(ye.m, n)) e = cpml<false>(g, e, div_row<FAST>(g, dhx[n]), cd[n], py[n], R, ye.k0 + ye.dk * n);
        ez[n] = e;
    }
}
// cells j0 .. j0+N-1 of a row at i >= 1 (cells outside the grid are kept;
// column 0 takes no interior update)
template <int N>
__device__ __forceinline__ void e_yrow(const Dev& g, const float* R, int j0, const YRun& ye, float (&ez)[N],
                                       const float (&dhy)[N], const float (&dhx)[N], const float* ca, const float* cb,
                                       const float (&cd)[N], float (&py)[N]) {
    if (div_row_fast<N>(g, ye.m & ye.in, dhx)) e_yrow_k<N, true>(g, R, j0, ye, ez, dhy, dhx, ca, cb, cd, py);
    else e_yrow_k<N, false>(g, R, j0, ye, ez, dhy, dhx, ca, cb, cd, py);
}

// ---------------------------------------------------------------------------
// Forward rows
// ---------------------------------------------------------------------------
// Row i of an x tile inside an x slab: Hx at j0-1 .. j0+W-1 as in the
// interior, Hy and E at j0 .. j0+W-1 with the row's x-slab terms.
template <int W>
__device__ __forceinline__ void fwd_xrow(const Dev& g, const float* R, int i, int j0, int lane, const FwdIn<W>& B,
                                         const float (&ezc)[W + 2], const float (&hyu)[W], const PsiG& rd,
                                         const PsiG& wr, float (&hxn)[W + 1], float (&hyn)[W], float (&ezn)[W]) {
    const XRow xh = x_row(g, i, false), xe = x_row(g, i, true);
    const uint32_t all = low_bits(W);
    float ci[W], cd[W], pxh[W], pxe[W];
    ld_coef_mask<W>(g, g.ci, i, j0, xh.on ? all : 0u, ci);
    ld_coef_mask<W>(g, g.cd, i, j0, xe.on ? all : 0u, cd);
    ld_xrun<W>(g, rd.hx, xh.r, j0, xh.on ? all : 0u, lane, pxh);
    ld_xrun<W>(g, rd.ex, xe.r, j0, xe.on ? all : 0u, lane, pxe);
#pragma unroll
    for (int k = 0; k <= W; ++k)
        hxn[k] = i >= 1 ? msub2(1.0f, B.hxo[k], B.ch[k], __fsub_rn(ezc[k + 1], ezc[k])) : B.hxo[k];
    float dzy[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
        hyn[w] = B.hyo[w];
        dzy[w] = __fsub_rn(B.en[w + 1], ezc[w + 1]);
    }
    hy_shot<W>(g, R, j0, xh, all, hyn, dzy, B.ch + 1, ci, pxh);
    float dhy[W], dhx[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
        ezn[w] = ezc[w + 1];
        dhy[w] = __fsub_rn(hyn[w], hyu[w]);
        dhx[w] = __fsub_rn(hxn[w + 1], hxn[w]);
    }
    e_xrow<W>(g, R, i >= 1, xe, ezn, dhy, dhx, B.ca, B.cb, cd, pxe);
    if (xh.on) st_xrun<W>(g, wr.hx, xh.r, j0, all, lane, pxh);
    if (xe.on) st_xrun<W>(g, wr.ex, xe.r, j0, all, lane, pxe);
}

// Row i of a y tile: Hx at j0-1 .. j0+W-1 and E at j0 .. j0+W-1 with the
// y-slab terms of their cells in the slab (the halo Hx's auxiliary is read,
// not stored), Hy as in the interior.
template <int W>
__device__ __forceinline__ void fwd_yrow(const Dev& g, const float* R, const BandY& by, int i, int j0, int lane,
                                         const FwdIn<W>& B, const float (&ezc)[W + 2], const float (&hyu)[W],
                                         const PsiG& rd, const PsiG& wr, float (&hxn)[W + 1], float (&hyn)[W],
                                         float (&ezn)[W]) {
    float ci[W + 1], cd[W], pyh[W + 1], pye[W];
    ld_coef_mask<W + 1>(g, g.ci, i, j0 - 1, by.h.m, ci);
    ld_coef_mask<W>(g, g.cd, i, j0, by.e.m, cd);
    ld_yrun<W + 1>(g, rd.hy, i, by.h, lane, pyh);
    ld_yrun<W>(g, rd.ey, i, by.e, lane, pye);
    float dzx[W + 1];
#pragma unroll
    for (int k = 0; k <= W; ++k) {
        hxn[k] = B.hxo[k];
        dzx[k] = __fsub_rn(ezc[k + 1], ezc[k]);
    }
    hx_shot<W + 1>(g, R, i, by.h, hxn, dzx, B.ch, ci, pyh);
#pragma unroll
    for (int w = 0; w < W; ++w)
        hyn[w] = bit(by.e.in, w) && j0 + w >= 1 ? madd2(1.0f, B.hyo[w], B.ch[w + 1], __fsub_rn(B.en[w + 1], ezc[w + 1]))
                                                : B.hyo[w];
    float dhy[W], dhx[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
        ezn[w] = ezc[w + 1];
        dhy[w] = __fsub_rn(hyn[w], hyu[w]);
        dhx[w] = __fsub_rn(hxn[w + 1], hxn[w]);
    }
    e_yrow<W>(g, R, j0, by.e, ezn, dhy, dhx, B.ca, B.cb, cd, pye);
    st_yrun<W + 1>(g, wr.hy, i, by.h, ~1u, lane, pyh);
    st_yrun<W>(g, wr.ey, i, by.e, ~0u, lane, pye);
}

// ---------------------------------------------------------------------------
// Forward step t on the slab tiles
// ---------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(128, 4) k_fwd_slab(const Dev g, const int t) {
    griddep_launch_dependents();   // the interior kernel behind this one may start
    extern __shared__ __align__(128) unsigned char smem[];
    const float* R = stage_profile(g, smem);
    if (blockIdx.x == 0 && threadIdx.x == 0) g.tile_ctr[4 + ((t + 1) & 1)] = 0;   // the next launch's counter
    int* ctr = g.tile_ctr + 4 + (t & 1);
    const int lane = threadIdx.x & 31;
    const int rp = t & 1, wp = rp ^ 1;
    const int nx = g.nx, th = g.th;
    const long long rowS = (long long)g.P * 32, hrow = (long long)g.Ph * 32;
    for (;;) {
        const int pos = fetch_tile(ctr, lane) + g.slab0;
        if (pos >= g.core0) break;
        const bool xt = pos < g.yslab0;
        const CoreTile T = core_tile<W>(g, pos);
        const PsiG rd = psi_group(g, rp, T.grp), wr = psi_group(g, wp, T.grp);
        const BandY by = band_fwd<W>(g, T.j0);
        const long long o = (long long)T.grp * g.plane + ((long long)T.i0 * g.P + T.j0 + PADC) * 32 + lane;
        const float* ez = g.ez[rp] + o;   // cell (i, j0) of the current row i
        const float* hx = g.hx[rp] + o;
        const float* hy = g.hy[rp] + o;
        float* ezw = g.ez[wp] + o;
        float* hxw = g.hx[wp] + o;
        float* hyw = g.hy[wp] + o;
        const long long co = (long long)T.i0 * g.P + T.j0 + PADC;
        const float* ca = g.ca + co;
        const float* cb = g.cb + co;
        const float* ch = g.ch + co;
        float* hs = g.hist ? g.hist + ((((long long)(t - g.hist_t0) * g.ngroups + T.grp) * g.nx + T.i0) * g.Ph + T.j0) *
                                          32 + lane
                           : nullptr;
        // Ez_old of row i0 (columns j0-1 .. j0+W) and the new Hy of row i0-1
        // (its auxiliaries are only read: the tile of that row stores them)
        float ezc[W + 2], hyu[W];
#pragma unroll
        for (int k = 0; k < W + 2; ++k) ezc[k] = ldro(g, ez + (k - 1) * 32);
#pragma unroll
        for (int w = 0; w < W; ++w) hyu[w] = 0.f;
        if (T.i0 >= 1) {
            float ea[W], cu[W], dz[W];
            ld_cells<W, 32>(g, ea, ez - rowS);
            ld_cells<W, 32>(g, hyu, hy - rowS);
            ld_coef<W, CALIGN<W>>(g, cu, ch - g.P);
#pragma unroll
            for (int w = 0; w < W; ++w) dz[w] = __fsub_rn(ezc[w + 1], ea[w]);
            fwd_hy_halo_shot<W>(g, R, by, T.i0 - 1, T.j0, lane, hyu, dz, cu, rd);
        }
        for (int i = T.i0; i < T.i1; ++i) {
            FwdIn<W> B;
#pragma unroll
            for (int k = 0; k < W + 2; ++k) B.en[k] = ldro(g, ez + rowS + (k - 1) * 32);
#pragma unroll
            for (int k = 0; k <= W; ++k) B.hxo[k] = ldro(g, hx + (k - 1) * 32);
            ld_cells<W, 32>(g, B.hyo, hy);
            ld_coef<W, CALIGN<W>>(g, B.ca, ca);
            ld_coef<W, CALIGN<W>>(g, B.cb, cb);
            B.ch[0] = ldro(g, ch - 1);
            ld_coef<W, CALIGN<W>>(g, B.ch + 1, ch);
            float hxn[W + 1], hyn[W], ezn[W];
            if (xt) {
                if (i >= th + 1 && i <= nx - th - 1) fwd_core<W>(B, ezc, hyu, hxn, hyn, ezn);
                else fwd_xrow<W>(g, R, i, T.j0, lane, B, ezc, hyu, rd, wr, hxn, hyn, ezn);
            } else {
                fwd_yrow<W>(g, R, by, i, T.j0, lane, B, ezc, hyu, rd, wr, hxn, hyn, ezn);
            }
            st_cells<W, 32>(g, ezw, ezn);
            st_cells<W, 32>(g, hxw, hxn + 1);
            st_cells<W, 32>(g, hyw, hyn);
            if (hs) {
                st_cells<W, 32, true>(g, hs, ezn);
                hs += hrow;
            }
#pragma unroll
            for (int k = 0; k < W + 2; ++k) ezc[k] = B.en[k];
#pragma unroll
            for (int w = 0; w < W; ++w) hyu[w] = hyn[w];
            ez += rowS;
            hx += rowS;
            hy += rowS;
            ezw += rowS;
            hxw += rowS;
            hyw += rowS;
            ca += g.P;
            cb += g.P;
            ch += g.P;
        }
    }
    griddep_wait();
}

// ---------------------------------------------------------------------------
// Adjoint rows (reference mode) of the slab tiles
// ---------------------------------------------------------------------------
// New E of row r, cells j0 .. j0+W (column j0+W is the halo), from the old
// operands A (hyu = old Hy of row r-1): interior, x-row or y-row update; the
// auxiliaries of the first W cells are stored when `own`.
template <int W>
__device__ __forceinline__ void adj_e_slab(const Dev& g, const float* R, const BandY& by, bool xt, int r, int j0,
                                           int lane, bool own, const AdjEIn<W>& A, const float (&hyu)[W + 1],
                                           const PsiG& rd, const PsiG& wr, float (&out)[W + 1]) {
    if (xt && r >= g.th + 1 && r <= g.nx - g.th - 1) {
        adj_e_core<W>(A, hyu, out);
        return;
    }
    float dhy[W + 1], dhx[W + 1], cd[W + 1], ps[W + 1];
#pragma unroll
    for (int k = 0; k <= W; ++k) {
        out[k] = A.ez[k];
        dhy[k] = __fsub_rn(A.hyo[k], hyu[k]);
        dhx[k] = __fsub_rn(A.hxo[k + 1], A.hxo[k]);
    }
    const uint32_t mine = low_bits(W);
    if (xt) {
        const XRow xe = x_row(g, r, true);
        const uint32_t all = low_bits(W + 1);
        ld_coef_mask<W + 1>(g, g.cd, r, j0, xe.on ? all : 0u, cd);
        ld_xrun<W + 1>(g, rd.ex, xe.r, j0, xe.on ? all : 0u, lane, ps);
        e_xrow<W + 1>(g, R, r >= 1, xe, out, dhy, dhx, A.ca, A.cb, cd, ps);
        if (own && xe.on) st_xrun<W + 1>(g, wr.ex, xe.r, j0, mine, lane, ps);
    } else {
        ld_coef_mask<W + 1>(g, g.cd, r, j0, by.e.m, cd);
        ld_yrun<W + 1>(g, rd.ey, r, by.e, lane, ps);
        e_yrow<W + 1>(g, R, j0, by.e, out, dhy, dhx, A.ca, A.cb, cd, ps);
        if (own) st_yrun<W + 1>(g, wr.ey, r, by.e, mine, lane, ps);
    }
}

// H of row i, cells j0 .. j0+W-1, from the new E of rows i (ezc) and i+1
// (ezr) and the old H (hxc from column j0-1, hyc from j0).
template <int W>
__device__ __forceinline__ void adj_h_slab(const Dev& g, const float* R, const BandY& by, bool xt, int i, int j0,
                                           int lane, const float (&ch)[W], const float (&ezc)[W + 1],
                                           const float (&ezr)[W + 1], const float (&hxc)[W + 2],
                                           const float (&hyc)[W + 1], const PsiG& rd, const PsiG& wr, float (&hx)[W],
                                           float (&hy)[W]) {
    if (xt && i >= g.th + 1 && i <= g.nx - g.th - 1) {
        adj_h_core<W>(ch, ezc, ezr, hxc, hyc, hx, hy);
        return;
    }
    float dzx[W], dzy[W], ci[W], ps[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
        hx[w] = hxc[w + 1];
        hy[w] = hyc[w];
        dzx[w] = __fsub_rn(ezc[w + 1], ezc[w]);
        dzy[w] = __fsub_rn(ezr[w], ezc[w]);
    }
    const uint32_t all = low_bits(W);
    if (xt) {
        const XRow xh = x_row(g, i, false);
        ld_coef_mask<W>(g, g.ci, i, j0, xh.on ? all : 0u, ci);
        ld_xrun<W>(g, rd.hx, xh.r, j0, xh.on ? all : 0u, lane, ps);
        if (i >= 1) {
#pragma unroll
            for (int w = 0; w < W; ++w) hx[w] = msub2(1.0f, hx[w], ch[w], dzx[w]);
        }
        hy_shot<W>(g, R, j0, xh, all, hy, dzy, ch, ci, ps);
        if (xh.on) st_xrun<W>(g, wr.hx, xh.r, j0, all, lane, ps);
    } else {
        ld_coef_mask<W>(g, g.ci, i, j0, by.h.m, ci);
        ld_yrun<W>(g, rd.hy, i, by.h, lane, ps);
        hx_shot<W>(g, R, i, by.h, hx, dzx, ch, ci, ps);
#pragma unroll
        for (int w = 0; w < W; ++w)
            if (bit(by.h.in, w) && j0 + w >= 1) hy[w] = madd2(1.0f, hy[w], ch[w], dzy[w]);
        st_yrun<W>(g, wr.hy, i, by.h, ~0u, lane, ps);
    }
}

// ---------------------------------------------------------------------------
// Reference-mode adjoint iteration it on the slab tiles
// ---------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(128, 2) k_adj_slab(const Dev g, const int it, const int rp) {
    griddep_launch_dependents();
    extern __shared__ __align__(128) unsigned char smem[];
    const float* R = stage_profile(g, smem);
    if (blockIdx.x == 0 && threadIdx.x == 0) g.tile_ctr[4 + (rp ^ 1)] = 0;   // the next launch's counter
    int* ctr = g.tile_ctr + 4 + rp;
    const int lane = threadIdx.x & 31;
    const int wp = rp ^ 1;
    const long long rowS = (long long)g.P * 32, hrow = (long long)g.Ph * 32;
    const long long n = (long long)g.nx * g.ny;
    for (;;) {
        const int pos = fetch_tile(ctr, lane) + g.slab0;
        if (pos >= g.core0) break;
        const bool xt = pos < g.yslab0;
        const CoreTile T = core_tile<W>(g, pos);
        const PsiG rd = psi_group(g, rp, T.grp), wr = psi_group(g, wp, T.grp);
        const BandY by = band_adj<W>(g, T.j0);
        const long long o = (long long)T.grp * g.plane + ((long long)T.i0 * g.P + T.j0 + PADC) * 32 + lane;
        const float* ez = g.ez[rp] + o;   // cell (r, j0) of the E row r
        const float* hx = g.hx[rp] + o;
        const float* hy = g.hy[rp] + o;
        float* ezw = g.ez[wp] + o;        // cell (i, j0) of the H row i
        float* hxw = g.hx[wp] + o;
        float* hyw = g.hy[wp] + o;
        const long long co = (long long)T.i0 * g.P + T.j0 + PADC;
        const float* ca = g.ca + co;      // row r
        const float* cb = g.cb + co;
        const float* ch = g.ch + co;      // row i
        const float* hs = g.hist + ((((long long)(it - g.hist_t0) * g.ngroups + T.grp) * g.nx + T.i0) * g.Ph + T.j0) *
                                       32 + lane;
        double* ge = g.gacc + (long long)T.grp * 2 * n + (long long)T.i0 * g.ny + T.j0;
        auto e_in = [&](AdjEIn<W>& A) {
            ld_cells<W, 32>(g, A.ez, ez);
            A.ez[W] = ldro(g, ez + W * 32);
#pragma unroll
            for (int k = 0; k < W + 2; ++k) A.hxo[k] = ldro(g, hx + (k - 1) * 32);
            ld_cells<W, 32>(g, A.hyo, hy);
            A.hyo[W] = ldro(g, hy + W * 32);
            ld_coef<W + 1, CALIGN<W>>(g, A.ca, ca);
            ld_coef<W + 1, CALIGN<W>>(g, A.cb, cb);
        };
        // new E of row i0 with the old H of rows i0-1 and i0; eoc keeps its old Ez
        float ezc[W + 1], hxc[W + 2], hyc[W + 1], eoc[W];
        {
            float hyu[W + 1];
#pragma unroll
            for (int k = 0; k <= W; ++k) hyu[k] = 0.f;
            if (T.i0 >= 1) {
                ld_cells<W, 32>(g, hyu, hy - rowS);
                hyu[W] = ldro(g, hy - rowS + W * 32);
            }
            AdjEIn<W> A;
            e_in(A);
#pragma unroll
            for (int w = 0; w < W; ++w) eoc[w] = A.ez[w];
            adj_e_slab<W>(g, R, by, xt, T.i0, T.j0, lane, true, A, hyu, rd, wr, ezc);
#pragma unroll
            for (int k = 0; k < W + 2; ++k) hxc[k] = A.hxo[k];
#pragma unroll
            for (int k = 0; k <= W; ++k) hyc[k] = A.hyo[k];
        }
        for (int i = T.i0; i < T.i1; ++i) {
            ez += rowS;
            hx += rowS;
            hy += rowS;
            ca += g.P;
            cb += g.P;
            AdjEIn<W> A;   // row r = i+1; the frame row nx is zero
            float chr[W], f1[W];
            ld_coef<W, CALIGN<W>>(g, chr, ch);
            ld_cells<W, 32>(g, f1, hs);
            float eor[W], ezr[W + 1], hxn[W], hyn[W];
            if (i + 1 < g.nx) {
                e_in(A);
#pragma unroll
                for (int w = 0; w < W; ++w) eor[w] = A.ez[w];
                adj_e_slab<W>(g, R, by, xt, i + 1, T.j0, lane, i + 1 < T.i1, A, hyc, rd, wr, ezr);
            } else {
#pragma unroll
                for (int w = 0; w < W; ++w) eor[w] = 0.f;
#pragma unroll
                for (int k = 0; k <= W; ++k) ezr[k] = A.hyo[k] = 0.f;
#pragma unroll
                for (int k = 0; k < W + 2; ++k) A.hxo[k] = 0.f;
            }
            adj_h_slab<W>(g, R, by, xt, i, T.j0, lane, chr, ezc, ezr, hxc, hyc, rd, wr, hxn, hyn);
            adj_image<W, true>(g, f1, ezc, eoc, ge, ge + n, T.j0, lane);
            st_cells<W, 32>(g, ezw, ezc);
            st_cells<W, 32>(g, hxw, hxn);
            st_cells<W, 32>(g, hyw, hyn);
#pragma unroll
            for (int k = 0; k <= W; ++k) {
                ezc[k] = ezr[k];
                hyc[k] = A.hyo[k];
            }
#pragma unroll
            for (int w = 0; w < W; ++w) eoc[w] = eor[w];
#pragma unroll
            for (int k = 0; k < W + 2; ++k) hxc[k] = A.hxo[k];
            ezw += rowS;
            hxw += rowS;
            hyw += rowS;
            ch += g.P;
            hs += hrow;
            ge += g.ny;
        }
    }
    griddep_wait();
}

}  // namespace fg
