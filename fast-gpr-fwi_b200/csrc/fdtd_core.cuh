// Interior step kernels (shot lanes): the lane march restricted to interior
// tiles, launched beside the general lane march, which takes the other tiles.
//
// A tile is interior when no cell it updates or recomputes as halo lies in a
// CPML slab or on the grid's first / last rows and columns, and no source,
// receiver or adjoint injection falls in it (the plan puts these tiles last
// in the fetch order, from position core0 on).  Such a tile needs none of
// the CPML, frame and event code of the general kernels, so its kernel holds
// only the interior arithmetic (fwd_core; adj_e_core, adj_h_core and the
// imaging) and the row pointers, which it advances row by row instead of
// recomputing every address: few registers, hence many warps per SM and
// many row loads in flight, and a few instructions per cell.  The updates
// are those of the general kernels' interior branches, so every cell gets the
// same bits.
//
// Scheduling: persistent warps take tile positions core0, core0+1, ... from
// their own launch counter (tile_ctr[2 + parity]); each warp marches the rows
// of its tile as in fdtd_lanes.cuh (previous row carried in registers, halo
// recomputed, ping-pong state).
//
// Overlap with the general kernel: both kernels of a step read the state of
// the previous step and write disjoint cells of the next one, so neither
// needs the other's results.  The general kernel of the step is launched
// first and lets its dependents start at once (griddepcontrol
// launch_dependents); the interior kernel is launched behind it with
// programmatic stream serialisation, runs beside it on the SMs it leaves
// free, and waits for it (griddepcontrol wait) only before it completes, so
// the next step's general kernel, launched behind the interior kernel the same
// way, waits for it (and so for both) before it touches the state.
#pragma once

#include "fdtd_common.cuh"
#include "fdtd_lanes.cuh"

namespace fg {

// Resident 128-thread blocks per SM the register budget is sized for.
template <int W>
constexpr int core_min_blocks() { return W <= 2 ? 8 : (W <= 4 ? 6 : 4); }

// Geometry of the interior tile at fetch position pos.
struct CoreTile {
    int i0, i1, j0, grp;
};
template <int W>
__device__ __forceinline__ CoreTile core_tile(const Dev& g, int pos) {
    const int id = __ldg(g.order + pos);
    const int band = id % g.nb, rest = id / g.nb, chunk = rest % g.nc;
    CoreTile T;
    T.grp = rest / g.nc;
    T.i0 = __ldg(g.chunk_row + chunk);
    T.i1 = __ldg(g.chunk_row + chunk + 1);
    T.j0 = band * W;
    return T;
}

// ---------------------------------------------------------------------------
// Forward step t on the interior tiles
// ---------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(128, core_min_blocks<W>()) k_fwd_core(const Dev g, const int t) {
    // the next step's general kernel may launch now (it waits for this one)
    griddep_launch_dependents();
    if (blockIdx.x == 0 && threadIdx.x == 0) g.tile_ctr[2 + ((t + 1) & 1)] = 0;   // the next launch's counter
    int* ctr = g.tile_ctr + 2 + (t & 1);
    const int lane = threadIdx.x & 31;
    const int rp = t & 1, wp = rp ^ 1;
    const long long rowS = (long long)g.P * 32, hrow = (long long)g.Ph * 32;
    for (;;) {
        const int pos = fetch_tile(ctr, lane) + g.core0;
        if (pos >= g.ntiles) break;
        const CoreTile T = core_tile<W>(g, pos);
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
        float ezc[W + 2], hyu[W];
#pragma unroll
        for (int k = 0; k < W + 2; ++k) ezc[k] = ldro(g, ez + (k - 1) * 32);
        {
            float ea[W], ha[W], cu[W];
            ld_cells<W, 32>(g, ea, ez - rowS);
            ld_cells<W, 32>(g, ha, hy - rowS);
            ld_coef<W, CALIGN<W>>(g, cu, ch - g.P);
#pragma unroll
            for (int w = 0; w < W; ++w) hyu[w] = __fadd_rn(ha[w], __fmul_rn(cu[w], __fsub_rn(ezc[w + 1], ea[w])));
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
            fwd_core<W>(B, ezc, hyu, hxn, hyn, ezn);
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
// Reference-mode adjoint iteration it on the interior tiles
// ---------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(128, core_min_blocks<W>()) k_adj_core(const Dev g, const int it, const int rp) {
    griddep_launch_dependents();
    if (blockIdx.x == 0 && threadIdx.x == 0) g.tile_ctr[2 + (rp ^ 1)] = 0;   // the next launch's counter
    int* ctr = g.tile_ctr + 2 + rp;
    const int lane = threadIdx.x & 31;
    const int wp = rp ^ 1;
    const long long rowS = (long long)g.P * 32, hrow = (long long)g.Ph * 32;
    const long long n = (long long)g.nx * g.ny;
    for (;;) {
        const int pos = fetch_tile(ctr, lane) + g.core0;
        if (pos >= g.ntiles) break;
        const CoreTile T = core_tile<W>(g, pos);
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
            ld_cells<W, 32>(g, hyu, hy - rowS);
            hyu[W] = ldro(g, hy - rowS + W * 32);
            AdjEIn<W> A;
            e_in(A);
#pragma unroll
            for (int w = 0; w < W; ++w) eoc[w] = A.ez[w];
            adj_e_core<W>(A, hyu, ezc);
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
            AdjEIn<W> A;   // row r = i+1
            e_in(A);
            float chr[W], f1[W];
            ld_coef<W, CALIGN<W>>(g, chr, ch);
            ld_cells<W, 32>(g, f1, hs);
            float eor[W], ezr[W + 1], hxn[W], hyn[W];
#pragma unroll
            for (int w = 0; w < W; ++w) eor[w] = A.ez[w];
            adj_e_core<W>(A, hyc, ezr);
            adj_h_core<W>(chr, ezc, ezr, hxc, hyc, hxn, hyn);
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
