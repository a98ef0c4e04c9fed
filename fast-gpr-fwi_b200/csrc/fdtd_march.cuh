// Prefetching warp-march kernels (kernel 3).
//
// A warp owns a tile (shot group of G shots, row chunk [i0, i1), column band
// [b0, b0+32V)); lane l holds columns b0+lV .. b0+lV+V-1.  For each shot of
// the group the warp marches down the rows of its chunk.  The operands of the
// next row (old Ez/Hx/Hy, coefficient rows, halo cells, and in the adjoint the
// stored forward Ez) are loaded into registers one iteration ahead, so their
// latency overlaps the current row's arithmetic; there is no block-level
// synchronisation at all (warps of a CTA are independent tiles).
//
// Warps whose cells are all interior (no CPML slab, not on the i==0 / j==0
// edges, all columns < ny) use the lean update; others the general per-cell
// device code.  Both perform the same floating-point operation sequence
// (fdtd_device.cuh), so the kernels are bit-identical to the rest.
//
// Adjoint imaging: each warp accumulates the shots of its group per cell in
// shared memory (fp32, in shot order) and adds the group sum to the fp64
// accumulator once per step.
#pragma once

#include "fdtd_device.cuh"

namespace fg {

constexpr int MARCH_WARPS = 4;   // warps (independent tiles) per CTA

struct TileM {
    int band, chunk, grp, i0, i1, b0, be;
};

__device__ __forceinline__ bool march_tile(const GridDev& g, int V, int tile, TileM& t) {
    if (tile >= g.ntiles) return false;
    t.band = tile % g.nb;
    const int rest = tile / g.nb;
    t.chunk = rest % g.nc;
    t.grp = rest / g.nc;
    t.i0 = g.chunk_row[t.chunk];
    t.i1 = g.chunk_row[t.chunk + 1];
    t.b0 = t.band * 32 * V;
    t.be = t.b0 + 32 * V;
    return true;
}

// Rows whose H and E updates involve no x-slab CPML and no i == 0 edge.
__device__ __forceinline__ bool core_row(const GridDev& g, int i) {
    return i >= g.th + 1 && i <= g.nx - g.th - 1;
}
// Bands whose columns involve no y-slab CPML, no j == 0 edge and no j >= ny.
__device__ __forceinline__ bool core_band(const GridDev& g, int b0, int be) {
    return b0 >= g.th + 1 && be <= g.ny - g.th;
}

template <int V>
__device__ __forceinline__ void ldv(const GridDev& g, float (&x)[V], const float* p, bool ok) {
    if (ok) {
        ld_state<V>(g, x, p);
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v) x[v] = 0.f;
    }
}
template <int V>
__device__ __forceinline__ void ldcv(const GridDev& g, float (&x)[V], const float* p, bool ok) {
    if (ok) {
        ld_coef<V>(g, x, p);
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v) x[v] = 0.f;
    }
}

// Advance an event cursor (events sorted by row, then shot slot) to the first
// event of (row, slot) or past it; returns true while such an event is current.
__device__ __forceinline__ bool ev_seek(const Ev* ev, int& cur, int end, int row, int slot) {
    while (cur < end) {
        const Ev e = __ldg(ev + cur);
        if (e.x > row || (e.x == row && e.y > slot)) return false;
        if (e.x == row && e.y == slot) return true;
        ++cur;
    }
    return false;
}

// ---------------------------------------------------------------------------
// Forward step
// ---------------------------------------------------------------------------
template <int V>
struct FwdRow {            // operands of row r: Ez_old[r+1], Hx_old[r], Hy_old[r], coefficients of r
    float en[V], hx[V], hy[V], ca[V], cb[V], ch[V];
    float ezR;             // lane 31: Ez_old[r][be]
    float ezL, hxL, chL;   // lane 0:  Ez_old[r][b0-1], Hx_old[r][b0-1], uH1[r][b0-1]
};

template <int V>
__device__ __forceinline__ void fwd_row_load(const GridDev& g, FwdRow<V>& B, const float* ez, const float* hx,
                                             const float* hy, int r, int jb, int lane, int b0, int be, bool act) {
    const int o = r * g.P + jb;
    ldv<V>(g, B.en, ez + o + g.P, act);
    ldv<V>(g, B.hx, hx + o, act);
    ldv<V>(g, B.hy, hy + o, act);
    ldcv<V>(g, B.ca, g.ca + o, act);
    ldcv<V>(g, B.cb, g.cb + o, act);
    ldcv<V>(g, B.ch, g.ch + o, act);
    B.ezR = 0.f;
    B.ezL = 0.f;
    B.hxL = 0.f;
    B.chL = 0.f;
    if (lane == 31 && be < g.P) B.ezR = ld1(g, ez + r * g.P + be);
    if (lane == 0 && b0 > 0) {
        const int ol = r * g.P + b0 - 1;
        B.ezL = ld1(g, ez + ol);
        B.hxL = ld1(g, hx + ol);
        B.chL = ldc1(g, g.ch + ol);
    }
}

// Per-warp state of a forward march over one shot.
template <int V>
struct FwdMarch {
    float ezc[V];   // Ez_old of the current row
    float hyu[V];   // Hy_new of the row above
};

template <int V>
__device__ __forceinline__ void fwd_row(const GridDev& g, FwdMarch<V>& M, const FwdRow<V>& B, int i, int t, int q,
                                        int s, long long so, int jb, int lane, int b0, bool bcore, bool act,
                                        const PsiShot& rd, const PsiShot& wr, int& sc, int se, int& rc, int re) {
    const int P = g.P, ny = g.ny;
    const int wp = (t & 1) ^ 1;
    const bool core = bcore && core_row(g, i);
    // ---- H of row i
    float right = __shfl_down_sync(FULL, M.ezc[0], 1);
    if (lane == 31) right = B.ezR;
    float hx[V], hy[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        hx[v] = B.hx[v];
        hy[v] = B.hy[v];
    }
    float hxl;
    if (core) {
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const float er = (v + 1 < V) ? M.ezc[(v + 1) % V] : right;
            hx[v] = __fsub_rn(hx[v], __fmul_rn(B.ch[v], __fsub_rn(er, M.ezc[v])));
            hy[v] = __fadd_rn(hy[v], __fmul_rn(B.ch[v], __fsub_rn(B.en[v], M.ezc[v])));
        }
        hxl = __shfl_up_sync(FULL, hx[V - 1], 1);
        // column b0-1 is interior too (b0 >= th+1): the lean Hx update
        if (lane == 0) hxl = __fsub_rn(B.hxL, __fmul_rn(B.chL, __fsub_rn(M.ezc[0], B.ezL)));
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const float er = (v + 1 < V) ? M.ezc[(v + 1) % V] : right;
            if (jb + v < ny)
                h_update<true, true, true>(g, i, jb + v, hx[v], hy[v], __fsub_rn(er, M.ezc[v]),
                                           __fsub_rn(B.en[v], M.ezc[v]), B.ch[v], rd, wr);
        }
        hxl = __shfl_up_sync(FULL, hx[V - 1], 1);
        if (lane == 0) {
            hxl = 0.f;
            if (b0 > 0) {
                float h = B.hxL, hy_unused = 0.f;
                h_update<false, true, false>(g, i, b0 - 1, h, hy_unused, __fsub_rn(M.ezc[0], B.ezL), 0.f, B.chL, rd,
                                             rd);
                hxl = h;
            }
        }
    }
    // ---- E of row i
    float ezw[V];
    if (core) {
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const float l = (v > 0) ? hx[(v + V - 1) % V] : hxl;
            ezw[v] = __fmaf_rn(-B.cb[v], __fsub_rn(hx[v], l),
                               madd2(B.ca[v], M.ezc[v], B.cb[v], __fsub_rn(hy[v], M.hyu[v])));
        }
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const float l = (v > 0) ? hx[(v + V - 1) % V] : hxl;
            ezw[v] = M.ezc[v];
            if (jb + v < ny)
                ezw[v] = e_update<true>(g, i, jb + v, M.ezc[v], __fsub_rn(hy[v], M.hyu[v]), __fsub_rn(hx[v], l),
                                        B.ca[v], B.cb[v], rd, wr);
        }
    }
    // Hertzian dipole (sourcereceiver.cu:84)
    while (ev_seek(g.src_ev, sc, se, i, q)) {
        const Ev e = __ldg(g.src_ev + sc);
#pragma unroll
        for (int v = 0; v < V; ++v)
            if (jb + v == e.z) {
                const float cd = ldc1(g, g.cd + (long long)i * P + e.z);
                ezw[v] = __fmaf_rn(-cd, __ldg(g.srcw + (long long)e.w * g.nt + t), ezw[v]);
            }
        ++sc;
    }
    if (act) {
        const long long o = so + (long long)i * P + jb;
        st_state<V>(g, g.ez[wp] + o, ezw);
        st_state<V>(g, g.hx[wp] + o, hx);
        st_state<V>(g, g.hy[wp] + o, hy);
    }
    if (g.hist && jb < g.Ph)
        st_state<V>(g, g.hist + ((long long)t * g.S + s) * ((long long)g.nx * g.Ph) + (long long)i * g.Ph + jb, ezw);
    while (ev_seek(g.rx_ev, rc, re, i, q)) {
        const Ev e = __ldg(g.rx_ev + rc);
        if (t + 1 < g.nt) {
#pragma unroll
            for (int v = 0; v < V; ++v)
                if (jb + v == e.z) g.traces[((long long)s * g.nt + t + 1) * g.nrx + e.w] = ezw[v];
        }
        ++rc;
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
        M.ezc[v] = B.en[v];
        M.hyu[v] = hy[v];
    }
}

template <int V>
__global__ void __launch_bounds__(32 * MARCH_WARPS) k_forward_march(const GridDev g, const int t, const int G) {
    const int lane = threadIdx.x & 31;
    TileM T;
    const int tile = blockIdx.x * MARCH_WARPS + (threadIdx.x >> 5);
    if (!march_tile(g, V, tile, T)) return;
    const int P = g.P, ny = g.ny;
    const int rp = t & 1, wp = rp ^ 1;
    const int jb = T.b0 + lane * V;
    const bool act = jb < P;
    const bool bcore = core_band(g, T.b0, T.be);
    const int sc0 = g.src_off[tile], se = g.src_off[tile + 1];
    const int rc0 = g.rx_off[tile], re = g.rx_off[tile + 1];

    for (int q = 0; q < G; ++q) {
        const int s = T.grp * G + q;
        if (s >= g.S) break;
        const long long so = (long long)s * g.plane;
        const float* ezR = g.ez[rp] + so;
        const float* hxR = g.hx[rp] + so;
        const float* hyR = g.hy[rp] + so;
        const PsiShot rd = psi_shot(g, rp, s), wr = psi_shot(g, wp, s);
        FwdMarch<V> M;
        ldv<V>(g, M.ezc, ezR + T.i0 * P + jb, act);
#pragma unroll
        for (int v = 0; v < V; ++v) M.hyu[v] = 0.f;
        if (T.i0 >= 1) {
            // new Hy of the row above the chunk, from the old state (auxiliaries read only)
            const int ih = T.i0 - 1;
            float ea[V], ha[V], ca[V];
            ldv<V>(g, ea, ezR + ih * P + jb, act);
            ldv<V>(g, ha, hyR + ih * P + jb, act);
            ldcv<V>(g, ca, g.ch + ih * P + jb, act);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                float hx_unused = 0.f, h = ha[v];
                if (jb + v < ny)
                    h_update<false, false, true>(g, ih, jb + v, hx_unused, h, 0.f, __fsub_rn(M.ezc[v], ea[v]), ca[v],
                                                 rd, rd);
                M.hyu[v] = h;
            }
        }
        int sc = sc0, rc = rc0;
        // double-buffered row operands: X holds row i, Y is being loaded with row i+1
        FwdRow<V> X, Y;
        fwd_row_load<V>(g, X, ezR, hxR, hyR, T.i0, jb, lane, T.b0, T.be, act);
        for (int i = T.i0; i < T.i1; i += 2) {
            if (i + 1 < T.i1) fwd_row_load<V>(g, Y, ezR, hxR, hyR, i + 1, jb, lane, T.b0, T.be, act);
            fwd_row<V>(g, M, X, i, t, q, s, so, jb, lane, T.b0, bcore, act, rd, wr, sc, se, rc, re);
            if (i + 1 >= T.i1) break;
            if (i + 2 < T.i1) fwd_row_load<V>(g, X, ezR, hxR, hyR, i + 2, jb, lane, T.b0, T.be, act);
            fwd_row<V>(g, M, Y, i + 1, t, q, s, so, jb, lane, T.b0, bcore, act, rd, wr, sc, se, rc, re);
        }
    }
}

// ---------------------------------------------------------------------------
// Reference-mode adjoint step
// ---------------------------------------------------------------------------
template <int V>
struct AdjRow {            // operands of row r
    float ez[V], hx[V], hy[V], ca[V], cb[V], ch[V], f1[V], f0[V];
    float hxL;                         // lane 0:  Hx_old[r][b0-1]
    float ezR, hxR, hyR, caR, cbR;     // lane 31: column be of row r
};

template <int V>
__device__ __forceinline__ void adj_row_load(const GridDev& g, AdjRow<V>& B, const float* ez, const float* hx,
                                             const float* hy, const float* f1, const float* f0, int r, int jb, int lane,
                                             int b0, int be, bool act, bool hist) {
    const long long o = (long long)r * g.P + jb;
    ldv<V>(g, B.ez, ez + o, act);
    ldv<V>(g, B.hx, hx + o, act);
    ldv<V>(g, B.hy, hy + o, act);
    ldcv<V>(g, B.ca, g.ca + o, act);
    ldcv<V>(g, B.cb, g.cb + o, act);
    ldcv<V>(g, B.ch, g.ch + o, act);
    const bool hok = hist && jb < g.Ph;
    const long long ho = (long long)r * g.Ph + jb;
    ldv<V>(g, B.f1, f1 + ho, hok);
    ldv<V>(g, B.f0, f0 + ho, hok);
    B.hxL = 0.f;
    B.ezR = B.hxR = B.hyR = B.caR = B.cbR = 0.f;
    if (lane == 0 && b0 > 0) B.hxL = ld1(g, hx + (long long)r * g.P + b0 - 1);
    if (lane == 31 && be < g.ny) {
        const long long oc = (long long)r * g.P + be;
        B.ezR = ld1(g, ez + oc);
        B.hxR = ld1(g, hx + oc);
        B.hyR = ld1(g, hy + oc);
        B.caR = ldc1(g, g.ca + oc);
        B.cbR = ldc1(g, g.cb + oc);
    }
}

// Adjoint E of row r for this lane's cells: residual injection (list order),
// then the E update from the old H (hu = Hy_old[r-1], hxl = Hx_old[r][b0+lV-1]).
template <int V, bool STORE>
__device__ __forceinline__ void adj_e_march(const GridDev& g, const AdjRow<V>& B, const float (&hu)[V], float hxl,
                                            int r, int q, int jb, bool core, const float* resid_s, int& cur, int end,
                                            const PsiShot& rd, const PsiShot& wr, float (&out)[V]) {
    float ez[V];
#pragma unroll
    for (int v = 0; v < V; ++v) ez[v] = B.ez[v];
    while (ev_seek(g.inj_ev, cur, end, r, q)) {
        const Ev e = __ldg(g.inj_ev + cur);
#pragma unroll
        for (int v = 0; v < V; ++v)
            if (jb + v == e.z) ez[v] = __fsub_rn(ez[v], resid_s[e.w]);
        ++cur;
    }
    if (core) {
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const float l = (v > 0) ? B.hx[(v + V - 1) % V] : hxl;
            out[v] = __fmaf_rn(-B.cb[v], __fsub_rn(B.hx[v], l), madd2(B.ca[v], ez[v], B.cb[v], __fsub_rn(B.hy[v], hu[v])));
        }
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const float l = (v > 0) ? B.hx[(v + V - 1) % V] : hxl;
            out[v] = ez[v];
            if (jb + v < g.ny)
                out[v] = e_update<STORE>(g, r, jb + v, ez[v], __fsub_rn(B.hy[v], hu[v]), __fsub_rn(B.hx[v], l), B.ca[v],
                                         B.cb[v], rd, wr);
        }
    }
}

// Adjoint E of the column be of row r (lane 31), old values from B, Hy_old[r-1][be] = huR.
template <int V>
__device__ __forceinline__ float adj_e_col(const GridDev& g, const AdjRow<V>& B, float huR, int r, int q, int be,
                                           const float* resid_s, int& cur, int end, const PsiShot& rd, bool active) {
    float ez = B.ezR;
    while (ev_seek(g.injh_ev, cur, end, r, q)) {
        const Ev e = __ldg(g.injh_ev + cur);
        if (active) ez = __fsub_rn(ez, resid_s[e.w]);
        ++cur;
    }
    if (!active || be >= g.ny) return 0.f;
    return e_update<false>(g, r, be, ez, __fsub_rn(B.hyR, huR), __fsub_rn(B.hxR, B.hx[V - 1]), B.caR, B.cbR, rd, rd);
}

__host__ __device__ inline size_t march_adj_smem(int TI, int V) {
    return (size_t)MARCH_WARPS * 2 * TI * 32 * V * sizeof(float);
}

template <int V>
__global__ void __launch_bounds__(32 * MARCH_WARPS) k_adjoint_march(const GridDev g, const int it, const int rp,
                                                                   const int G, const int TI) {
    extern __shared__ __align__(16) float acc_sm[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    TileM T;
    const int tile = blockIdx.x * MARCH_WARPS + warp;
    if (!march_tile(g, V, tile, T)) return;
    const int P = g.P, nx = g.nx, ny = g.ny;
    const int wp = rp ^ 1;
    const int jb = T.b0 + lane * V;
    const bool act = jb < P;
    const bool bcore_band = core_band(g, T.b0, T.be);
    const long long hplane = (long long)nx * g.Ph;
    const int ic0 = g.inj_off[tile], ie = g.inj_off[tile + 1];
    const int hc0 = g.injh_off[tile], he = g.injh_off[tile + 1];
    const bool bcore = bcore_band && ic0 == ie;
    // per-warp imaging accumulators [2][TI][32V], shot order within the group
    float* acc = acc_sm + (size_t)warp * 2 * TI * 32 * V;
    const int rows = T.i1 - T.i0;
    for (int k = lane; k < 2 * rows * 32 * V; k += 32) acc[k] = 0.f;
    __syncwarp();

    for (int q = 0; q < G; ++q) {
        const int s = T.grp * G + q;
        if (s >= g.S) break;
        const long long so = (long long)s * g.plane;
        const float* ezR = g.ez[rp] + so;
        const float* hxR = g.hx[rp] + so;
        const float* hyR = g.hy[rp] + so;
        const float* f1 = g.hist + ((long long)it * g.S + s) * hplane;
        const float* f0 = f1 - (long long)g.S * hplane;
        const float* resid_s = g.resid + ((long long)s * g.nt + it) * g.nrx;
        const PsiShot rd = psi_shot(g, rp, s), wr = psi_shot(g, wp, s);
        int ic = ic0, hc = hc0;

        AdjRow<V> B, Bn, Bnn;
        // old Hy of the row above the chunk (for E of row i0), and its column be
        float hu[V], huR = 0.f;
        ldv<V>(g, hu, hyR + (long long)(T.i0 - 1) * P + jb, act && T.i0 >= 1);
        if (lane == 31 && T.i0 >= 1 && T.be < ny) huR = ld1(g, hyR + (long long)(T.i0 - 1) * P + T.be);
        adj_row_load<V>(g, B, ezR, hxR, hyR, f1, f0, T.i0, jb, lane, T.b0, T.be, act, true);
        if (T.i0 + 1 < nx)
            adj_row_load<V>(g, Bn, ezR, hxR, hyR, f1, f0, T.i0 + 1, jb, lane, T.b0, T.be, act, T.i0 + 1 < T.i1);
        // E_new of row i0 and of its column be
        float ezc[V];
        {
            float hxl = __shfl_up_sync(FULL, B.hx[V - 1], 1);
            if (lane == 0) hxl = B.hxL;
            adj_e_march<V, true>(g, B, hu, hxl, T.i0, q, jb, bcore && core_row(g, T.i0), resid_s, ic, ie, rd, wr, ezc);
        }
        float ecol = adj_e_col<V>(g, B, huR, T.i0, q, T.be, resid_s, hc, he, rd, lane == 31);

#define FG_ADJ_ITER(CUR, NXT, LD)                                                                              \
    {                                                                                                          \
        const int r = i + 1;                                                                                   \
        if (r + 1 < nx && r + 1 <= T.i1)                                                                       \
            adj_row_load<V>(g, LD, ezR, hxR, hyR, f1, f0, r + 1, jb, lane, T.b0, T.be, act, r + 1 < T.i1);     \
        float ezr[V], ecol_r = 0.f;                                                                            \
        _Pragma("unroll") for (int v = 0; v < V; ++v) ezr[v] = 0.f;                                            \
        if (r < nx) {                                                                                          \
            float hxl = __shfl_up_sync(FULL, NXT.hx[V - 1], 1);                                                \
            if (lane == 0) hxl = NXT.hxL;                                                                      \
            const bool core_r = bcore && core_row(g, r);                                                       \
            if (r < T.i1) {                                                                                    \
                adj_e_march<V, true>(g, NXT, CUR.hy, hxl, r, q, jb, core_r, resid_s, ic, ie, rd, wr, ezr);     \
                ecol_r = adj_e_col<V>(g, NXT, CUR.hyR, r, q, T.be, resid_s, hc, he, rd, lane == 31);           \
            } else {                                                                                           \
                adj_e_march<V, false>(g, NXT, CUR.hy, hxl, r, q, jb, core_r, resid_s, ic, ie, rd, rd, ezr);    \
            }                                                                                                  \
        }                                                                                                      \
        float right = __shfl_down_sync(FULL, ezc[0], 1);                                                       \
        if (lane == 31) right = ecol;                                                                          \
        float hx[V], hy[V];                                                                                    \
        _Pragma("unroll") for (int v = 0; v < V; ++v) {                                                        \
            hx[v] = CUR.hx[v];                                                                                 \
            hy[v] = CUR.hy[v];                                                                                 \
        }                                                                                                      \
        if (bcore_band && core_row(g, i)) {                                                                    \
            _Pragma("unroll") for (int v = 0; v < V; ++v) {                                                    \
                const float er = (v + 1 < V) ? ezc[(v + 1) % V] : right;                                       \
                hx[v] = __fsub_rn(hx[v], __fmul_rn(CUR.ch[v], __fsub_rn(er, ezc[v])));                         \
                hy[v] = __fadd_rn(hy[v], __fmul_rn(CUR.ch[v], __fsub_rn(ezr[v], ezc[v])));                     \
            }                                                                                                  \
        } else {                                                                                               \
            _Pragma("unroll") for (int v = 0; v < V; ++v) {                                                    \
                const float er = (v + 1 < V) ? ezc[(v + 1) % V] : right;                                       \
                if (jb + v < ny)                                                                               \
                    h_update<true, true, true>(g, i, jb + v, hx[v], hy[v], __fsub_rn(er, ezc[v]),              \
                                               __fsub_rn(ezr[v], ezc[v]), CUR.ch[v], rd, wr);                  \
            }                                                                                                  \
        }                                                                                                      \
        {                                                                                                      \
            float* ae = acc + ((i - T.i0) * 32 + lane) * V;                                                    \
            float* as = ae + rows * 32 * V;                                                                    \
            _Pragma("unroll") for (int v = 0; v < V; ++v) {                                                    \
                ae[v] = __fadd_rn(ae[v], __fmul_rn(__fsub_rn(CUR.f1[v], CUR.f0[v]), ezc[v]));                  \
                as[v] = __fadd_rn(as[v], __fmul_rn(__fmul_rn(CUR.f1[v], ezc[v]), g.dt));                       \
            }                                                                                                  \
        }                                                                                                      \
        if (act) {                                                                                             \
            const long long o = so + (long long)i * P + jb;                                                    \
            st_state<V>(g, g.ez[wp] + o, ezc);                                                                 \
            st_state<V>(g, g.hx[wp] + o, hx);                                                                  \
            st_state<V>(g, g.hy[wp] + o, hy);                                                                  \
        }                                                                                                      \
        _Pragma("unroll") for (int v = 0; v < V; ++v) ezc[v] = ezr[v];                                         \
        ecol = ecol_r;                                                                                         \
    }

        // rotating row operands: iteration i uses (row i, row i+1) and loads row i+2
        for (int i = T.i0; i < T.i1;) {
            FG_ADJ_ITER(B, Bn, Bnn)
            if (++i >= T.i1) break;
            FG_ADJ_ITER(Bn, Bnn, B)
            if (++i >= T.i1) break;
            FG_ADJ_ITER(Bnn, B, Bn)
            ++i;
        }
#undef FG_ADJ_ITER
    }
    // group sums into the fp64 accumulators
    double* gae = g.gacc + (long long)T.grp * 2 * ((long long)nx * ny);
    double* gas = gae + (long long)nx * ny;
    for (int i = T.i0; i < T.i1; ++i) {
        const float* ae = acc + ((i - T.i0) * 32 + lane) * V;
        const float* as = ae + rows * 32 * V;
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int j = jb + v;
            if (j < ny) {
                const long long o = (long long)i * ny + j;
                gae[o] += (double)ae[v];
                gas[o] += (double)as[v];
            }
        }
    }
}

}  // namespace fg
