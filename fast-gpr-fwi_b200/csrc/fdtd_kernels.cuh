// The time-step kernels of the TMz FDTD solver.
//
// Work decomposition.  A solve has S shots on one (nx, ny) grid.  A *tile* is
// (shot group of G shots, row chunk [i0, i1), column band [b0, b0 + 32V)) and
// is owned by one warp; lane l holds columns b0 + l*V .. b0 + l*V + V-1 of every
// row.  The warp marches down the rows of its chunk, carrying the previous
// row in registers, so each cell's Ez/Hx/Hy is read once and written once per
// time step; left/right neighbours come from warp shuffles.  All state lives in
// ping-pong buffers (parity t&1 read, the other written), so the few values a
// tile needs from its neighbours (one halo row, one halo column) are recomputed
// from the previous step's state without any synchronisation inside a step.
//
// Forward step t (compute.py:574-712), per cell in this order: H interior,
// H CPML, E interior, E CPML, source injection, then receiver sample and Ez
// history store.  Receivers are sampled from the new Ez as trace[t+1], which is
// what the reference's store_outputs reads at the start of step t+1.
//
// Reference-mode adjoint step (compute.py:1048-1172): residual injection at
// the receivers, E interior (Ucgeta uE0) + E CPML from the old H, then H
// interior + H CPML from the new E, then the imaging sums with the stored
// forward Ez.  The march computes E one row ahead of H.
#pragma once

#include "fdtd_device.cuh"

namespace fg {

// ---------------------------------------------------------------------------
// Update coefficients: the reference's ucget / ucgeta (src/lib/uc.cu:11-45,
// :60-91) on the (nx, ny) model, written into pitched planes whose i == nx
// row and j >= ny columns stay zero.
// ---------------------------------------------------------------------------
__global__ void k_coefficients(const float* __restrict__ er, const float* __restrict__ se,
                               const float* __restrict__ mr, int nx, int ny, float dt, float dx,
                               int adjoint, float* __restrict__ out, int P) {
    const long long plane = (long long)(nx + 1) * P;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= plane) return;
    const int i = (int)(idx / P), j = (int)(idx % P);
    float uE0 = 0.f, uE1 = 0.f, uE4 = 0.f, uH1 = 0.f, uH4 = 0.f;
    if (i < nx && j < ny) {
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

struct TileInfo {
    int band, chunk, grp, i0, i1, b0, be, jb, lane;
};

__device__ __forceinline__ bool tile_info(const GridDev& g, int V, TileInfo& ti) {
    ti.lane = threadIdx.x & 31;
    const int tile = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (tile >= g.ntiles) return false;
    ti.band = tile % g.nb;
    const int rest = tile / g.nb;
    ti.chunk = rest % g.nc;
    ti.grp = rest / g.nc;
    ti.i0 = g.chunk_row[ti.chunk];
    ti.i1 = g.chunk_row[ti.chunk + 1];
    ti.b0 = ti.band * 32 * V;
    ti.be = ti.b0 + 32 * V;
    ti.jb = ti.b0 + ti.lane * V;
    return true;
}

__device__ __forceinline__ int tile_index() { return blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); }

// ---------------------------------------------------------------------------
// Forward step
// ---------------------------------------------------------------------------
template <int V, int G>
__global__ void __launch_bounds__(128) k_forward_step(const GridDev g, const int t) {
    TileInfo ti;
    if (!tile_info(g, V, ti)) return;
    const int tile = tile_index();
    const int nx = g.nx, ny = g.ny, P = g.P;
    const int rp = t & 1, wp = rp ^ 1;
    const int lane = ti.lane, jb = ti.jb, b0 = ti.b0, be = ti.be;
    const bool act = jb < P;
    const int s0 = ti.grp * G;

    float ezc[G][V], hyu[G][V];

    // Prologue: Ez of row i0 and the new Hy of the halo row i0-1.
#pragma unroll
    for (int q = 0; q < G; ++q) {
        const int s = s0 + q;
#pragma unroll
        for (int v = 0; v < V; ++v) { ezc[q][v] = 0.f; hyu[q][v] = 0.f; }
        if (s >= g.S) continue;
        const long long so = (long long)s * g.plane;
        if (act) ld_state<V>(g, ezc[q], g.ez[rp] + so + (long long)ti.i0 * P + jb);
        if (ti.i0 >= 1 && act) {
            const int ih = ti.i0 - 1;
            float eza[V], hyo[V], chv[V];
            ld_state<V>(g, eza, g.ez[rp] + so + (long long)ih * P + jb);
            ld_state<V>(g, hyo, g.hy[rp] + so + (long long)ih * P + jb);
            ld_coef<V>(g, chv, g.ch + (long long)ih * P + jb);
            const PsiShot rd = psi_shot(g, rp, s);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int j = jb + v;
                float hx_unused = 0.f, hy = hyo[v];
                if (j < ny) {
                    const float dzy = __fsub_rn(ezc[q][v], eza[v]);
                    h_update<false, false, true>(g, ih, j, hx_unused, hy, 0.f, dzy, chv[v], rd, rd);
                }
                hyu[q][v] = hy;
            }
        }
    }

    int sc = g.src_off[tile];
    const int se = g.src_off[tile + 1];
    int rc = g.rx_off[tile];
    const int re = g.rx_off[tile + 1];
    const long long hstride = (long long)nx * g.Ph;

    for (int i = ti.i0; i < ti.i1; ++i) {
        float cav[V], cbv[V], chv[V];
        if (act) {
            ld_coef<V>(g, cav, g.ca + (long long)i * P + jb);
            ld_coef<V>(g, cbv, g.cb + (long long)i * P + jb);
            ld_coef<V>(g, chv, g.ch + (long long)i * P + jb);
        } else {
#pragma unroll
            for (int v = 0; v < V; ++v) { cav[v] = 0.f; cbv[v] = 0.f; chv[v] = 0.f; }
        }
#pragma unroll
        for (int q = 0; q < G; ++q) {
            const int s = s0 + q;
            if (s >= g.S) continue;
            const long long so = (long long)s * g.plane;
            const long long ro = so + (long long)i * P;
            float ezn[V], hxo[V], hyo[V];
            if (act) {
                ld_state<V>(g, ezn, g.ez[rp] + ro + P + jb);
                ld_state<V>(g, hxo, g.hx[rp] + ro + jb);
                ld_state<V>(g, hyo, g.hy[rp] + ro + jb);
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) { ezn[v] = 0.f; hxo[v] = 0.f; hyo[v] = 0.f; }
            }
            const PsiShot rd = psi_shot(g, rp, s);
            const PsiShot wr = psi_shot(g, wp, s);

            // Ez[i][b0 + 32V] for the band's last column: from the next lane,
            // or the neighbouring band for lane 31.
            float ez_r = __shfl_down_sync(FULL, ezc[q][0], 1);
            if (lane == 31) ez_r = (be < P) ? ld1(g, g.ez[rp] + ro + be) : 0.f;

            float hxn[V], hyn[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int j = jb + v;
                hxn[v] = hxo[v];
                hyn[v] = hyo[v];
                if (j < ny) {
                    const float er_ = (v + 1 < V) ? ezc[q][(v + 1) % V] : ez_r;
                    const float dzx = __fsub_rn(er_, ezc[q][v]);
                    const float dzy = __fsub_rn(ezn[v], ezc[q][v]);
                    h_update<true, true, true>(g, i, j, hxn[v], hyn[v], dzx, dzy, chv[v], rd, wr);
                }
            }
            // new Hx of column b0-1: from the previous lane, or recomputed for lane 0
            float hx_l = __shfl_up_sync(FULL, hxn[V - 1], 1);
            if (lane == 0) {
                hx_l = 0.f;
                if (b0 > 0) {
                    const int j = b0 - 1;
                    float hx = ld1(g, g.hx[rp] + ro + j), hy_unused = 0.f;
                    const float dzx = __fsub_rn(ezc[q][0], ld1(g, g.ez[rp] + ro + j));
                    h_update<false, true, false>(g, i, j, hx, hy_unused, dzx, 0.f, ldc1(g, g.ch + (long long)i * P + j),
                                                 rd, rd);
                    hx_l = hx;
                }
            }
            float ezw[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int j = jb + v;
                ezw[v] = ezc[q][v];
                if (j < ny) {
                    const float hxl = (v > 0) ? hxn[(v + V - 1) % V] : hx_l;
                    const float dhy = __fsub_rn(hyn[v], hyu[q][v]);
                    const float dhx = __fsub_rn(hxn[v], hxl);
                    ezw[v] = e_update<true>(g, i, j, ezc[q][v], dhy, dhx, cav[v], cbv[v], rd, wr);
                }
            }
            // Hertzian dipole, Ez -= uE4 * w[n][t] * dl/(dx dy dz)  (sourcereceiver.cu:84)
            while (sc < se) {
                const Ev e = __ldg(g.src_ev + sc);
                if (e.x != i || e.y != q) break;
#pragma unroll
                for (int v = 0; v < V; ++v)
                    if (jb + v == e.z) {
                        const float cd = ldc1(g, g.cd + (long long)i * P + e.z);
                        ezw[v] = __fmaf_rn(-cd, ldc1(g, g.srcw + (long long)e.w * g.nt + t), ezw[v]);
                    }
                ++sc;
            }
            if (act) {
                st_state<V>(g, g.ez[wp] + ro + jb, ezw);
                st_state<V>(g, g.hx[wp] + ro + jb, hxn);
                st_state<V>(g, g.hy[wp] + ro + jb, hyn);
            }
            if (g.hist) {
                float* hrow = g.hist + ((long long)t * g.S + s) * hstride + (long long)i * g.Ph;
#pragma unroll
                for (int v = 0; v < V; ++v)
                    if (jb + v < ny) hrow[jb + v] = ezw[v];
            }
            // receivers: trace[s][t+1][r] = Ez after this step (store_outputs of step t+1)
            while (rc < re) {
                const Ev e = __ldg(g.rx_ev + rc);
                if (e.x != i || e.y != q) break;
                if (t + 1 < g.nt) {
#pragma unroll
                    for (int v = 0; v < V; ++v)
                        if (jb + v == e.z) g.traces[((long long)s * g.nt + t + 1) * g.nrx + e.w] = ezw[v];
                }
                ++rc;
            }
#pragma unroll
            for (int v = 0; v < V; ++v) { ezc[q][v] = ezn[v]; hyu[q][v] = hyn[v]; }
        }
    }
}

// ---------------------------------------------------------------------------
// Reference-mode adjoint step (one reversed iteration `it`, reading parity rp).
// ---------------------------------------------------------------------------

// Adjoint E of one cell computed from the previous-step state only (used for
// the halo column b0+32V).  ez is Ez_old[i][j] after residual injection,
// hx_l is Hx_old[i][j-1].
__device__ __forceinline__ float adj_e_cell(const GridDev& g, int rp, int s, int i, int j, float hx_l,
                                            float ez) {
    const int P = g.P;
    const long long o = (long long)s * g.plane + (long long)i * P + j;
    const float hy_c = ld1(g, g.hy[rp] + o);
    const float hy_u = (i >= 1) ? ld1(g, g.hy[rp] + o - P) : 0.f;
    const float hx_c = ld1(g, g.hx[rp] + o);
    const PsiShot rd = psi_shot(g, rp, s);
    const float ca = ldc1(g, g.ca + (long long)i * P + j);
    const float cb = ldc1(g, g.cb + (long long)i * P + j);
    return e_update<false>(g, i, j, ez, __fsub_rn(hy_c, hy_u), __fsub_rn(hx_c, hx_l), ca, cb, rd, rd);
}

template <int V, int G>
__global__ void __launch_bounds__(128) k_adjoint_step(const GridDev g, const int it, const int rp) {
    TileInfo ti;
    if (!tile_info(g, V, ti)) return;
    const int tile = tile_index();
    const int nx = g.nx, ny = g.ny, P = g.P;
    const int wp = rp ^ 1;
    const int lane = ti.lane, jb = ti.jb, b0 = ti.b0, be = ti.be;
    const bool act = jb < P;
    const int s0 = ti.grp * G;
    const float* resid_t = g.resid + (long long)it * g.nrx;   // + s*nt*nrx + r

    float ezc[G][V], hyc[G][V], hxc[G][V];   // E_new, Hy_old, Hx_old of the current row
    int ic = g.inj_off[tile];
    const int ie = g.inj_off[tile + 1];
    int hc = g.injh_off[tile];
    const int he = g.injh_off[tile + 1];

    // Prologue: E_new of row i0.
#pragma unroll
    for (int q = 0; q < G; ++q) {
        const int s = s0 + q;
#pragma unroll
        for (int v = 0; v < V; ++v) { ezc[q][v] = 0.f; hyc[q][v] = 0.f; hxc[q][v] = 0.f; }
        if (s >= g.S) continue;
        const long long ro = (long long)s * g.plane + (long long)ti.i0 * P;
        const int i = ti.i0;
        float ezo[V], hyu[V], cav[V], cbv[V];
#pragma unroll
        for (int v = 0; v < V; ++v) { ezo[v] = 0.f; hyu[v] = 0.f; cav[v] = 0.f; cbv[v] = 0.f; }
        if (act) {
            ld_state<V>(g, ezo, g.ez[rp] + ro + jb);
            ld_state<V>(g, hyc[q], g.hy[rp] + ro + jb);
            ld_state<V>(g, hxc[q], g.hx[rp] + ro + jb);
            if (i >= 1) ld_state<V>(g, hyu, g.hy[rp] + ro - P + jb);
            ld_coef<V>(g, cav, g.ca + (long long)i * P + jb);
            ld_coef<V>(g, cbv, g.cb + (long long)i * P + jb);
        }
        float hx_l = __shfl_up_sync(FULL, hxc[q][V - 1], 1);
        if (lane == 0) hx_l = (b0 > 0) ? ld1(g, g.hx[rp] + ro + b0 - 1) : 0.f;
        while (ic < ie) {
            const Ev e = __ldg(g.inj_ev + ic);
            if (e.x != i || e.y != q) break;
#pragma unroll
            for (int v = 0; v < V; ++v)
                if (jb + v == e.z) ezo[v] = __fsub_rn(ezo[v], resid_t[(long long)s * g.nt * g.nrx + e.w]);
            ++ic;
        }
        const PsiShot rd = psi_shot(g, rp, s);
        const PsiShot wr = psi_shot(g, wp, s);
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int j = jb + v;
            ezc[q][v] = ezo[v];
            if (j < ny) {
                const float hxl = (v > 0) ? hxc[q][(v + V - 1) % V] : hx_l;
                ezc[q][v] = e_update<true>(g, i, j, ezo[v], __fsub_rn(hyc[q][v], hyu[v]), __fsub_rn(hxc[q][v], hxl),
                                           cav[v], cbv[v], rd, wr);
            }
        }
    }

    const long long hstride = (long long)nx * g.Ph;
    const long long gstride = (long long)nx * ny;
    const float* f1b = g.hist + (long long)it * g.S * hstride;
    const float* f0b = g.hist + (long long)(it - 1) * g.S * hstride;
    double* gae = g.gacc + (long long)ti.grp * 2 * gstride;
    double* gas = gae + gstride;

    for (int i = ti.i0; i < ti.i1; ++i) {
        const int r = i + 1;
        float cav[V], cbv[V], chv[V];
#pragma unroll
        for (int v = 0; v < V; ++v) { cav[v] = 0.f; cbv[v] = 0.f; chv[v] = 0.f; }
        if (act) {
            if (r < nx) {
                ld_coef<V>(g, cav, g.ca + (long long)r * P + jb);
                ld_coef<V>(g, cbv, g.cb + (long long)r * P + jb);
            }
            ld_coef<V>(g, chv, g.ch + (long long)i * P + jb);
        }
        float acc_e[V], acc_s[V];
#pragma unroll
        for (int v = 0; v < V; ++v) { acc_e[v] = 0.f; acc_s[v] = 0.f; }

#pragma unroll
        for (int q = 0; q < G; ++q) {
            const int s = s0 + q;
            if (s >= g.S) continue;
            const long long so = (long long)s * g.plane;
            const long long ro = so + (long long)i * P;
            const PsiShot rd = psi_shot(g, rp, s);
            const PsiShot wr = psi_shot(g, wp, s);

            // --- E of row r = i+1 (stored auxiliaries only for owned rows)
            float ezr[V], hyr[V], hxr[V];
#pragma unroll
            for (int v = 0; v < V; ++v) { ezr[v] = 0.f; hyr[v] = 0.f; hxr[v] = 0.f; }
            if (r < nx) {
                float ezo[V];
#pragma unroll
                for (int v = 0; v < V; ++v) ezo[v] = 0.f;
                if (act) {
                    ld_state<V>(g, ezo, g.ez[rp] + ro + P + jb);
                    ld_state<V>(g, hyr, g.hy[rp] + ro + P + jb);
                    ld_state<V>(g, hxr, g.hx[rp] + ro + P + jb);
                }
                float hx_l = __shfl_up_sync(FULL, hxr[V - 1], 1);
                if (lane == 0) hx_l = (b0 > 0) ? ld1(g, g.hx[rp] + ro + P + b0 - 1) : 0.f;
                while (ic < ie) {
                    const Ev e = __ldg(g.inj_ev + ic);
                    if (e.x != r || e.y != q) break;
#pragma unroll
                    for (int v = 0; v < V; ++v)
                        if (jb + v == e.z) ezo[v] = __fsub_rn(ezo[v], resid_t[(long long)s * g.nt * g.nrx + e.w]);
                    ++ic;
                }
                const bool own = r < ti.i1;
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const int j = jb + v;
                    ezr[v] = ezo[v];
                    if (j < ny) {
                        const float hxl = (v > 0) ? hxr[(v + V - 1) % V] : hx_l;
                        const float dhy = __fsub_rn(hyr[v], hyc[q][v]);
                        const float dhx = __fsub_rn(hxr[v], hxl);
                        ezr[v] = own ? e_update<true>(g, r, j, ezo[v], dhy, dhx, cav[v], cbv[v], rd, wr)
                                     : e_update<false>(g, r, j, ezo[v], dhy, dhx, cav[v], cbv[v], rd, rd);
                    }
                }
            }

            // --- H of row i from E_new of rows i and i+1
            // E_new[i][b0 + 32V]: from the next lane, or recomputed by lane 31
            // (including any residual injected at that cell, in order).
            float ez_r = __shfl_down_sync(FULL, ezc[q][0], 1);
            float ez_h = 0.f;
            if (lane == 31 && be < ny) ez_h = ld1(g, g.ez[rp] + ro + be);
            while (hc < he) {
                const Ev e = __ldg(g.injh_ev + hc);
                if (e.x != i || e.y != q) break;
                if (lane == 31) ez_h = __fsub_rn(ez_h, resid_t[(long long)s * g.nt * g.nrx + e.w]);
                ++hc;
            }
            if (lane == 31) ez_r = (be < ny) ? adj_e_cell(g, rp, s, i, be, hxc[q][V - 1], ez_h) : 0.f;

            float hxn[V], hyn[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int j = jb + v;
                hxn[v] = hxc[q][v];
                hyn[v] = hyc[q][v];
                if (j < ny) {
                    const float er_ = (v + 1 < V) ? ezc[q][(v + 1) % V] : ez_r;
                    const float dzx = __fsub_rn(er_, ezc[q][v]);
                    const float dzy = __fsub_rn(ezr[v], ezc[q][v]);
                    h_update<true, true, true>(g, i, j, hxn[v], hyn[v], dzx, dzy, chv[v], rd, wr);
                    // imaging, compute.py:1167-1172
                    const long long hidx = (long long)s * hstride + (long long)i * g.Ph + j;
                    const float f1 = __ldg(f1b + hidx), f0 = __ldg(f0b + hidx);
                    acc_e[v] = __fadd_rn(acc_e[v], __fmul_rn(__fsub_rn(f1, f0), ezc[q][v]));
                    acc_s[v] = __fadd_rn(acc_s[v], __fmul_rn(__fmul_rn(f1, ezc[q][v]), g.dt));
                }
            }
            if (act) {
                st_state<V>(g, g.ez[wp] + ro + jb, ezc[q]);
                st_state<V>(g, g.hx[wp] + ro + jb, hxn);
                st_state<V>(g, g.hy[wp] + ro + jb, hyn);
            }
#pragma unroll
            for (int v = 0; v < V; ++v) { ezc[q][v] = ezr[v]; hyc[q][v] = hyr[v]; hxc[q][v] = hxr[v]; }
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int j = jb + v;
            if (j < ny) {
                const long long o = (long long)i * ny + j;
                gae[o] += (double)acc_e[v];
                gas[o] += (double)acc_s[v];
            }
        }
    }
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
    for (int k = 0; k < nblocks; ++k) { a += partial[2 * k]; b += partial[2 * k + 1]; }
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
