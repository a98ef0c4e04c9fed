// Tiled time-step kernels: one CTA per (shot group, row chunk, column band)
// tile of TH rows x 32V columns, one warp per row.  Each CTA stages the old
// state of its tile plus a one-cell halo in shared memory, computes the
// first-half update (H in the forward, E in the adjoint) on the tile and the
// halo cells its second half needs, synchronises, and finishes the step.
// Everything a CTA reads comes from the previous step's buffers (ping-pong),
// so CTAs never wait on each other within a step; latency is hidden by
// running many small CTAs per SM.
//
// The per-cell arithmetic is the device code of fdtd_device.cuh, so results
// are bit-identical to the other kernels and to the reference.
#pragma once

#include "fdtd_device.cuh"

namespace fg {

struct TileT {
    int band, chunk, grp, i0, i1, b0, be;
};

__device__ __forceinline__ TileT tile_t(const GridDev& g, int V) {
    TileT t;
    const int tile = blockIdx.x;
    t.band = tile % g.nb;
    const int rest = tile / g.nb;
    t.chunk = rest % g.nc;
    t.grp = rest / g.nc;
    t.i0 = g.chunk_row[t.chunk];
    t.i1 = g.chunk_row[t.chunk + 1];
    t.b0 = t.band * 32 * V;
    t.be = t.b0 + 32 * V;
    return t;
}

// ---------------------------------------------------------------------------
// Forward step.  Shared memory (floats):
//   ez_s  [TH+2][SE]   Ez_old rows i0-1 .. i0+TH, columns b0-1 .. be   (SE = 32V+2)
//   hx_s  [TH  ][SX]   Hx_new rows i0 .. i0+TH-1, columns b0-1 .. be-1 (SX = 32V+1)
//   hy_s  [TH+1][SY]   Hy_new rows i0-1 .. i0+TH-1, columns b0 .. be-1 (SY = 32V)
// ---------------------------------------------------------------------------
__host__ __device__ inline size_t tile_fwd_smem(int TH, int V) {
    return sizeof(float) * ((size_t)(TH + 2) * (32 * V + 2) + (size_t)TH * (32 * V + 1) + (size_t)(TH + 1) * 32 * V);
}

template <int V>
__global__ void __launch_bounds__(512, 2) k_forward_tile(const GridDev g, const int t, const int G) {
    extern __shared__ float sm[];
    const int TH = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const TileT T = tile_t(g, V);
    const int SE = 32 * V + 2, SX = 32 * V + 1, SY = 32 * V;
    float* ez_s = sm;
    float* hx_s = ez_s + (TH + 2) * SE;
    float* hy_s = hx_s + TH * SX;
    const int nx = g.nx, ny = g.ny, P = g.P;
    const int rp = t & 1, wp = rp ^ 1;
    const int i = T.i0 + ty;
    const bool row_ok = i < T.i1;
    const int rows = T.i1 - T.i0;
    const int jb = T.b0 + lane * V;
    const int cs = lane * V;          // column of this thread's first cell within the band
    const bool act = jb < P;
    const long long hplane = (long long)nx * g.Ph;

    // per-tile event cursors; events are sorted by (row, shot slot, column)
    const int sc0 = g.src_off[blockIdx.x], se = g.src_off[blockIdx.x + 1];
    const int rc0 = g.rx_off[blockIdx.x], re = g.rx_off[blockIdx.x + 1];

    float ca[V], cb[V], ch[V];
    for (int v = 0; v < V; ++v) { ca[v] = 0.f; cb[v] = 0.f; ch[v] = 0.f; }
    if (row_ok && act) {
        ld_coef<V>(g, ca, g.ca + (long long)i * P + jb);
        ld_coef<V>(g, cb, g.cb + (long long)i * P + jb);
        ld_coef<V>(g, ch, g.ch + (long long)i * P + jb);
    }

    for (int q = 0; q < G; ++q) {
        const int s = T.grp * G + q;
        if (s >= g.S) break;
        const long long so = (long long)s * g.plane;
        const PsiShot rd = psi_shot(g, rp, s), wr = psi_shot(g, wp, s);
        // ---- stage Ez_old (tile + halo) and the old H values this thread updates
        float hx[V], hy[V], ezo[V];
        for (int v = 0; v < V; ++v) { hx[v] = 0.f; hy[v] = 0.f; ezo[v] = 0.f; }
        if (row_ok) {
            if (act) {
                ld_state<V>(g, ezo, g.ez[rp] + so + (long long)i * P + jb);
                ld_state<V>(g, hx, g.hx[rp] + so + (long long)i * P + jb);
                ld_state<V>(g, hy, g.hy[rp] + so + (long long)i * P + jb);
            }
            for (int v = 0; v < V; ++v) ez_s[(1 + ty) * SE + 1 + cs + v] = ezo[v];
            if (lane == 0) ez_s[(1 + ty) * SE] = T.b0 > 0 ? ld1(g, g.ez[rp] + so + (long long)i * P + T.b0 - 1) : 0.f;
            if (lane == 31) ez_s[(1 + ty) * SE + SE - 1] = T.be < P ? ld1(g, g.ez[rp] + so + (long long)i * P + T.be) : 0.f;
        }
        if (ty == 0) {
            // row above the tile (for the halo Hy) and row below (Ez[i1], the frame when i1 == nx)
            float a[V], b[V];
            for (int v = 0; v < V; ++v) { a[v] = 0.f; b[v] = 0.f; }
            if (act && T.i0 >= 1) ld_state<V>(g, a, g.ez[rp] + so + (long long)(T.i0 - 1) * P + jb);
            if (act) ld_state<V>(g, b, g.ez[rp] + so + (long long)T.i1 * P + jb);
            for (int v = 0; v < V; ++v) {
                ez_s[cs + 1 + v] = a[v];
                ez_s[(rows + 1) * SE + 1 + cs + v] = b[v];
            }
        }
        __syncthreads();
        // ---- H of the tile, the halo column b0-1 (Hx) and the halo row i0-1 (Hy)
        if (row_ok) {
            const float* er = ez_s + (1 + ty) * SE + 1;
            const float* en = er + SE;
            for (int v = 0; v < V; ++v) {
                const int j = jb + v, c = cs + v;
                if (j < ny)
                    h_update<true, true, true>(g, i, j, hx[v], hy[v], __fsub_rn(er[c + 1], er[c]),
                                               __fsub_rn(en[c], er[c]), ch[v], rd, wr);
                hx_s[ty * SX + 1 + c] = hx[v];
                hy_s[(1 + ty) * SY + c] = hy[v];
            }
            if (lane == 0) {
                float hl = 0.f, hy_unused = 0.f;
                if (T.b0 > 0) {
                    const int j = T.b0 - 1;
                    hl = ld1(g, g.hx[rp] + so + (long long)i * P + j);
                    h_update<false, true, false>(g, i, j, hl, hy_unused, __fsub_rn(er[0], er[-1]), 0.f,
                                                 ldc1(g, g.ch + (long long)i * P + j), rd, rd);
                }
                hx_s[ty * SX] = hl;
            }
        }
        if (ty == 0) {
            const int ih = T.i0 - 1;
            for (int v = 0; v < V; ++v) {
                const int j = jb + v, c = cs + v;
                float h = 0.f, hx_unused = 0.f;
                if (ih >= 0 && j < ny) {
                    h = ld1(g, g.hy[rp] + so + (long long)ih * P + j);
                    h_update<false, false, true>(g, ih, j, hx_unused, h, 0.f,
                                                 __fsub_rn(ez_s[SE + 1 + c], ez_s[1 + c]),
                                                 ldc1(g, g.ch + (long long)ih * P + j), rd, rd);
                }
                hy_s[c] = h;
            }
        }
        __syncthreads();
        // ---- E of the tile, sources, stores, history, receivers
        if (row_ok) {
            float ezw[V];
            for (int v = 0; v < V; ++v) {
                const int j = jb + v, c = cs + v;
                ezw[v] = ezo[v];
                if (j < ny) {
                    const float dhy = __fsub_rn(hy_s[(1 + ty) * SY + c], hy_s[ty * SY + c]);
                    const float dhx = __fsub_rn(hx_s[ty * SX + 1 + c], hx_s[ty * SX + c]);
                    ezw[v] = e_update<true>(g, i, j, ezo[v], dhy, dhx, ca[v], cb[v], rd, wr);
                }
            }
            for (int k = sc0; k < se; ++k) {
                const Ev e = __ldg(g.src_ev + k);
                if (e.x != i || e.y != q) continue;
                for (int v = 0; v < V; ++v)
                    if (jb + v == e.z) {
                        const float cd = ldc1(g, g.cd + (long long)i * P + e.z);
                        ezw[v] = __fmaf_rn(-cd, __ldg(g.srcw + (long long)e.w * g.nt + t), ezw[v]);
                    }
            }
            if (act) {
                const long long ro = so + (long long)i * P + jb;
                st_state<V>(g, g.ez[wp] + ro, ezw);
                st_state<V>(g, g.hx[wp] + ro, hx);
                st_state<V>(g, g.hy[wp] + ro, hy);
            }
            if (g.hist && jb < g.Ph)
                st_state<V>(g, g.hist + ((long long)t * g.S + s) * hplane + (long long)i * g.Ph + jb, ezw);
            if (t + 1 < g.nt) {
                for (int k = rc0; k < re; ++k) {
                    const Ev e = __ldg(g.rx_ev + k);
                    if (e.x != i || e.y != q) continue;
                    for (int v = 0; v < V; ++v)
                        if (jb + v == e.z) g.traces[((long long)s * g.nt + t + 1) * g.nrx + e.w] = ezw[v];
                }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Reference-mode adjoint step.  Shared memory (floats):
//   hy_s  [TH+2][SB]   Hy_old rows i0-1 .. i1,      columns b0 .. be     (SB = 32V+1)
//   hx_s  [TH+1][SX2]  Hx_old rows i0 .. i1,        columns b0-1 .. be   (SX2 = 32V+2)
//   en_s  [TH+1][SB]   E_new  rows i0 .. i1,        columns b0 .. be
// ---------------------------------------------------------------------------
__host__ __device__ inline size_t tile_adj_smem(int TH, int V) {
    return sizeof(float) * ((size_t)(TH + 2) * (32 * V + 1) + (size_t)(TH + 1) * (32 * V + 2) +
                            (size_t)(TH + 1) * (32 * V + 1));
}

// Adjoint E of cell (r, j) of shot s (with the residuals injected there, in
// list order) from the staged old H values; STORE writes the auxiliaries.
template <bool STORE>
__device__ __forceinline__ float adj_e_tile(const GridDev& g, int r, int j, int q, int s, float ez, float hy_c,
                                            float hy_u, float hx_c, float hx_l, const Ev* ev, int k0, int k1,
                                            const float* resid_s, const PsiShot& rd, const PsiShot& wr) {
    for (int k = k0; k < k1; ++k) {
        const Ev e = __ldg(ev + k);
        if (e.x == r && e.y == q && e.z == j) ez = __fsub_rn(ez, resid_s[e.w]);
    }
    const long long c = (long long)r * g.P + j;
    return e_update<STORE>(g, r, j, ez, __fsub_rn(hy_c, hy_u), __fsub_rn(hx_c, hx_l), ldc1(g, g.ca + c),
                           ldc1(g, g.cb + c), rd, wr);
}

template <int V>
__global__ void __launch_bounds__(512, 2) k_adjoint_tile(const GridDev g, const int it, const int rp, const int G) {
    extern __shared__ float sm[];
    const int TH = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const TileT T = tile_t(g, V);
    const int SB = 32 * V + 1, SX2 = 32 * V + 2;
    float* hy_s = sm;
    float* hx_s = hy_s + (TH + 2) * SB;
    float* en_s = hx_s + (TH + 1) * SX2;
    const int nx = g.nx, ny = g.ny, P = g.P;
    const int wp = rp ^ 1;
    const int i = T.i0 + ty;
    const bool row_ok = i < T.i1;
    const int rows = T.i1 - T.i0;
    const bool last_row = ty == rows - 1;
    const int jb = T.b0 + lane * V;
    const int cs = lane * V;
    const bool act = jb < P;
    const int i1 = T.i1, be = T.be;
    const long long hplane = (long long)nx * g.Ph;
    const int ic0 = g.inj_off[blockIdx.x], ie = g.inj_off[blockIdx.x + 1];
    const int hc0 = g.injh_off[blockIdx.x], he = g.injh_off[blockIdx.x + 1];

    float acc_e[V], acc_s[V];
    for (int v = 0; v < V; ++v) { acc_e[v] = 0.f; acc_s[v] = 0.f; }

    for (int q = 0; q < G; ++q) {
        const int s = T.grp * G + q;
        if (s >= g.S) break;
        const long long so = (long long)s * g.plane;
        const PsiShot rd = psi_shot(g, rp, s), wr = psi_shot(g, wp, s);
        const float* resid_s = g.resid + ((long long)s * g.nt + it) * g.nrx;
        // ---- stage old H (tile + halo) and this thread's old Ez
        float ezo[V], hxo[V], hyo[V];
        for (int v = 0; v < V; ++v) { ezo[v] = 0.f; hxo[v] = 0.f; hyo[v] = 0.f; }
        if (row_ok) {
            const long long ro = so + (long long)i * P;
            if (act) {
                ld_state<V>(g, ezo, g.ez[rp] + ro + jb);
                ld_state<V>(g, hxo, g.hx[rp] + ro + jb);
                ld_state<V>(g, hyo, g.hy[rp] + ro + jb);
            }
            for (int v = 0; v < V; ++v) {
                hy_s[(1 + ty) * SB + cs + v] = hyo[v];
                hx_s[ty * SX2 + 1 + cs + v] = hxo[v];
            }
            if (lane == 0) hx_s[ty * SX2] = T.b0 > 0 ? ld1(g, g.hx[rp] + ro + T.b0 - 1) : 0.f;
            if (lane == 31) {
                hx_s[ty * SX2 + SX2 - 1] = be < P ? ld1(g, g.hx[rp] + ro + be) : 0.f;
                hy_s[(1 + ty) * SB + SB - 1] = be < P ? ld1(g, g.hy[rp] + ro + be) : 0.f;
            }
        }
        if (ty == 0) {
            // Hy row i0-1 (columns b0 .. be); Hx and Hy of the halo row i1
            float a[V], bx[V], by[V];
            for (int v = 0; v < V; ++v) { a[v] = 0.f; bx[v] = 0.f; by[v] = 0.f; }
            if (act && T.i0 >= 1) ld_state<V>(g, a, g.hy[rp] + so + (long long)(T.i0 - 1) * P + jb);
            if (act && i1 < nx) {
                ld_state<V>(g, bx, g.hx[rp] + so + (long long)i1 * P + jb);
                ld_state<V>(g, by, g.hy[rp] + so + (long long)i1 * P + jb);
            }
            for (int v = 0; v < V; ++v) {
                hy_s[cs + v] = a[v];
                hx_s[rows * SX2 + 1 + cs + v] = bx[v];
                hy_s[(rows + 1) * SB + cs + v] = by[v];
            }
            if (lane == 0) {
                hy_s[SB - 1] = (T.i0 >= 1 && be < P) ? ld1(g, g.hy[rp] + so + (long long)(T.i0 - 1) * P + be) : 0.f;
                hx_s[rows * SX2] = (T.b0 > 0 && i1 < nx) ? ld1(g, g.hx[rp] + so + (long long)i1 * P + T.b0 - 1) : 0.f;
            }
        }
        __syncthreads();
        // ---- E_new of the tile, of the halo row i1 and of the halo column be
        if (row_ok) {
            for (int v = 0; v < V; ++v) {
                const int j = jb + v, c = cs + v;
                float e = ezo[v];
                if (j < ny)
                    e = adj_e_tile<true>(g, i, j, q, s, ezo[v], hy_s[(1 + ty) * SB + c], hy_s[ty * SB + c],
                                         hx_s[ty * SX2 + 1 + c], hx_s[ty * SX2 + c], g.inj_ev, ic0, ie, resid_s, rd,
                                         wr);
                en_s[ty * SB + c] = e;
            }
            if (lane == 31) {
                float e = 0.f;
                if (be < ny) {
                    const float ez = ld1(g, g.ez[rp] + so + (long long)i * P + be);
                    e = adj_e_tile<false>(g, i, be, q, s, ez, hy_s[(1 + ty) * SB + SB - 1], hy_s[ty * SB + SB - 1],
                                          hx_s[ty * SX2 + SX2 - 1], hx_s[ty * SX2 + SX2 - 2], g.injh_ev, hc0, he,
                                          resid_s, rd, rd);
                }
                en_s[ty * SB + SB - 1] = e;
            }
        }
        if (last_row) {
            for (int v = 0; v < V; ++v) {
                const int j = jb + v, c = cs + v;
                float e = 0.f;
                if (i1 < nx && j < ny) {
                    const float ez = ld1(g, g.ez[rp] + so + (long long)i1 * P + j);
                    e = adj_e_tile<false>(g, i1, j, q, s, ez, hy_s[(rows + 1) * SB + c], hy_s[rows * SB + c],
                                          hx_s[rows * SX2 + 1 + c], hx_s[rows * SX2 + c], g.inj_ev, ic0, ie, resid_s,
                                          rd, rd);
                }
                en_s[rows * SB + c] = e;
            }
        }
        __syncthreads();
        // ---- H of the tile, imaging, stores
        if (row_ok) {
            float hxn[V], hyn[V], ezn[V];
            const float* er = en_s + ty * SB;
            const float* enx = er + SB;
            float ch[V];
            for (int v = 0; v < V; ++v) ch[v] = 0.f;
            if (act) ld_coef<V>(g, ch, g.ch + (long long)i * P + jb);
            float f1[V], f0[V];
            for (int v = 0; v < V; ++v) { f1[v] = 0.f; f0[v] = 0.f; }
            if (jb < g.Ph) {
                const float* h1 = g.hist + (((long long)it * g.S + s) * nx + i) * g.Ph + jb;
                ld_state<V>(g, f1, h1);
                ld_state<V>(g, f0, h1 - (long long)g.S * hplane);
            }
            for (int v = 0; v < V; ++v) {
                const int j = jb + v, c = cs + v;
                hxn[v] = hxo[v];
                hyn[v] = hyo[v];
                ezn[v] = er[c];
                if (j < ny) {
                    h_update<true, true, true>(g, i, j, hxn[v], hyn[v], __fsub_rn(er[c + 1], er[c]),
                                               __fsub_rn(enx[c], er[c]), ch[v], rd, wr);
                    acc_e[v] = __fadd_rn(acc_e[v], __fmul_rn(__fsub_rn(f1[v], f0[v]), er[c]));
                    acc_s[v] = __fadd_rn(acc_s[v], __fmul_rn(__fmul_rn(f1[v], er[c]), g.dt));
                }
            }
            if (act) {
                const long long ro = so + (long long)i * P + jb;
                st_state<V>(g, g.ez[wp] + ro, ezn);
                st_state<V>(g, g.hx[wp] + ro, hxn);
                st_state<V>(g, g.hy[wp] + ro, hyn);
            }
        }
        __syncthreads();
    }
    if (row_ok) {
        double* gae = g.gacc + (long long)T.grp * 2 * ((long long)nx * ny);
        double* gas = gae + (long long)nx * ny;
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

}  // namespace fg
