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

// Whether every cell a warp updates in row i is a plain interior cell: no
// CPML slab, not on the i == 0 / j == 0 edges, all columns < ny.  Such warps
// take the lean path (same arithmetic, no per-cell boundary tests).
__device__ __forceinline__ bool core_warp(const GridDev& g, int i, int b0, int be) {
    const int th = g.th;
    return i >= th + 1 && i <= g.nx - th - 1 && b0 >= th + 1 && be <= g.ny - th;
}

template <int V>
__device__ __forceinline__ void lds_v(float (&x)[V], const float* p) {
    if constexpr (V == 4) {
        const float4 q = *reinterpret_cast<const float4*>(p);
        x[0] = q.x; x[1] = q.y; x[2] = q.z; x[3] = q.w;
    } else if constexpr (V == 2) {
        const float2 q = *reinterpret_cast<const float2*>(p);
        x[0] = q.x; x[1] = q.y;
    } else {
        x[0] = *p;
    }
}
template <int V>
__device__ __forceinline__ void sts_v(float* p, const float (&x)[V]) {
    if constexpr (V == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(x[0], x[1], x[2], x[3]);
    } else if constexpr (V == 2) {
        *reinterpret_cast<float2*>(p) = make_float2(x[0], x[1]);
    } else {
        *p = x[0];
    }
}

// ---------------------------------------------------------------------------
// Forward step.  Shared memory (floats), own cells of a row at offset 4 so
// that vector accesses are aligned:
//   ez_s  [TH+2][SE]   Ez_old rows i0-1 .. i0+TH; col 3 = b0-1, 4.. = b0.., 4+32V = be
//   hx_s  [TH  ][SE]   Hx_new rows i0 .. i0+TH-1; col 3 = b0-1, 4.. = b0..
//   hy_s  [TH+1][SY]   Hy_new rows i0-1 .. i0+TH-1; col 0.. = b0..        (SY = 32V)
// ---------------------------------------------------------------------------
__host__ __device__ inline size_t tile_fwd_smem(int TH, int V) {
    return sizeof(float) * ((size_t)(2 * TH + 2) * (32 * V + 8) + (size_t)(TH + 1) * 32 * V);
}

template <int V>
__global__ void __launch_bounds__(512, 2) k_forward_tile(const GridDev g, const int t, const int G) {
    extern __shared__ __align__(16) float sm[];
    const int TH = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const TileT T = tile_t(g, V);
    const int SE = 32 * V + 8, SY = 32 * V;
    float* ez_s = sm;
    float* hx_s = ez_s + (TH + 2) * SE;
    float* hy_s = hx_s + TH * SE;
    const int ny = g.ny, P = g.P;
    const int rp = t & 1, wp = rp ^ 1;
    const int i = T.i0 + ty;
    const bool row_ok = i < T.i1;
    const int rows = T.i1 - T.i0;
    const int cs = lane * V;          // column of this thread's first cell within the band
    const int jb = T.b0 + cs;
    const bool act = jb < P;
    const bool core = core_warp(g, i, T.b0, T.be);
    const long long hplane = (long long)g.nx * g.Ph;
    const int sc0 = g.src_off[blockIdx.x], se = g.src_off[blockIdx.x + 1];
    const int rc0 = g.rx_off[blockIdx.x], re = g.rx_off[blockIdx.x + 1];

    float ca[V], cb[V], ch[V];
#pragma unroll
    for (int v = 0; v < V; ++v) { ca[v] = 0.f; cb[v] = 0.f; ch[v] = 0.f; }
    const long long io = (long long)i * P + jb;   // this thread's cell offset within a plane
    if (row_ok && act) {
        ld_coef<V>(g, ca, g.ca + io);
        ld_coef<V>(g, cb, g.cb + io);
        ld_coef<V>(g, ch, g.ch + io);
    }
    float* er_s = ez_s + (1 + ty) * SE + 4;      // this warp's row of Ez_old, own cells
    float* hxr_s = hx_s + ty * SE + 4;

    for (int q = 0; q < G; ++q) {
        const int s = T.grp * G + q;
        if (s >= g.S) break;
        const long long so = (long long)s * g.plane;
        const PsiShot rd = psi_shot(g, rp, s), wr = psi_shot(g, wp, s);
        // ---- stage Ez_old (tile + halo) and the old H values this thread updates
        float hx[V], hy[V], ezo[V];
#pragma unroll
        for (int v = 0; v < V; ++v) { hx[v] = 0.f; hy[v] = 0.f; ezo[v] = 0.f; }
        if (row_ok) {
            if (act) {
                ld_state<V>(g, ezo, g.ez[rp] + so + io);
                ld_state<V>(g, hx, g.hx[rp] + so + io);
                ld_state<V>(g, hy, g.hy[rp] + so + io);
            }
            sts_v<V>(er_s + cs, ezo);
            if (lane == 0) er_s[-1] = T.b0 > 0 ? ld1(g, g.ez[rp] + so + io - 1) : 0.f;
            if (lane == 31) er_s[32 * V] = T.be < P ? ld1(g, g.ez[rp] + so + io + V) : 0.f;
        }
        if (ty == 0) {
            // row above the tile (for the halo Hy) and row below (Ez[i1], the frame when i1 == nx)
            float a[V], b[V];
#pragma unroll
            for (int v = 0; v < V; ++v) { a[v] = 0.f; b[v] = 0.f; }
            if (act && T.i0 >= 1) ld_state<V>(g, a, g.ez[rp] + so + io - P);
            if (act) ld_state<V>(g, b, g.ez[rp] + so + io + (long long)rows * P);
            sts_v<V>(ez_s + 4 + cs, a);
            sts_v<V>(ez_s + (rows + 1) * SE + 4 + cs, b);
        }
        __syncthreads();
        // ---- H of the tile, the halo column b0-1 (Hx) and the halo row i0-1 (Hy)
        if (row_ok) {
            float e0[V], e1[V];
            lds_v<V>(e0, er_s + cs);
            lds_v<V>(e1, er_s + SE + cs);
            const float eR = er_s[cs + V];
            if (core) {
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const float right = (v + 1 < V) ? e0[(v + 1) % V] : eR;
                    hx[v] = __fsub_rn(hx[v], __fmul_rn(ch[v], __fsub_rn(right, e0[v])));
                    hy[v] = __fadd_rn(hy[v], __fmul_rn(ch[v], __fsub_rn(e1[v], e0[v])));
                }
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const int j = jb + v;
                    const float right = (v + 1 < V) ? e0[(v + 1) % V] : eR;
                    if (j < ny)
                        h_update<true, true, true>(g, i, j, hx[v], hy[v], __fsub_rn(right, e0[v]),
                                                   __fsub_rn(e1[v], e0[v]), ch[v], rd, wr);
                }
            }
            sts_v<V>(hxr_s + cs, hx);
            sts_v<V>(hy_s + (1 + ty) * SY + cs, hy);
            if (lane == 0) {
                float hl = 0.f, hy_unused = 0.f;
                if (T.b0 > 0) {
                    const int j = T.b0 - 1;
                    hl = ld1(g, g.hx[rp] + so + io - 1);
                    h_update<false, true, false>(g, i, j, hl, hy_unused, __fsub_rn(e0[0], er_s[-1]), 0.f,
                                                 ldc1(g, g.ch + io - 1), rd, rd);
                }
                hxr_s[-1] = hl;
            }
        }
        if (ty == 0) {
            const int ih = T.i0 - 1;
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int j = jb + v, c = cs + v;
                float h = 0.f, hx_unused = 0.f;
                if (ih >= 0 && j < ny) {
                    h = ld1(g, g.hy[rp] + so + io - P + v);
                    h_update<false, false, true>(g, ih, j, hx_unused, h, 0.f,
                                                 __fsub_rn(ez_s[SE + 4 + c], ez_s[4 + c]), ldc1(g, g.ch + io - P + v),
                                                 rd, rd);
                }
                hy_s[c] = h;
            }
        }
        __syncthreads();
        // ---- E of the tile, sources, stores, history, receivers
        if (row_ok) {
            float hyu[V], hxl[V];
            lds_v<V>(hyu, hy_s + ty * SY + cs);
            hxl[0] = hxr_s[cs - 1];
#pragma unroll
            for (int v = 1; v < V; ++v) hxl[v] = hx[v - 1];
            float ezw[V];
            if (core) {
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const float dhy = __fsub_rn(hy[v], hyu[v]);
                    const float dhx = __fsub_rn(hx[v], hxl[v]);
                    ezw[v] = __fmaf_rn(-cb[v], dhx, madd2(ca[v], ezo[v], cb[v], dhy));
                }
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const int j = jb + v;
                    ezw[v] = ezo[v];
                    if (j < ny)
                        ezw[v] = e_update<true>(g, i, j, ezo[v], __fsub_rn(hy[v], hyu[v]), __fsub_rn(hx[v], hxl[v]),
                                                ca[v], cb[v], rd, wr);
                }
            }
            for (int k = sc0; k < se; ++k) {
                const Ev e = __ldg(g.src_ev + k);
                if (e.x != i || e.y != q) continue;
#pragma unroll
                for (int v = 0; v < V; ++v)
                    if (jb + v == e.z) {
                        const float cd = ldc1(g, g.cd + io + v);
                        ezw[v] = __fmaf_rn(-cd, __ldg(g.srcw + (long long)e.w * g.nt + t), ezw[v]);
                    }
            }
            if (act) {
                st_state<V>(g, g.ez[wp] + so + io, ezw);
                st_state<V>(g, g.hx[wp] + so + io, hx);
                st_state<V>(g, g.hy[wp] + so + io, hy);
            }
            if (g.hist && jb < g.Ph)
                st_state<V>(g, g.hist + ((long long)t * g.S + s) * hplane + (long long)i * g.Ph + jb, ezw);
            if (t + 1 < g.nt) {
                for (int k = rc0; k < re; ++k) {
                    const Ev e = __ldg(g.rx_ev + k);
                    if (e.x != i || e.y != q) continue;
#pragma unroll
                    for (int v = 0; v < V; ++v)
                        if (jb + v == e.z) g.traces[((long long)s * g.nt + t + 1) * g.nrx + e.w] = ezw[v];
                }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Reference-mode adjoint step.  Shared memory (floats), own cells at offset 4:
//   hy_s  [TH+2][SE]   Hy_old rows i0-1 .. i1; col 4.. = b0.., 4+32V = be
//   hx_s  [TH+1][SE]   Hx_old rows i0 .. i1;   col 3 = b0-1, 4.. = b0.., 4+32V = be
//   en_s  [TH+1][SE]   E_new  rows i0 .. i1;   col 4.. = b0.., 4+32V = be
// ---------------------------------------------------------------------------
__host__ __device__ inline size_t tile_adj_smem(int TH, int V) {
    return sizeof(float) * ((size_t)(3 * TH + 4) * (32 * V + 8));
}

// Adjoint E of cell (r, j) of shot s (with the residuals injected there, in
// list order) from the staged old H values; STORE writes the auxiliaries.
template <bool STORE>
__device__ __forceinline__ float adj_e_tile(const GridDev& g, int r, int j, int q, float ez, float hy_c, float hy_u,
                                            float hx_c, float hx_l, float ca, float cb, const Ev* ev, int k0, int k1,
                                            const float* resid_s, const PsiShot& rd, const PsiShot& wr) {
    for (int k = k0; k < k1; ++k) {
        const Ev e = __ldg(ev + k);
        if (e.x == r && e.y == q && e.z == j) ez = __fsub_rn(ez, resid_s[e.w]);
    }
    return e_update<STORE>(g, r, j, ez, __fsub_rn(hy_c, hy_u), __fsub_rn(hx_c, hx_l), ca, cb, rd, wr);
}

template <int V>
__global__ void __launch_bounds__(512, 2) k_adjoint_tile(const GridDev g, const int it, const int rp, const int G) {
    extern __shared__ __align__(16) float sm[];
    const int TH = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const TileT T = tile_t(g, V);
    const int SE = 32 * V + 8;
    float* hy_s = sm;
    float* hx_s = hy_s + (TH + 2) * SE;
    float* en_s = hx_s + (TH + 1) * SE;
    const int nx = g.nx, ny = g.ny, P = g.P;
    const int wp = rp ^ 1;
    const int i = T.i0 + ty;
    const bool row_ok = i < T.i1;
    const int rows = T.i1 - T.i0;
    const bool last_row = ty == rows - 1;
    const int cs = lane * V;
    const int jb = T.b0 + cs;
    const bool act = jb < P;
    const int i1 = T.i1, be = T.be;
    const long long hplane = (long long)nx * g.Ph;
    const int ic0 = g.inj_off[blockIdx.x], ie = g.inj_off[blockIdx.x + 1];
    const int hc0 = g.injh_off[blockIdx.x], he = g.injh_off[blockIdx.x + 1];
    const bool core = core_warp(g, i, T.b0, T.be) && ic0 == ie;
    const long long io = (long long)i * P + jb;
    float* hyr_s = hy_s + (1 + ty) * SE + 4;     // Hy_old of row i, own cells
    float* hxr_s = hx_s + ty * SE + 4;           // Hx_old of row i
    float* enr_s = en_s + ty * SE + 4;           // E_new of row i

    float ca[V], cb[V], ch[V];
#pragma unroll
    for (int v = 0; v < V; ++v) { ca[v] = 0.f; cb[v] = 0.f; ch[v] = 0.f; }
    if (row_ok && act) {
        ld_coef<V>(g, ca, g.ca + io);
        ld_coef<V>(g, cb, g.cb + io);
        ld_coef<V>(g, ch, g.ch + io);
    }
    float acc_e[V], acc_s[V];
#pragma unroll
    for (int v = 0; v < V; ++v) { acc_e[v] = 0.f; acc_s[v] = 0.f; }

    for (int q = 0; q < G; ++q) {
        const int s = T.grp * G + q;
        if (s >= g.S) break;
        const long long so = (long long)s * g.plane;
        const PsiShot rd = psi_shot(g, rp, s), wr = psi_shot(g, wp, s);
        const float* resid_s = g.resid + ((long long)s * g.nt + it) * g.nrx;
        // ---- stage old H (tile + halo) and this thread's old Ez
        float ezo[V], hxo[V], hyo[V];
#pragma unroll
        for (int v = 0; v < V; ++v) { ezo[v] = 0.f; hxo[v] = 0.f; hyo[v] = 0.f; }
        if (row_ok) {
            if (act) {
                ld_state<V>(g, ezo, g.ez[rp] + so + io);
                ld_state<V>(g, hxo, g.hx[rp] + so + io);
                ld_state<V>(g, hyo, g.hy[rp] + so + io);
            }
            sts_v<V>(hyr_s + cs, hyo);
            sts_v<V>(hxr_s + cs, hxo);
            if (lane == 0) hxr_s[-1] = T.b0 > 0 ? ld1(g, g.hx[rp] + so + io - 1) : 0.f;
            if (lane == 31) {
                hxr_s[32 * V] = be < P ? ld1(g, g.hx[rp] + so + io + V) : 0.f;
                hyr_s[32 * V] = be < P ? ld1(g, g.hy[rp] + so + io + V) : 0.f;
            }
        }
        if (ty == 0) {
            // Hy row i0-1 (columns b0 .. be); Hx and Hy of the halo row i1
            float a[V], bx[V], by[V];
#pragma unroll
            for (int v = 0; v < V; ++v) { a[v] = 0.f; bx[v] = 0.f; by[v] = 0.f; }
            if (act && T.i0 >= 1) ld_state<V>(g, a, g.hy[rp] + so + io - P);
            if (act && i1 < nx) {
                ld_state<V>(g, bx, g.hx[rp] + so + io + (long long)rows * P);
                ld_state<V>(g, by, g.hy[rp] + so + io + (long long)rows * P);
            }
            sts_v<V>(hy_s + 4 + cs, a);
            sts_v<V>(hx_s + rows * SE + 4 + cs, bx);
            sts_v<V>(hy_s + (rows + 1) * SE + 4 + cs, by);
            if (lane == 0) {
                hy_s[4 + 32 * V] = (T.i0 >= 1 && be < P) ? ld1(g, g.hy[rp] + so + io - P + 32 * V) : 0.f;
                hx_s[rows * SE + 3] = (T.b0 > 0 && i1 < nx) ? ld1(g, g.hx[rp] + so + io + (long long)rows * P - 1) : 0.f;
            }
        }
        __syncthreads();
        // ---- E_new of the tile, of the halo row i1 and of the halo column be
        if (row_ok) {
            float hu[V], hl[V], e[V];
            lds_v<V>(hu, hyr_s - SE + cs);
            hl[0] = hxr_s[cs - 1];
#pragma unroll
            for (int v = 1; v < V; ++v) hl[v] = hxo[v - 1];
            if (core) {
#pragma unroll
                for (int v = 0; v < V; ++v)
                    e[v] = __fmaf_rn(-cb[v], __fsub_rn(hxo[v], hl[v]),
                                     madd2(ca[v], ezo[v], cb[v], __fsub_rn(hyo[v], hu[v])));
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const int j = jb + v;
                    e[v] = ezo[v];
                    if (j < ny)
                        e[v] = adj_e_tile<true>(g, i, j, q, ezo[v], hyo[v], hu[v], hxo[v], hl[v], ca[v], cb[v],
                                                g.inj_ev, ic0, ie, resid_s, rd, wr);
                }
            }
            sts_v<V>(enr_s + cs, e);
            if (lane == 31) {
                float eh = 0.f;
                if (be < ny) {
                    const long long c = io + V;
                    const float ez = ld1(g, g.ez[rp] + so + c);
                    eh = adj_e_tile<false>(g, i, be, q, ez, hyr_s[32 * V], hyr_s[32 * V - SE], hxr_s[32 * V],
                                           hxr_s[32 * V - 1], ldc1(g, g.ca + c), ldc1(g, g.cb + c), g.injh_ev, hc0, he,
                                           resid_s, rd, rd);
                }
                enr_s[32 * V] = eh;
            }
        }
        if (last_row) {
            const float* hyb = hy_s + (rows + 1) * SE + 4;   // Hy_old row i1
            const float* hxb = hx_s + rows * SE + 4;         // Hx_old row i1
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int j = jb + v, c = cs + v;
                float eb = 0.f;
                if (i1 < nx && j < ny) {
                    const long long o = io + (long long)P + v;   // (i1, j): the row after this warp's
                    const float ez = ld1(g, g.ez[rp] + so + o);
                    eb = adj_e_tile<false>(g, i1, j, q, ez, hyb[c], hyb[c - SE], hxb[c], hxb[c - 1],
                                           ldc1(g, g.ca + o), ldc1(g, g.cb + o), g.inj_ev, ic0, ie, resid_s, rd, rd);
                }
                en_s[rows * SE + 4 + c] = eb;
            }
        }
        __syncthreads();
        // ---- H of the tile, imaging, stores
        if (row_ok) {
            float e0[V], e1[V], f1[V], f0[V];
            lds_v<V>(e0, enr_s + cs);
            lds_v<V>(e1, enr_s + SE + cs);
            const float eR = enr_s[cs + V];
#pragma unroll
            for (int v = 0; v < V; ++v) { f1[v] = 0.f; f0[v] = 0.f; }
            if (jb < g.Ph) {
                const float* h1 = g.hist + (((long long)it * g.S + s) * nx + i) * g.Ph + jb;
                ld_state<V>(g, f1, h1);
                ld_state<V>(g, f0, h1 - (long long)g.S * hplane);
            }
            if (core) {
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const float right = (v + 1 < V) ? e0[(v + 1) % V] : eR;
                    hxo[v] = __fsub_rn(hxo[v], __fmul_rn(ch[v], __fsub_rn(right, e0[v])));
                    hyo[v] = __fadd_rn(hyo[v], __fmul_rn(ch[v], __fsub_rn(e1[v], e0[v])));
                    acc_e[v] = __fadd_rn(acc_e[v], __fmul_rn(__fsub_rn(f1[v], f0[v]), e0[v]));
                    acc_s[v] = __fadd_rn(acc_s[v], __fmul_rn(__fmul_rn(f1[v], e0[v]), g.dt));
                }
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const int j = jb + v;
                    const float right = (v + 1 < V) ? e0[(v + 1) % V] : eR;
                    if (j < ny) {
                        h_update<true, true, true>(g, i, j, hxo[v], hyo[v], __fsub_rn(right, e0[v]),
                                                   __fsub_rn(e1[v], e0[v]), ch[v], rd, wr);
                        acc_e[v] = __fadd_rn(acc_e[v], __fmul_rn(__fsub_rn(f1[v], f0[v]), e0[v]));
                        acc_s[v] = __fadd_rn(acc_s[v], __fmul_rn(__fmul_rn(f1[v], e0[v]), g.dt));
                    }
                }
            }
            if (act) {
                st_state<V>(g, g.ez[wp] + so + io, e0);
                st_state<V>(g, g.hx[wp] + so + io, hxo);
                st_state<V>(g, g.hy[wp] + so + io, hyo);
            }
        }
        __syncthreads();
    }
    if (row_ok) {
        double* gae = g.gacc + (long long)T.grp * 2 * ((long long)nx * ny);
        double* gas = gae + (long long)nx * ny;
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

}  // namespace fg
