// Shot-pair lane march: the lane-march step kernels with two shots per lane.
//
// A group holds 64 shots (CS = 64 floats per cell, shot slot fastest); lane l
// of a warp owns slots 2l and 2l+1 of the same cells as a float2.  One warp
// access is then 256 contiguous bytes, and every per-cell cost that does not
// depend on the shot -- addresses, coefficient loads, boundary tests, loop
// control -- is paid once for two shots.  The interior arithmetic runs on the
// paired fp32 instructions of sm_100 (add/sub/fma .rn.f32x2), which round each
// element exactly as the scalar instruction does, so every cell is the scalar
// kernels' (and the reference's) value bit for bit.  One exception is kept
// out: ptxas fuses a paired multiply into a paired add or subtract that
// consumes it (one rounding instead of two) even when both carry .rn, so a
// product that feeds an add is taken as two scalar multiplies (mulbc).
//
// Rows outside the interior core (CPML slabs, the grid edges) take the
// per-cell update of fdtd_common.cuh for each of the two slots in turn.
// Tiles, scheduling and the halo recompute are those of fdtd_lanes.cuh.
#pragma once

#include "fdtd_common.cuh"
#include "fdtd_lanes.cuh"

namespace fg {

using f2 = float2;

// Paired fp32 operations as PTX with an explicit .rn rounding.
__device__ __forceinline__ f2 bc2(float s) { return make_float2(s, s); }
__device__ __forceinline__ unsigned long long as_u64(f2 a) {
    unsigned long long x;
    memcpy(&x, &a, 8);
    return x;
}
__device__ __forceinline__ f2 as_f2(unsigned long long x) {
    f2 r;
    memcpy(&r, &x, 8);
    return r;
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(as_u64(a)), "l"(as_u64(b)));
    return as_f2(d);
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(as_u64(a)), "l"(as_u64(b)));
    return as_f2(d);
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(as_u64(a)), "l"(as_u64(b)));
    return as_f2(d);
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(as_u64(a)), "l"(as_u64(b)), "l"(as_u64(c)));
    return as_f2(d);
}
// s * x rounded per element by scalar multiplies, for a product that an add
// or subtract consumes (see the file comment).
__device__ __forceinline__ f2 mulbc(float s, f2 x) { return make_float2(__fmul_rn(s, x.x), __fmul_rn(s, x.y)); }
__device__ __forceinline__ float comp(f2 v, int k) { return k ? v.y : v.x; }
__device__ __forceinline__ void set_comp(f2& v, int k, float x) {
    if (k) v.y = x;
    else v.x = x;
}
__device__ __forceinline__ f2 ld2(const Dev& g, const float* p) {
    if (!FG_OK_PTR(g, p, 8)) return make_float2(0.f, 0.f);
    return __ldg(reinterpret_cast<const float2*>(p));
}
template <bool STREAM = false>
__device__ __forceinline__ void st2(const Dev& g, float* p, f2 v) {
    if (!FG_OK_PTR(g, p, 8)) return;
    if (STREAM) __stcs(reinterpret_cast<float2*>(p), v);
    else __stcg(reinterpret_cast<float2*>(p), v);
}

template <int W>
struct FwdIn2 {                // operands of forward row i
    f2 en[W + 2];              // Ez_old(i+1, j0-1 .. j0+W)
    f2 hxo[W + 1];             // Hx_old(i, j0-1 .. j0+W-1)
    f2 hyo[W];                 // Hy_old(i, j0 .. j0+W-1)
    float ca[W], cb[W];        // uE0, uE1 (i, j0 ..)
    float ch[W + 1];           // uH1 (i, j0-1 ..)
};

template <int W>
__global__ void __launch_bounds__(128, 3) k_fwd2(const Dev g, const int t) {
    constexpr int CS = 64;
    extern __shared__ __align__(128) unsigned char smem[];
    const float* R = stage_profile(g, smem);
    if (blockIdx.x == 0 && threadIdx.x == 0) g.tile_ctr[(t + 1) & 1] = 0;   // the next launch's counter
    int* ctr = g.tile_ctr + (t & 1);
    const int lane = threadIdx.x & 31, l0 = 2 * lane;
    const int P = g.P, nx = g.nx, ny = g.ny, th = g.th, nt_ = g.ntiles;
    const int rp = t & 1, wp = rp ^ 1;
    const long long hrow = (long long)g.Ph * CS;
    int cur = fetch_tile(ctr, lane);
    int nxt = cur < nt_ ? fetch_tile(ctr, lane) : nt_;
#define FG_CELL2(i, j) (((long long)(i) * P + (j) + PADC) * CS + l0)
    while (cur < nt_) {
        const LaneTile<true> T = decode_tile<W, true>(g, __ldg(g.order + cur), lane);
        const int j0 = T.j0;
        const long long go = (long long)T.grp * g.plane;
        const float* ezR = g.ez[rp] + go;
        const float* hyR = g.hy[rp] + go;
        const float* hxR = g.hx[rp] + go;
        float* ezW = g.ez[wp] + go;
        float* hxW = g.hx[wp] + go;
        float* hyW = g.hy[wp] + go;
        const PsiG rd = psi_group(g, rp, T.grp), wr = psi_group(g, wp, T.grp);
        const bool bcore = j0 >= th + 1 && j0 + W <= ny - th;
        int sc = __ldg(g.src_off + T.id);
        const int se = __ldg(g.src_off + T.id + 1);
        int rc = __ldg(g.rx_off + T.id);
        const int re = __ldg(g.rx_off + T.id + 1);
        float* hist = g.hist ? g.hist + (((long long)(t - g.hist_t0) * g.ngroups + T.grp) * nx) * hrow +
                                   (long long)j0 * CS + l0
                             : nullptr;
        FwdIn2<W> B;
        auto load_row = [&](int i) {
            const long long crow = coef_at(g, i, j0);
            const long long oz = FG_CELL2(i + 1, j0 - 1), oh = FG_CELL2(i, j0 - 1);
#pragma unroll
            for (int k = 0; k < W + 2; ++k) B.en[k] = ld2(g, ezR + oz + k * CS);
#pragma unroll
            for (int k = 0; k <= W; ++k) B.hxo[k] = ld2(g, hxR + oh + k * CS);
#pragma unroll
            for (int w = 0; w < W; ++w) B.hyo[w] = ld2(g, hyR + oh + (w + 1) * CS);
            ld_coef<W, CALIGN<W>>(g, B.ca, g.ca + crow);
            ld_coef<W, CALIGN<W>>(g, B.cb, g.cb + crow);
            B.ch[0] = ldro(g, g.ch + crow - 1);
            ld_coef<W, CALIGN<W>>(g, B.ch + 1, g.ch + crow);
        };
        // Ez_old of row i0 (columns j0-1 .. j0+W) and the new Hy of row i0-1
        f2 ezc[W + 2], hyu[W];
        {
            const long long oz = FG_CELL2(T.i0, j0 - 1);
#pragma unroll
            for (int k = 0; k < W + 2; ++k) ezc[k] = ld2(g, ezR + oz + k * CS);
        }
        load_row(T.i0);   // goes out with the halo row's loads
#pragma unroll
        for (int w = 0; w < W; ++w) hyu[w] = make_float2(0.f, 0.f);
        if (T.i0 >= 1) {
            const int ih = T.i0 - 1;
            const long long oa = FG_CELL2(ih, j0);
            f2 ea[W];
            float cah[W];
#pragma unroll
            for (int w = 0; w < W; ++w) {
                ea[w] = ld2(g, ezR + oa + w * CS);
                hyu[w] = ld2(g, hyR + oa + w * CS);
            }
            ld_coef<W, CALIGN<W>>(g, cah, g.ch + coef_at(g, ih, j0));
            const bool hcore = (th == 0 || (ih >= th && ih <= nx - th - 1)) && j0 >= 1 && j0 + W <= ny;
            if (hcore) {
#pragma unroll
                for (int w = 0; w < W; ++w) hyu[w] = add2(hyu[w], mulbc(cah[w], sub2(ezc[w + 1], ea[w])));
            } else {
#pragma unroll
                for (int w = 0; w < W; ++w)
                    if (j0 + w < ny)
#pragma unroll
                        for (int k = 0; k < 2; ++k)
                            set_comp(hyu[w], k,
                                     hy_cell<CS, false>(g, R, ih, j0 + w, l0 + k, comp(hyu[w], k),
                                                        __fsub_rn(comp(ezc[w + 1], k), comp(ea[w], k)), cah[w], rd,
                                                        rd));
            }
        }
        const int nrow = T.i1 - T.i0;
        for (int n = 0; n < nrow; ++n) {
            const int i = T.i0 + n;
            if (n > 0) load_row(i);
            f2 hxn[W + 1], hyn[W], ezn[W];
            if (bcore && i >= th + 1 && i <= nx - th - 1) {
#pragma unroll
                for (int k = 0; k <= W; ++k) hxn[k] = sub2(B.hxo[k], mulbc(B.ch[k], sub2(ezc[k + 1], ezc[k])));
#pragma unroll
                for (int w = 0; w < W; ++w)
                    hyn[w] = add2(B.hyo[w], mulbc(B.ch[w + 1], sub2(B.en[w + 1], ezc[w + 1])));
#pragma unroll
                for (int w = 0; w < W; ++w)
                    ezn[w] = fma2(bc2(-B.cb[w]), sub2(hxn[w + 1], hxn[w]),
                                  fma2(bc2(B.ca[w]), ezc[w + 1], mul2(bc2(B.cb[w]), sub2(hyn[w], hyu[w]))));
            } else {
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const int l = l0 + k;
#pragma unroll
                    for (int q = 0; q <= W; ++q) {
                        const int j = j0 - 1 + q;
                        float h = comp(B.hxo[q], k);
                        if (j >= 0 && j < ny) {
                            const float dz = __fsub_rn(comp(ezc[q + 1], k), comp(ezc[q], k));
                            if (q == 0) h = hx_cell<CS, false>(g, R, i, j, l, h, dz, B.ch[q], rd, rd);
                            else h = hx_cell<CS, true>(g, R, i, j, l, h, dz, B.ch[q], rd, wr);
                        }
                        set_comp(hxn[q], k, h);
                    }
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        const int j = j0 + w;
                        float h = comp(B.hyo[w], k);
                        if (j < ny)
                            h = hy_cell<CS, true>(g, R, i, j, l, h, __fsub_rn(comp(B.en[w + 1], k), comp(ezc[w + 1], k)),
                                                  B.ch[w + 1], rd, wr);
                        set_comp(hyn[w], k, h);
                    }
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        const int j = j0 + w;
                        float e = comp(ezc[w + 1], k);
                        if (j < ny)
                            e = e_cell<CS, true>(g, R, i, j, l, e, __fsub_rn(comp(hyn[w], k), comp(hyu[w], k)),
                                                 __fsub_rn(comp(hxn[w + 1], k), comp(hxn[w], k)), B.ca[w], B.cb[w], rd,
                                                 wr);
                        set_comp(ezn[w], k, e);
                    }
                }
            }
            // Hertzian dipole (sourcereceiver.cu:84), in list order
            for (; sc < se; ++sc) {
                const Ev e = __ldg(g.src_ev + sc);
                if (e.x != i) break;
                if ((e.y >> 1) != lane) continue;
#pragma unroll
                for (int w = 0; w < W; ++w)
                    if (j0 + w == e.z) {
                        const float cd = ldro(g, g.cd + coef_at(g, i, e.z));
                        const int k = e.y & 1;
                        set_comp(ezn[w], k, __fmaf_rn(-cd, __ldg(g.srcw + (long long)e.w * g.nt + t), comp(ezn[w], k)));
                    }
            }
            const long long o = FG_CELL2(i, j0);
#pragma unroll
            for (int w = 0; w < W; ++w) {
                st2(g, ezW + o + w * CS, ezn[w]);
                st2(g, hxW + o + w * CS, hxn[w + 1]);
                st2(g, hyW + o + w * CS, hyn[w]);
            }
            if (hist && j0 < g.Ph) {
#pragma unroll
                for (int w = 0; w < W; ++w) st2<true>(g, hist + (long long)i * hrow + w * CS, ezn[w]);
            }
            for (; rc < re; ++rc) {
                const Ev e = __ldg(g.rx_ev + rc);
                if (e.x != i) break;
                if ((e.y >> 1) != lane || t + 1 >= g.nt) continue;
#pragma unroll
                for (int w = 0; w < W; ++w)
                    if (j0 + w == e.z && g.traces)
                        g.traces[((long long)(T.grp * 64 + e.y) * g.nt + t + 1) * g.nrx + e.w] = comp(ezn[w], e.y & 1);
            }
#pragma unroll
            for (int k = 0; k < W + 2; ++k) ezc[k] = B.en[k];
#pragma unroll
            for (int w = 0; w < W; ++w) hyu[w] = hyn[w];
        }
        cur = nxt;
        nxt = cur < nt_ ? fetch_tile(ctr, lane) : nt_;
    }
#undef FG_CELL2
}

// ---------------------------------------------------------------------------
// Reference-mode adjoint step, two shots per lane
// ---------------------------------------------------------------------------
template <int W>
struct AdjEIn2 {               // operands of the E update of row r
    f2 ez[W + 1];              // Ez_old(r, j0 .. j0+W)
    f2 hxo[W + 2];             // Hx_old(r, j0-1 .. j0+W)
    f2 hyo[W + 1];             // Hy_old(r, j0 .. j0+W)
    float ca[W + 1], cb[W + 1];
};

template <int W>
__device__ __forceinline__ void adj_e_load2(const Dev& g, AdjEIn2<W>& A, int r, int j0, int l0, const float* ezR,
                                            const float* hxR, const float* hyR) {
    constexpr int CS = 64;
    const long long rb = (long long)r * g.P + j0 + PADC;
    const long long o = rb * CS + l0;
#pragma unroll
    for (int k = 0; k <= W; ++k) {
        A.ez[k] = ld2(g, ezR + o + k * CS);
        A.hyo[k] = ld2(g, hyR + o + k * CS);
    }
#pragma unroll
    for (int k = 0; k < W + 2; ++k) A.hxo[k] = ld2(g, hxR + o + (k - 1) * CS);
    ld_coef<W + 1, CALIGN<W>>(g, A.ca, g.ca + rb);
    ld_coef<W + 1, CALIGN<W>>(g, A.cb, g.cb + rb);
}

// New E of row r, columns j0 .. j0+W (the last is the halo column), from the
// old state: residuals injected first (list order), then the E update with
// the old H (hyu = Hy_old of row r-1).  Auxiliaries of the own cells are
// stored when `own`.
template <int W>
__device__ __forceinline__ void adj_e_row2(const Dev& g, const float* R, AdjEIn2<W>& A, int r, int j0, int lane,
                                           int grp, int it, bool core, bool own, const f2 (&hyu)[W + 1],
                                           f2 (&out)[W + 1], int& ic, int ie, const PsiG& rd, const PsiG& wr) {
    constexpr int CS = 64;
    // back_source (back.cu:34): Ez -= residual, no scaling
    for (; ic < ie; ++ic) {
        const Ev e = __ldg(g.inj_ev + ic);
        if (e.x != r) break;
        if ((e.y >> 1) != lane) continue;
        const float v = inj_value(g, ((long long)(grp * 64 + e.y) * g.nt + it) * g.nrx + e.w);
#pragma unroll
        for (int k = 0; k <= W; ++k)
            if (j0 + k == e.z) set_comp(A.ez[k], e.y & 1, __fsub_rn(comp(A.ez[k], e.y & 1), v));
    }
    if (core) {
#pragma unroll
        for (int k = 0; k <= W; ++k)
            out[k] = fma2(bc2(-A.cb[k]), sub2(A.hxo[k + 1], A.hxo[k]),
                          fma2(bc2(A.ca[k]), A.ez[k], mul2(bc2(A.cb[k]), sub2(A.hyo[k], hyu[k]))));
        return;
    }
    const int ny = g.ny;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const int l = 2 * lane + c;
#pragma unroll
        for (int k = 0; k <= W; ++k) {
            const int j = j0 + k;
            float e = comp(A.ez[k], c);
            if (j < ny) {
                const float dhy = __fsub_rn(comp(A.hyo[k], c), comp(hyu[k], c));
                const float dhx = __fsub_rn(comp(A.hxo[k + 1], c), comp(A.hxo[k], c));
                if (k < W && own) e = e_cell<CS, true>(g, R, r, j, l, e, dhy, dhx, A.ca[k], A.cb[k], rd, wr);
                else e = e_cell<CS, false>(g, R, r, j, l, e, dhy, dhx, A.ca[k], A.cb[k], rd, rd);
            }
            set_comp(out[k], c, e);
        }
    }
}

template <int W>
__global__ void __launch_bounds__(128, 3) k_adj2(const Dev g, const int it, const int rp) {
    constexpr int CS = 64;
    extern __shared__ __align__(128) unsigned char smem[];
    const float* R = stage_profile(g, smem);
    if (blockIdx.x == 0 && threadIdx.x == 0) g.tile_ctr[rp ^ 1] = 0;   // the next launch's counter
    int* ctr = g.tile_ctr + rp;
    const int lane = threadIdx.x & 31, l0 = 2 * lane;
    const int P = g.P, nx = g.nx, ny = g.ny, th = g.th, nt_ = g.ntiles;
    const int wp = rp ^ 1;
    const long long hrow = (long long)g.Ph * CS;
    int cur = fetch_tile(ctr, lane);
    int nxt = cur < nt_ ? fetch_tile(ctr, lane) : nt_;
    while (cur < nt_) {
        const LaneTile<true> T = decode_tile<W, true>(g, __ldg(g.order + cur), lane);
        const int j0 = T.j0;
        const long long go = (long long)T.grp * g.plane;
        const float* ezR = g.ez[rp] + go;
        const float* hxR = g.hx[rp] + go;
        const float* hyR = g.hy[rp] + go;
        float* ezW = g.ez[wp] + go;
        float* hxW = g.hx[wp] + go;
        float* hyW = g.hy[wp] + go;
        const PsiG rd = psi_group(g, rp, T.grp), wr = psi_group(g, wp, T.grp);
        const bool bcore = j0 >= th + 1 && j0 + W <= ny - th - 1;
        int ic = __ldg(g.inj_off + T.id);
        const int ie = __ldg(g.inj_off + T.id + 1);
        const float* f1g = g.hist + ((long long)(it - g.hist_t0) * g.ngroups + T.grp) * nx * hrow + (long long)j0 * CS + l0;
        double* gae = g.gacc + (long long)T.grp * 2 * ((long long)nx * ny);
        double* gas = gae + (long long)nx * ny;
        const bool hist_ok = j0 < g.Ph;

        // new E of row i0 (own), with the old H of rows i0-1 and i0
        f2 ezc[W + 1], hxc[W + 2], hyc[W + 1], eoc[W];
        {
            f2 hyu[W + 1];
#pragma unroll
            for (int k = 0; k <= W; ++k) hyu[k] = make_float2(0.f, 0.f);
            if (T.i0 >= 1) {
                const long long o = ((long long)(T.i0 - 1) * P + j0 + PADC) * CS + l0;
#pragma unroll
                for (int k = 0; k <= W; ++k) hyu[k] = ld2(g, hyR + o + k * CS);
            }
            AdjEIn2<W> A;
            adj_e_load2<W>(g, A, T.i0, j0, l0, ezR, hxR, hyR);
#pragma unroll
            for (int w = 0; w < W; ++w) eoc[w] = A.ez[w];
            adj_e_row2<W>(g, R, A, T.i0, j0, lane, T.grp, it, bcore && T.i0 >= th + 1 && T.i0 <= nx - th - 1, true,
                          hyu, ezc, ic, ie, rd, wr);
#pragma unroll
            for (int k = 0; k < W + 2; ++k) hxc[k] = A.hxo[k];
#pragma unroll
            for (int k = 0; k <= W; ++k) hyc[k] = A.hyo[k];
        }
        const int nrow = T.i1 - T.i0;
        for (int n = 0; n < nrow; ++n) {
            const int i = T.i0 + n, r = i + 1;
            AdjEIn2<W> A;
            float ch[W];
            f2 f1[W];
            if (r < nx) adj_e_load2<W>(g, A, r, j0, l0, ezR, hxR, hyR);
            ld_coef<W, CALIGN<W>>(g, ch, g.ch + coef_at(g, i, j0));
#pragma unroll
            for (int w = 0; w < W; ++w) f1[w] = hist_ok ? ld2(g, f1g + (long long)i * hrow + w * CS) : make_float2(0.f, 0.f);
            // new E of row r (own if inside the chunk, else the halo row below)
            f2 ezr[W + 1], eor[W];
            if (r < nx) {
#pragma unroll
                for (int w = 0; w < W; ++w) eor[w] = A.ez[w];
                adj_e_row2<W>(g, R, A, r, j0, lane, T.grp, it, bcore && r >= th + 1 && r <= nx - th - 1, r < T.i1, hyc,
                              ezr, ic, ie, rd, wr);
            } else {
#pragma unroll
                for (int w = 0; w < W; ++w) eor[w] = make_float2(0.f, 0.f);
#pragma unroll
                for (int k = 0; k <= W; ++k) ezr[k] = A.hyo[k] = make_float2(0.f, 0.f);
#pragma unroll
                for (int k = 0; k < W + 2; ++k) A.hxo[k] = make_float2(0.f, 0.f);
            }
            // H of row i from the new E
            f2 hx[W], hy[W];
            if (bcore && i >= th + 1 && i <= nx - th - 1) {
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    hx[w] = sub2(hxc[w + 1], mulbc(ch[w], sub2(ezc[w + 1], ezc[w])));
                    hy[w] = add2(hyc[w], mulbc(ch[w], sub2(ezr[w], ezc[w])));
                }
            } else {
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    hx[w] = hxc[w + 1];
                    hy[w] = hyc[w];
                    const int j = j0 + w;
                    if (j < ny)
#pragma unroll
                        for (int c = 0; c < 2; ++c) {
                            set_comp(hx[w], c,
                                     hx_cell<CS, true>(g, R, i, j, l0 + c, comp(hxc[w + 1], c),
                                                       __fsub_rn(comp(ezc[w + 1], c), comp(ezc[w], c)), ch[w], rd, wr));
                            set_comp(hy[w], c,
                                     hy_cell<CS, true>(g, R, i, j, l0 + c, comp(hyc[w], c),
                                                       __fsub_rn(comp(ezr[w], c), comp(ezc[w], c)), ch[w], rd, wr));
                        }
                }
            }
            // imaging (compute.py:1167-1172), summed by parts as in k_adj: the two
            // shots of a lane first, then the lanes by a reduce-scatter
            float v[2 * W];
#pragma unroll
            for (int w = 0; w < W; ++w) {
                // products that an add consumes: scalar multiplies (see the file comment)
                const f2 d = sub2(ezc[w], eoc[w]);
                v[w] = __fadd_rn(__fmul_rn(f1[w].x, d.x), __fmul_rn(f1[w].y, d.y));
                v[W + w] = __fadd_rn(__fmul_rn(__fmul_rn(f1[w].x, ezc[w].x), g.dt),
                                     __fmul_rn(__fmul_rn(f1[w].y, ezc[w].y), g.dt));
            }
            const long long go2 = (long long)i * ny + j0;
            {
                constexpr int s = (2 * W) == 4 ? 3 : ((2 * W) == 8 ? 2 : 1);
                const float x = lane_reduce_scatter<2 * W>(v, lane);
                if ((lane & ((1 << s) - 1)) == 0) {
                    const int e = lane >> s;
                    const int w = e < W ? e : e - W;
                    if (j0 + w < ny) acc_add(g, (e < W ? gae : gas) + go2 + w, (double)x);
                }
            }
            const long long o = ((long long)i * P + j0 + PADC) * CS + l0;
#pragma unroll
            for (int w = 0; w < W; ++w) {
                st2(g, ezW + o + w * CS, ezc[w]);
                st2(g, hxW + o + w * CS, hx[w]);
                st2(g, hyW + o + w * CS, hy[w]);
            }
#pragma unroll
            for (int k = 0; k <= W; ++k) {
                ezc[k] = ezr[k];
                hyc[k] = A.hyo[k];
            }
#pragma unroll
            for (int w = 0; w < W; ++w) eoc[w] = eor[w];
#pragma unroll
            for (int k = 0; k < W + 2; ++k) hxc[k] = A.hxo[k];
        }
        cur = nxt;
        nxt = cur < nt_ ? fetch_tile(ctr, lane) : nt_;
    }
}

}  // namespace fg
