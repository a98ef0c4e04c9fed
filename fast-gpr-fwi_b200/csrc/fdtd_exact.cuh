// Exact discrete adjoint of the forward step (adjoint = "exact").  The
// reference has no counterpart: its gradient (src/compute.py:1020-1180)
// re-runs the forward operator in reverse time with other coefficients.
//
// The forward step maps the state x_t = (Ez, Hx, Hy, CPML auxiliaries) to
// x_{t+1} = E(H(x_t)) + source, where H is the H leapfrog plus the H-slab
// CPML corrections (fields_updates_gpu.cu:47-78, pml_updates_h.cu) and E the
// E leapfrog plus the E-slab corrections (fields_updates_gpu.cu:8-33,
// pml_updates_e.cu); both are linear in the state.  The traces read Ez of x_t
// at the receivers.  For J = sum w * traces the adjoint state runs
//   lambda_{nt-1} = R^T w_{nt-1},   lambda_{t-1} = H^T E^T lambda_t + R^T w_{t-1},
// and one launch of k_adj_exact applies H^T E^T to every cell: with the
// adjoint state after the step (parity rp) it forms the adjoints of the E
// phase's differences (dHy, dHx) of the cell and its four neighbours, the H
// adjoint between the phases, the adjoints of the H phase's differences
// (dEz) and from them the adjoint state before the step (parity rp ^ 1), so
// every cell reads the old state only (ping-pong, like the forward).
//
// Imaging: the model enters step t-1 only through the E coefficients of
// x_t's Ez (uE0 = EB/EA, uE1 = uE4/dx, uE4 = 1/EA), so the gradient needs the
// per-cell sums s1 = sum_t sum_s lambda_t Ez(x_{t-1}) and s2 = sum_t sum_s
// lambda_t Ez(x_t) (k_grad_exact turns them into dJ/d eps_r and dJ/d sigma).
// They are accumulated in fp64, one addition per cell and launch.
#pragma once

#include "fdtd_common.cuh"

namespace fg {

// Adjoint state of one shot group and parity: fields and auxiliaries.
template <int CS>
struct ExactView {
    const Dev& g;
    const float *ez, *hx, *hy, *ex, *ey, *hxp, *hyp;   // old (after the step)
    const float* R;                                    // CPML profile (8 x th)
    int l;
    __device__ __forceinline__ long long cell(int i, int j) const { return ((long long)i * g.P + j + PADC) * CS + l; }
    __device__ __forceinline__ long long coef(int i, int j) const { return (long long)i * g.P + j + PADC; }
    // E-slab rows / columns: x0 i in [1, th] (row th-i), xmax i >= nx-th (row th + i-(nx-th));
    // y0 j in [1, th] (column th-j), ymax j >= ny-th (column j-(ny-th), rows nx+1+i)
    // adjoint of dHy = Hy[a][b] - Hy[a-1][b] in the E update of cell (a, b)
    __device__ __forceinline__ float dhy(int a, int b) const {
        if (a < 0 || a >= g.nx || b < 0 || b >= g.ny) return 0.f;
        const float e = ldro(g, ez + cell(a, b));
        float v = (a >= 1 && b >= 1) ? __fmul_rn(ldro(g, g.cb + coef(a, b)), e) : 0.f;
        const int th = g.th;
        if (th > 0) {
            const float u4 = ldro(g, g.cd + coef(a, b));
            if (a >= 1 && a <= th) {
                const int k = th - a;
                const float p = ldro(g, ex + ((long long)k * g.P + b) * CS + l);
                v = __fadd_rn(v, __fdiv_rn(__fmaf_rn(__fmul_rn(u4, __fsub_rn(R[k], 1.f)), e, -__fmul_rn(R[3 * th + k], p)), g.d));
            }
            if (a >= g.nx - th) {
                const int k = a - (g.nx - th);
                const float p = ldro(g, ex + ((long long)(th + k) * g.P + b) * CS + l);
                v = __fadd_rn(v, __fdiv_rn(__fmaf_rn(__fmul_rn(u4, __fsub_rn(R[k], 1.f)), e, -__fmul_rn(R[3 * th + k], p)), g.d));
            }
        }
        return v;
    }
    // adjoint of dHx = Hx[a][b] - Hx[a][b-1] in the E update of cell (a, b)
    __device__ __forceinline__ float dhx(int a, int b) const {
        if (a < 0 || a >= g.nx || b < 0 || b >= g.ny) return 0.f;
        const float e = ldro(g, ez + cell(a, b));
        float v = (a >= 1 && b >= 1) ? -__fmul_rn(ldro(g, g.cb + coef(a, b)), e) : 0.f;
        const int th = g.th;
        if (th > 0) {
            const float u4 = ldro(g, g.cd + coef(a, b));
            if (b >= 1 && b <= th) {
                const int k = th - b;
                const float p = ldro(g, ey + ((long long)a * g.TY + k) * CS + l);
                v = __fadd_rn(v, __fdiv_rn(__fmaf_rn(-__fmul_rn(u4, __fsub_rn(R[k], 1.f)), e, -__fmul_rn(R[3 * th + k], p)), g.d));
            }
            if (b >= g.ny - th) {
                const int k = b - (g.ny - th);
                const float p = ldro(g, ey + ((long long)(g.nx + 1 + a) * g.TY + k) * CS + l);
                v = __fadd_rn(v, __fdiv_rn(__fmaf_rn(-__fmul_rn(u4, __fsub_rn(R[k], 1.f)), e, -__fmul_rn(R[3 * th + k], p)), g.d));
            }
        }
        return v;
    }
    // H adjoint between the phases (after E^T, before H^T)
    __device__ __forceinline__ float hx_mid(int a, int b) const {
        return __fsub_rn(__fadd_rn(ldro(g, hx + cell(a, b)), dhx(a, b)), dhx(a, b + 1));
    }
    __device__ __forceinline__ float hy_mid(int a, int b) const {
        return __fsub_rn(__fadd_rn(ldro(g, hy + cell(a, b)), dhy(a, b)), dhy(a + 1, b));
    }
    // H-slab rows: x0 i <= th-1 (row th-1-i), xmax i >= nx-th; y0 j <= th-1, ymax j >= ny-th.
    // adjoint of dEz = Ez[a][b+1] - Ez[a][b] in the Hx update of cell (a, b), given its H adjoint hb
    __device__ __forceinline__ float dzx(int a, int b, float hb) const {
        float v = a >= 1 ? -__fmul_rn(ldro(g, g.ch + coef(a, b)), hb) : 0.f;
        const int th = g.th;
        if (th > 0) {
            const float* HR = R + 4 * th;
            const float u4 = ldro(g, g.ci + coef(a, b));
            if (b <= th - 1) {
                const int k = th - 1 - b;
                const float p = ldro(g, hyp + ((long long)a * g.TY + k) * CS + l);
                v = __fadd_rn(v, __fdiv_rn(__fmaf_rn(-__fmul_rn(u4, __fsub_rn(HR[k], 1.f)), hb, -__fmul_rn(HR[3 * th + k], p)), g.d));
            }
            if (b >= g.ny - th) {
                const int k = b - (g.ny - th);
                const float p = ldro(g, hyp + ((long long)(g.nx + 1 + a) * g.TY + k) * CS + l);
                v = __fadd_rn(v, __fdiv_rn(__fmaf_rn(-__fmul_rn(u4, __fsub_rn(HR[k], 1.f)), hb, -__fmul_rn(HR[3 * th + k], p)), g.d));
            }
        }
        return v;
    }
    // adjoint of dEz = Ez[a+1][b] - Ez[a][b] in the Hy update of cell (a, b)
    __device__ __forceinline__ float dzy(int a, int b, float hb) const {
        float v = b >= 1 ? __fmul_rn(ldro(g, g.ch + coef(a, b)), hb) : 0.f;
        const int th = g.th;
        if (th > 0) {
            const float* HR = R + 4 * th;
            const float u4 = ldro(g, g.ci + coef(a, b));
            if (a <= th - 1) {
                const int k = th - 1 - a;
                const float p = ldro(g, hxp + ((long long)k * g.P + b) * CS + l);
                v = __fadd_rn(v, __fdiv_rn(__fmaf_rn(__fmul_rn(u4, __fsub_rn(HR[k], 1.f)), hb, -__fmul_rn(HR[3 * th + k], p)), g.d));
            }
            if (a >= g.nx - th) {
                const int k = a - (g.nx - th);
                const float p = ldro(g, hxp + ((long long)(th + k) * g.P + b) * CS + l);
                v = __fadd_rn(v, __fdiv_rn(__fmaf_rn(__fmul_rn(u4, __fsub_rn(HR[k], 1.f)), hb, -__fmul_rn(HR[3 * th + k], p)), g.d));
            }
        }
        return v;
    }
};

// One adjoint iteration it (lambda_it -> H^T E^T lambda_it) for every cell and
// shot slot, plus the imaging sums of lambda_it.  One thread per (group, cell,
// slot), slot fastest.
//
// proj: row 0 (Ez, Hx and the y-slab auxiliaries of the row) and column 0
// (Ez, Hy and the x-slab auxiliaries of the column) are closed subsystems of
// the forward step -- updated only by the CPML terms of their own cells, they
// feed the rest of the grid without being fed by it -- so with no source on
// them they stay exactly zero in the forward and no functional depends on
// them.  Their transposed dynamics (an unstable CPML-only recursion that the
// rest of the grid drives in the adjoint) would overflow in FP32 after a few
// hundred steps; with proj set their adjoint is held at zero, which leaves
// the gradient unchanged.
template <int CS>
__global__ void __launch_bounds__(256) k_adj_exact(const Dev g, const int it, const int rp, const int proj) {
    extern __shared__ __align__(16) float Rs[];
    for (int k = threadIdx.x; k < 8 * g.th; k += blockDim.x) Rs[k] = __ldg(g.pml + k);
    __syncthreads();
    const long long n = (long long)g.ngroups * g.nx * g.ny * CS;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    // every lane of a shot-lane warp takes part in the imaging shuffles
    const bool in = idx < n;
    const long long q = in ? idx : n - 1;
    const int l = (int)(q % CS);
    long long rest = q / CS;
    const int j = (int)(rest % g.ny);
    rest /= g.ny;
    const int i = (int)(rest % g.nx);
    const int grp = (int)(rest / g.nx);
    const int wp = rp ^ 1;
    const long long go = (long long)grp * g.plane;
    const PsiG rd = psi_group(g, rp, grp), wr = psi_group(g, wp, grp);
    ExactView<CS> V{g, g.ez[rp] + go, g.hx[rp] + go, g.hy[rp] + go, rd.ex, rd.ey, rd.hx, rd.hy, Rs, l};
    const long long c = V.cell(i, j);
    const float lam = ldro(g, V.ez + c);
    // imaging: lambda_it with Ez(x_it) = hist[it-1] and Ez(x_{it-1}) = hist[it-2]
    {
        const long long hrow = (long long)g.Ph * CS;
        const long long hs = (long long)g.ngroups * g.nx * hrow;
        const float* h1 = g.hist + (long long)(it - 1 - g.hist_t0) * hs + ((long long)grp * g.nx + i) * hrow +
                          (long long)j * CS + l;
        const double x1 = (double)ldro(g, h1);
        const double x0 = it >= 2 ? (double)ldro(g, h1 - hs) : 0.0;
        double a = in ? (double)lam * x0 : 0.0, b = in ? (double)lam * x1 : 0.0;
        if (CS == 32) {
#pragma unroll
            for (int m = 16; m >= 1; m >>= 1) {
                a += __shfl_xor_sync(FULL, a, m);
                b += __shfl_xor_sync(FULL, b, m);
            }
        }
        if (in && (CS == 1 || l == 0)) {
            double* s1 = g.gacc + (long long)grp * 2 * ((long long)g.nx * g.ny) + (long long)i * g.ny + j;
            acc_add(g, s1, a);
            acc_add(g, s1 + (long long)g.nx * g.ny, b);
        }
    }
    if (!in) return;
    const int th = g.th, nx = g.nx, ny = g.ny;
    // H adjoints of this cell between the phases (the new Hx / Hy adjoints)
    const float hxm = V.hx_mid(i, j), hym = V.hy_mid(i, j);
    // Ez: E^T (coefficient uE0 on leapfrog cells, 1 on the others), then H^T
    float e = (i >= 1 && j >= 1) ? __fmul_rn(ldro(g, g.ca + V.coef(i, j)), lam) : lam;
    e = __fsub_rn(e, V.dzx(i, j, hxm));
    e = __fsub_rn(e, V.dzy(i, j, hym));
    if (j >= 1) e = __fadd_rn(e, V.dzx(i, j - 1, V.hx_mid(i, j - 1)));
    if (i >= 1) e = __fadd_rn(e, V.dzy(i - 1, j, V.hy_mid(i - 1, j)));
    const bool row0 = proj && i == 0, col0 = proj && j == 0;
    st1(g, g.ez[wp] + go + c, (row0 || col0) ? 0.f : e);
    st1(g, g.hx[wp] + go + c, row0 ? 0.f : hxm);
    st1(g, g.hy[wp] + go + c, col0 ? 0.f : hym);
    if (th <= 0) return;
    // auxiliaries: psi' = RE psi - RF D gives psi_bar = RE psi_bar' + (coefficient of psi in the field update) F_bar'
    const float u4 = ldro(g, g.cd + V.coef(i, j)), h4 = ldro(g, g.ci + V.coef(i, j));
    const float* HR = Rs + 4 * th;
    // x-slab auxiliaries of column 0 and y-slab auxiliaries of row 0 are held
    // at zero with proj (see above)
    auto upd = [&](const float* src, float* dst, long long o, float re, float coefb) {
        const bool zero = (src == rd.ex || src == rd.hx) ? col0 : row0;
        st1(g, dst + o, zero ? 0.f : __fmaf_rn(re, ldro(g, src + o), coefb));
    };
    if (i >= 1 && i <= th) {   // E x0
        const int k = th - i;
        upd(rd.ex, wr.ex, ((long long)k * g.P + j) * CS + l, Rs[2 * th + k], __fmul_rn(__fmul_rn(u4, Rs[th + k]), lam));
    }
    if (i >= nx - th) {        // E xmax
        const int k = i - (nx - th);
        upd(rd.ex, wr.ex, ((long long)(th + k) * g.P + j) * CS + l, Rs[2 * th + k],
            __fmul_rn(__fmul_rn(u4, Rs[th + k]), lam));
    }
    if (j >= 1 && j <= th) {   // E y0
        const int k = th - j;
        upd(rd.ey, wr.ey, ((long long)i * g.TY + k) * CS + l, Rs[2 * th + k], -__fmul_rn(__fmul_rn(u4, Rs[th + k]), lam));
    }
    if (j >= ny - th) {        // E ymax
        const int k = j - (ny - th);
        upd(rd.ey, wr.ey, ((long long)(nx + 1 + i) * g.TY + k) * CS + l, Rs[2 * th + k],
            -__fmul_rn(__fmul_rn(u4, Rs[th + k]), lam));
    }
    if (i <= th - 1) {         // H x0 (Hy)
        const int k = th - 1 - i;
        upd(rd.hx, wr.hx, ((long long)k * g.P + j) * CS + l, HR[2 * th + k], __fmul_rn(__fmul_rn(h4, HR[th + k]), hym));
    }
    if (i >= nx - th) {        // H xmax (Hy)
        const int k = i - (nx - th);
        upd(rd.hx, wr.hx, ((long long)(th + k) * g.P + j) * CS + l, HR[2 * th + k],
            __fmul_rn(__fmul_rn(h4, HR[th + k]), hym));
    }
    if (j <= th - 1) {         // H y0 (Hx)
        const int k = th - 1 - j;
        upd(rd.hy, wr.hy, ((long long)i * g.TY + k) * CS + l, HR[2 * th + k], -__fmul_rn(__fmul_rn(h4, HR[th + k]), hxm));
    }
    if (j >= ny - th) {        // H ymax (Hx)
        const int k = j - (ny - th);
        upd(rd.hy, wr.hy, ((long long)(nx + 1 + i) * g.TY + k) * CS + l, HR[2 * th + k],
            -__fmul_rn(__fmul_rn(h4, HR[th + k]), hxm));
    }
}

// lambda_t += R^T w_t at the receivers of every shot (parity par), in receiver
// order; one thread per shot.  rxpos: (S, nrx) (i, j), i < 0 for inert ones.
template <int CS>
__global__ void k_inject_exact(const Dev g, const int2* __restrict__ rxpos, const float* __restrict__ w, const int t,
                               const int par) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.S) return;
    const int grp = s / CS, l = s % CS;
    float* ez = g.ez[par] + (long long)grp * g.plane;
    for (int r = 0; r < g.nrx; ++r) {
        const int2 p = __ldg(rxpos + (long long)s * g.nrx + r);
        if (p.x < 0) continue;
        float* a = ez + ((long long)p.x * g.P + p.y + PADC) * CS + l;
        if (!FG_OK_PTR(g, a, 4)) continue;
        *a = __fadd_rn(*a, __ldg(w + ((long long)s * g.nt + t) * g.nrx + r));
    }
}

// dJ/d eps_r and dJ/d sigma from the group-summed s1 (sums[c]) and s2
// (sums[n + c]): with a = e0/dt and EA = a er + se/2 (uc.cu:21-38),
//   d/der = (a/EA) (s1 - s2),  d/dse = -(s1 + s2) / (2 EA) on leapfrog cells
//   (i, j >= 1), -(s2 - s1) / (2 EA) on row / column 0; PEC cells (se > 100) 0.
__global__ void k_grad_exact(const double* __restrict__ sums, const float* __restrict__ er,
                             const float* __restrict__ se, int nx, int ny, double a, float* __restrict__ ge,
                             float* __restrict__ gs) {
    const long long n = (long long)nx * ny;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int i = (int)(c / ny), j = (int)(c % ny);
    const double s1 = sums[c], s2 = sums[n + c];
    const double sev = (double)se[c];
    const double EA = a * (double)er[c] + 0.5 * sev;
    double de = (a / EA) * (s1 - s2);
    double ds = (i >= 1 && j >= 1) ? -(s1 + s2) / (2.0 * EA) : -(s2 - s1) / (2.0 * EA);
    if (sev > 100.0) de = ds = 0.0;
    if (ge) ge[c] = (float)de;
    if (gs) gs[c] = (float)ds;
}

}  // namespace fg
