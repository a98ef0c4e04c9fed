// CPU oracle for the 2-D TMz FDTD forward solver and its reference-mode adjoint.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the shipped package links or calls this
// file; tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it
// as the checker.  It restates, loop by loop, the kernels of the reference
// Fast-GPR-FWI (paths relative to that project):
//
//   store_outputs            src/lib/sourcereceiver.cu:11-36
//   h_fields_updates_gpu     src/lib/fields_updates_gpu.cu:47-78
//   Order1_* (H slabs)       src/lib/pml_updates_h.cu:13-74, 129-193, 248-310, 363-426
//   e_fields_updates_gpu     src/lib/fields_updates_gpu.cu:8-33
//   Order1_* (E slabs)       src/lib/pml_updates_e.cu:12-77, 105-169, 223-286, 340-402
//   Update_hertzian_dipole   src/lib/sourcereceiver.cu:59-87
//   Back_source              src/lib/back.cu:8-37
//   Forward loop             src/compute.py:574-712
//   Backward loop + imaging  src/compute.py:1048-1172
//
// It also holds the exact discrete adjoint of that forward loop (the
// transpose of each time step, h_phase_T / e_phase_T below), which the
// reference does not have: its gradient (compute.py:1020-1180) re-runs the
// forward operator in reverse time instead.  The exact adjoint is checked by
// the dot-product test of one step and its transpose and by centred finite
// differences of the forward loop (tests/test_exact_adjoint.py).
//
// Only the TMz components are kept (Ez, Hx, Hy and the Ez/Hx/Hy CPML
// auxiliaries); Ex, Ey, Hz and their PHI arrays stay identically zero in the
// reference for a TMz source.  The dead k=1 plane of the reference layout is
// dropped.  Fields are stored as (S, nx+1, ny+1) so the i=nx / j=ny frame
// (zero coefficients in the reference, src/lib/uc.cu:19) reads as zero.
//
// Arithmetic is written with explicit fma() so that, compiled with
// -ffp-contract=off, the float build rounds exactly as the CUDA kernels of the
// package do (they use the same fused/unfused operation sequence).  The double
// build is the FP64 oracle of the same update equations.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// Flat description of one model with S shots.  Every array pointer refers to
// data of the selected dtype (float when dtype==0, double when dtype==1),
// except the int position tables.
typedef struct {
    int nx, ny;        // compute grid (axis 0 / axis 1 of the reference model)
    int th;            // CPML thickness in cells on each of the 4 sides (0 = none)
    int S;             // shots
    int nt;            // time steps ("iterations" in the reference)
    int nrx, nsrc;     // receivers / sources per shot
    int dtype;         // 0 = float, 1 = double
    double d;          // cell size used by the CPML derivative (dx == dy)
    double dt;         // time step used in the sigma imaging condition
    const void *uE0, *uE1, *uE4;   // (nx*ny) forward E coefficients
    const void *uH1, *uH4;         // (nx*ny) H coefficients (uH0 == 1)
    const void *uE0a;              // (nx*ny) reference-adjoint E coefficient
    const void *pml;               // (8*th): ERA ERB ERE ERF HRA HRB HRE HRF
    const int *src;                // (S*nsrc*2) (i, j); i<0 marks an inert entry
    const void *srcw;              // (nsrc*nt) waveform already scaled by dl/(dx dy dz)
    const int *rx;                 // (S*nrx*2) (i, j); i<0 marks an inert entry
} OracleProblem;

}  // extern "C"

namespace {

template <typename T> inline T fmaT(T a, T b, T c);
template <> inline float fmaT<float>(float a, float b, float c) { return std::fmaf(a, b, c); }
template <> inline double fmaT<double>(double a, double b, double c) { return std::fma(a, b, c); }

// a*b + c*d and a*b - c*d with one of the two products fused into the add.
// The reference is compiled by nvcc with FMA contraction on (src/Makefile:19
// passes no -fmad flag), so each such expression rounds as one fma plus one
// product.  ORACLE_FUSE_SECOND selects which product is fused; the default
// fuses the first, matching the package kernels.
template <typename T> inline T madd2(T a, T b, T c, T d) {
#ifdef ORACLE_FUSE_SECOND
    return fmaT<T>(c, d, a * b);
#else
    return fmaT<T>(a, b, c * d);
#endif
}
template <typename T> inline T msub2(T a, T b, T c, T d) {
#ifdef ORACLE_FUSE_SECOND
    return fmaT<T>(-c, d, a * b);
#else
    return fmaT<T>(a, b, -(c * d));
#endif
}

template <typename T>
struct State {
    int nx, ny, th, S;
    size_t F;  // floats per shot field = (nx+1)*(ny+1)
    std::vector<T> ez, hx, hy;
    // CPML auxiliaries, one array per slab, compact shapes of the reference
    // PHI arrays (pml_updates_*.cu INDEX4D_PHI*):
    //   E x-slabs (Ez, PHI2):  (th, ny)      E y-slabs (Ez, PHI2): (nx, th)
    //   H x-slabs (Hy, PHI1):  (th, ny)      H y-slabs (Hx, PHI1): (nx, th)
    std::vector<T> pe_x0, pe_xm, pe_y0, pe_ym, ph_x0, ph_xm, ph_y0, ph_ym;
    State(int nx_, int ny_, int th_, int S_) : nx(nx_), ny(ny_), th(th_), S(S_) {
        F = (size_t)(nx + 1) * (ny + 1);
        ez.assign(F * S, T(0)); hx.assign(F * S, T(0)); hy.assign(F * S, T(0));
        size_t px = (size_t)S * th * ny, py = (size_t)S * nx * th;
        pe_x0.assign(px, T(0)); pe_xm.assign(px, T(0)); pe_y0.assign(py, T(0)); pe_ym.assign(py, T(0));
        ph_x0.assign(px, T(0)); ph_xm.assign(px, T(0)); ph_y0.assign(py, T(0)); ph_ym.assign(py, T(0));
    }
    inline size_t at(int s, int i, int j) const { return (size_t)s * F + (size_t)i * (ny + 1) + j; }
};

template <typename T>
struct Coeffs {
    const T *uE0, *uE1, *uE4, *uH1, *uH4;
    const T *ERA, *ERB, *ERE, *ERF, *HRA, *HRB, *HRE, *HRF;
    T d;
    int ny;
    inline size_t c(int i, int j) const { return (size_t)i * ny + j; }
};

// ---- H phase: h_fields_updates_gpu then Order1_{xminus,yminus,xplus,yplus} (H)
template <typename T>
void h_phase(State<T>& st, const Coeffs<T>& k) {
    const int nx = st.nx, ny = st.ny, th = st.th, S = st.S;
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s)
        for (int i = 0; i < nx; ++i) {
            for (int j = 0; j < ny; ++j) {
                const size_t a = st.at(s, i, j);
                const T u1 = k.uH1[k.c(i, j)];
                // Hx: i in [1, nx), j in [0, ny)   (fields_updates_gpu.cu:57-64)
                if (i >= 1) {
                    const T dz = st.ez[st.at(s, i, j + 1)] - st.ez[a];
                    st.hx[a] = msub2<T>(T(1), st.hx[a], u1, dz);
                }
                // Hy: i in [0, nx), j in [1, ny)   (fields_updates_gpu.cu:67-76)
                if (j >= 1) {
                    const T dz = st.ez[st.at(s, i + 1, j)] - st.ez[a];
                    st.hy[a] = madd2<T>(T(1), st.hy[a], u1, dz);
                }
            }
        }
    if (th <= 0) return;
    // slab order of G.pmls: x0, y0, xmax, ymax (compute.py:267-313 over PML.boundaryIDs)
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s)
        for (int j = 0; j < ny; ++j) {
            // x0 (xminus): Hy at ii = th-1-i1 (pml_updates_h.cu:37-54)
            for (int i1 = 0; i1 < th; ++i1) {
                const int ii = th - 1 - i1;
                const size_t a = st.at(s, ii, j);
                const T dEz = (st.ez[st.at(s, ii + 1, j)] - st.ez[a]) / k.d;
                T& phi = st.ph_x0[((size_t)s * th + i1) * ny + j];
                const T ra1 = k.HRA[i1] - T(1);
                const T t = madd2<T>(ra1, dEz, k.HRB[i1], phi);
                st.hy[a] = fmaT<T>(k.uH4[k.c(ii, j)], t, st.hy[a]);
                phi = msub2<T>(k.HRE[i1], phi, k.HRF[i1], dEz);
            }
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s)
        for (int i = 0; i < nx; ++i) {
            // y0 (yminus): Hx at jj = th-1-j1 (pml_updates_h.cu:273-290)
            for (int j1 = 0; j1 < th; ++j1) {
                const int jj = th - 1 - j1;
                const size_t a = st.at(s, i, jj);
                const T dEz = (st.ez[st.at(s, i, jj + 1)] - st.ez[a]) / k.d;
                T& phi = st.ph_y0[((size_t)s * nx + i) * th + j1];
                const T ra1 = k.HRA[j1] - T(1);
                const T t = madd2<T>(ra1, dEz, k.HRB[j1], phi);
                st.hx[a] = fmaT<T>(-k.uH4[k.c(i, jj)], t, st.hx[a]);
                phi = msub2<T>(k.HRE[j1], phi, k.HRF[j1], dEz);
            }
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s)
        for (int j = 0; j < ny; ++j) {
            // xmax (xplus): Hy at ii = nx-th+i1 (pml_updates_h.cu:153-171)
            for (int i1 = 0; i1 < th; ++i1) {
                const int ii = nx - th + i1;
                const size_t a = st.at(s, ii, j);
                const T dEz = (st.ez[st.at(s, ii + 1, j)] - st.ez[a]) / k.d;
                T& phi = st.ph_xm[((size_t)s * th + i1) * ny + j];
                const T ra1 = k.HRA[i1] - T(1);
                const T t = madd2<T>(ra1, dEz, k.HRB[i1], phi);
                st.hy[a] = fmaT<T>(k.uH4[k.c(ii, j)], t, st.hy[a]);
                phi = msub2<T>(k.HRE[i1], phi, k.HRF[i1], dEz);
            }
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s)
        for (int i = 0; i < nx; ++i) {
            // ymax (yplus): Hx at jj = ny-th+j1 (pml_updates_h.cu:388-405)
            for (int j1 = 0; j1 < th; ++j1) {
                const int jj = ny - th + j1;
                const size_t a = st.at(s, i, jj);
                const T dEz = (st.ez[st.at(s, i, jj + 1)] - st.ez[a]) / k.d;
                T& phi = st.ph_ym[((size_t)s * nx + i) * th + j1];
                const T ra1 = k.HRA[j1] - T(1);
                const T t = madd2<T>(ra1, dEz, k.HRB[j1], phi);
                st.hx[a] = fmaT<T>(-k.uH4[k.c(i, jj)], t, st.hx[a]);
                phi = msub2<T>(k.HRE[j1], phi, k.HRF[j1], dEz);
            }
        }
}

// ---- E phase: e_fields_updates_gpu then Order1_{xminus,yminus,xplus,yplus} (E)
template <typename T>
void e_phase(State<T>& st, const Coeffs<T>& k, const T* uE0) {
    const int nx = st.nx, ny = st.ny, th = st.th, S = st.S;
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s)
        for (int i = 1; i < nx; ++i)
            for (int j = 1; j < ny; ++j) {
                // fields_updates_gpu.cu:21-32
                const size_t a = st.at(s, i, j);
                const size_t c = k.c(i, j);
                const T dHy = st.hy[a] - st.hy[st.at(s, i - 1, j)];
                const T dHx = st.hx[a] - st.hx[st.at(s, i, j - 1)];
                const T e = madd2<T>(uE0[c], st.ez[a], k.uE1[c], dHy);
                st.ez[a] = fmaT<T>(-k.uE1[c], dHx, e);
            }
    if (th <= 0) return;
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s)
        for (int j = 0; j < ny; ++j) {
            // x0 (xminus): Ez at ii = th - i2 (pml_updates_e.cu:58-76)
            for (int i2 = 0; i2 < th; ++i2) {
                const int ii = th - i2;
                const size_t a = st.at(s, ii, j);
                const T dHy = (st.hy[a] - st.hy[st.at(s, ii - 1, j)]) / k.d;
                T& phi = st.pe_x0[((size_t)s * th + i2) * ny + j];
                const T ra1 = k.ERA[i2] - T(1);
                const T t = madd2<T>(ra1, dHy, k.ERB[i2], phi);
                st.ez[a] = fmaT<T>(k.uE4[k.c(ii, j)], t, st.ez[a]);
                phi = msub2<T>(k.ERE[i2], phi, k.ERF[i2], dHy);
            }
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s)
        for (int i = 0; i < nx; ++i) {
            // y0 (yminus): Ez at jj = th - j2 (pml_updates_e.cu:267-285)
            for (int j2 = 0; j2 < th; ++j2) {
                const int jj = th - j2;
                const size_t a = st.at(s, i, jj);
                const T dHx = (st.hx[a] - st.hx[st.at(s, i, jj - 1)]) / k.d;
                T& phi = st.pe_y0[((size_t)s * nx + i) * th + j2];
                const T ra1 = k.ERA[j2] - T(1);
                const T t = madd2<T>(ra1, dHx, k.ERB[j2], phi);
                st.ez[a] = fmaT<T>(-k.uE4[k.c(i, jj)], t, st.ez[a]);
                phi = msub2<T>(k.ERE[j2], phi, k.ERF[j2], dHx);
            }
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s)
        for (int j = 0; j < ny; ++j) {
            // xmax (xplus): Ez at ii = nx-th+i2 (pml_updates_e.cu:150-168)
            for (int i2 = 0; i2 < th; ++i2) {
                const int ii = nx - th + i2;
                const size_t a = st.at(s, ii, j);
                const T dHy = (st.hy[a] - st.hy[st.at(s, ii - 1, j)]) / k.d;
                T& phi = st.pe_xm[((size_t)s * th + i2) * ny + j];
                const T ra1 = k.ERA[i2] - T(1);
                const T t = madd2<T>(ra1, dHy, k.ERB[i2], phi);
                st.ez[a] = fmaT<T>(k.uE4[k.c(ii, j)], t, st.ez[a]);
                phi = msub2<T>(k.ERE[i2], phi, k.ERF[i2], dHy);
            }
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s)
        for (int i = 0; i < nx; ++i) {
            // ymax (yplus): Ez at jj = ny-th+j2 (pml_updates_e.cu:384-401)
            for (int j2 = 0; j2 < th; ++j2) {
                const int jj = ny - th + j2;
                const size_t a = st.at(s, i, jj);
                const T dHx = (st.hx[a] - st.hx[st.at(s, i, jj - 1)]) / k.d;
                T& phi = st.pe_ym[((size_t)s * nx + i) * th + j2];
                const T ra1 = k.ERA[j2] - T(1);
                const T t = madd2<T>(ra1, dHx, k.ERB[j2], phi);
                st.ez[a] = fmaT<T>(-k.uE4[k.c(i, jj)], t, st.ez[a]);
                phi = msub2<T>(k.ERE[j2], phi, k.ERF[j2], dHx);
            }
        }
}

// ---- Transposes of the two phases (the exact discrete adjoint of a step).
// A phase is linear in the state; written as F' = F + sum of terms, its
// transpose maps the adjoint state after the phase (bars) to the one before.
// Derivative buffers: dzx(s,i,j) / dzy(s,i,j) hold the adjoint of the
// differences Ez[i][j+1]-Ez[i][j] / Ez[i+1][j]-Ez[i][j] (H phase), and
// dhx / dhy those of Hx[i][j]-Hx[i][j-1] / Hy[i][j]-Hy[i-1][j] (E phase).
template <typename T>
void h_phase_T(State<T>& L, const Coeffs<T>& k) {
    const int nx = L.nx, ny = L.ny, th = L.th, S = L.S;
    const size_t N = (size_t)nx * ny;
    std::vector<T> dzx(N * S, T(0)), dzy(N * S, T(0));
    auto at = [&](int s, int i, int j) { return (size_t)s * N + (size_t)i * ny + j; };
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                const T u1 = k.uH1[k.c(i, j)];
                const size_t a = L.at(s, i, j);
                if (i >= 1) dzx[at(s, i, j)] = -u1 * L.hx[a];   // Hx' = Hx - u1 dzx
                if (j >= 1) dzy[at(s, i, j)] = u1 * L.hy[a];    // Hy' = Hy + u1 dzy
            }
    if (th > 0) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int s = 0; s < S; ++s)
            for (int j = 0; j < ny; ++j)
                for (int i1 = 0; i1 < th; ++i1) {
                    // Hy' += uH4 (ra1 dz/d + RB phi), phi' = RE phi - RF dz/d  (x0 then xmax rows)
                    for (int side = 0; side < 2; ++side) {
                        const int ii = side == 0 ? th - 1 - i1 : nx - th + i1;
                        T& phi = (side == 0 ? L.ph_x0 : L.ph_xm)[((size_t)s * th + i1) * ny + j];
                        const T hb = L.hy[L.at(s, ii, j)], u4 = k.uH4[k.c(ii, j)];
                        const T dd = u4 * (k.HRA[i1] - T(1)) * hb - k.HRF[i1] * phi;
                        phi = k.HRE[i1] * phi + u4 * k.HRB[i1] * hb;
#pragma omp atomic
                        dzy[at(s, ii, j)] += dd / k.d;
                    }
                }
#pragma omp parallel for collapse(2) schedule(static)
        for (int s = 0; s < S; ++s)
            for (int i = 0; i < nx; ++i)
                for (int j1 = 0; j1 < th; ++j1) {
                    // Hx' -= uH4 (ra1 dz/d + RB phi), phi' = RE phi - RF dz/d  (y0 then ymax columns)
                    for (int side = 0; side < 2; ++side) {
                        const int jj = side == 0 ? th - 1 - j1 : ny - th + j1;
                        T& phi = (side == 0 ? L.ph_y0 : L.ph_ym)[((size_t)s * nx + i) * th + j1];
                        const T hb = L.hx[L.at(s, i, jj)], u4 = k.uH4[k.c(i, jj)];
                        const T dd = -u4 * (k.HRA[j1] - T(1)) * hb - k.HRF[j1] * phi;
                        phi = k.HRE[j1] * phi - u4 * k.HRB[j1] * hb;
#pragma omp atomic
                        dzx[at(s, i, jj)] += dd / k.d;
                    }
                }
    }
    // Ez[i][j+1] - Ez[i][j] and Ez[i+1][j] - Ez[i][j]; the zero frame (i == nx,
    // j == ny) is not part of the state, so its adjoint is dropped
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                T e = L.ez[L.at(s, i, j)] - dzx[at(s, i, j)] - dzy[at(s, i, j)];
                if (j >= 1) e += dzx[at(s, i, j - 1)];
                if (i >= 1) e += dzy[at(s, i - 1, j)];
                L.ez[L.at(s, i, j)] = e;
            }
}

template <typename T>
void e_phase_T(State<T>& L, const Coeffs<T>& k) {
    const int nx = L.nx, ny = L.ny, th = L.th, S = L.S;
    const size_t N = (size_t)nx * ny;
    std::vector<T> dhx(N * S, T(0)), dhy(N * S, T(0)), eb(N * S);
    auto at = [&](int s, int i, int j) { return (size_t)s * N + (size_t)i * ny + j; };
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                const T e = L.ez[L.at(s, i, j)];
                eb[at(s, i, j)] = e;
                if (i >= 1 && j >= 1) {
                    // Ez' = uE0 Ez + uE1 dHy - uE1 dHx
                    const size_t c = k.c(i, j);
                    dhy[at(s, i, j)] = k.uE1[c] * e;
                    dhx[at(s, i, j)] = -k.uE1[c] * e;
                    L.ez[L.at(s, i, j)] = k.uE0[c] * e;
                }
            }
    if (th > 0) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int s = 0; s < S; ++s)
            for (int j = 0; j < ny; ++j)
                for (int i2 = 0; i2 < th; ++i2) {
                    // Ez' += uE4 (ra1 dHy/d + RB phi), phi' = RE phi - RF dHy/d  (x0 then xmax rows)
                    for (int side = 0; side < 2; ++side) {
                        const int ii = side == 0 ? th - i2 : nx - th + i2;
                        T& phi = (side == 0 ? L.pe_x0 : L.pe_xm)[((size_t)s * th + i2) * ny + j];
                        const T e = eb[at(s, ii, j)], u4 = k.uE4[k.c(ii, j)];
                        const T dd = u4 * (k.ERA[i2] - T(1)) * e - k.ERF[i2] * phi;
                        phi = k.ERE[i2] * phi + u4 * k.ERB[i2] * e;
#pragma omp atomic
                        dhy[at(s, ii, j)] += dd / k.d;
                    }
                }
#pragma omp parallel for collapse(2) schedule(static)
        for (int s = 0; s < S; ++s)
            for (int i = 0; i < nx; ++i)
                for (int j2 = 0; j2 < th; ++j2) {
                    // Ez' -= uE4 (ra1 dHx/d + RB phi), phi' = RE phi - RF dHx/d  (y0 then ymax columns)
                    for (int side = 0; side < 2; ++side) {
                        const int jj = side == 0 ? th - j2 : ny - th + j2;
                        T& phi = (side == 0 ? L.pe_y0 : L.pe_ym)[((size_t)s * nx + i) * th + j2];
                        const T e = eb[at(s, i, jj)], u4 = k.uE4[k.c(i, jj)];
                        const T dd = -u4 * (k.ERA[j2] - T(1)) * e - k.ERF[j2] * phi;
                        phi = k.ERE[j2] * phi - u4 * k.ERB[j2] * e;
#pragma omp atomic
                        dhx[at(s, i, jj)] += dd / k.d;
                    }
                }
    }
    // Hy[i][j] - Hy[i-1][j] and Hx[i][j] - Hx[i][j-1]
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                const size_t a = L.at(s, i, j);
                T hy = L.hy[a] + dhy[at(s, i, j)], hx = L.hx[a] + dhx[at(s, i, j)];
                if (i + 1 < nx) hy -= dhy[at(s, i + 1, j)];
                if (j + 1 < ny) hx -= dhx[at(s, i, j + 1)];
                L.hy[a] = hy;
                L.hx[a] = hx;
            }
}

template <typename T>
Coeffs<T> make_coeffs(const OracleProblem* p) {
    Coeffs<T> k;
    k.uE0 = (const T*)p->uE0; k.uE1 = (const T*)p->uE1; k.uE4 = (const T*)p->uE4;
    k.uH1 = (const T*)p->uH1; k.uH4 = (const T*)p->uH4;
    const T* pm = (const T*)p->pml;
    const int th = p->th;
    k.ERA = pm; k.ERB = pm + th; k.ERE = pm + 2 * th; k.ERF = pm + 3 * th;
    k.HRA = pm + 4 * th; k.HRB = pm + 5 * th; k.HRE = pm + 6 * th; k.HRF = pm + 7 * th;
    k.d = (T)p->d;
    k.ny = p->ny;
    return k;
}

// Forward loop, compute.py:574-712.  traces: (S, nt, nrx); hist: (nt, S, nx, ny)
// holding Ez after each step (the reference's Ez_hist), or NULL.
template <typename T>
int forward_impl(const OracleProblem* p, T* traces, T* hist) {
    const int nx = p->nx, ny = p->ny, S = p->S, nt = p->nt, nrx = p->nrx, nsrc = p->nsrc;
    State<T> st(nx, ny, p->th, S);
    Coeffs<T> k = make_coeffs<T>(p);
    const T* srcw = (const T*)p->srcw;
    for (int t = 0; t < nt; ++t) {
        // store_outputs (sourcereceiver.cu:21-35): Ez at the start of the step
        for (int s = 0; s < S; ++s)
            for (int r = 0; r < nrx; ++r) {
                const int i = p->rx[((size_t)s * nrx + r) * 2], j = p->rx[((size_t)s * nrx + r) * 2 + 1];
                traces[((size_t)s * nt + t) * nrx + r] = (i < 0) ? T(0) : st.ez[st.at(s, i, j)];
            }
        h_phase<T>(st, k);
        e_phase<T>(st, k, k.uE0);
        // Update_hertzian_dipole (sourcereceiver.cu:68-86), polarisation z
        for (int s = 0; s < S; ++s)
            for (int n = 0; n < nsrc; ++n) {
                const int i = p->src[((size_t)s * nsrc + n) * 2], j = p->src[((size_t)s * nsrc + n) * 2 + 1];
                if (i < 0) continue;
                const size_t a = st.at(s, i, j);
                st.ez[a] = fmaT<T>(-k.uE4[k.c(i, j)], srcw[(size_t)n * nt + t], st.ez[a]);
            }
        if (hist) {
            // Ez[iteration] = G.Ez_gpu[:, :nx, :ny, :nz]  (compute.py:712)
            for (int s = 0; s < S; ++s)
                for (int i = 0; i < nx; ++i)
                    std::memcpy(hist + (((size_t)t * S + s) * nx + i) * ny, &st.ez[st.at(s, i, 0)], sizeof(T) * ny);
        }
    }
    return 0;
}

// Reference adjoint, compute.py:1048-1172 with backinitialization's source =
// receivers (compute.py:973) and Ucgeta's uE0 (uc.cu:85).  g: (S, nt, nrx)
// residual; ge/gs: (nx, ny) UNNORMALISED imaging sums in T, accumulated as the
// reference does (sum over shots, then add, once per step).
template <typename T>
int adjoint_ref_impl(const OracleProblem* p, const T* hist, const T* g, T* ge, T* gs) {
    const int nx = p->nx, ny = p->ny, S = p->S, nt = p->nt, nrx = p->nrx;
    State<T> st(nx, ny, p->th, S);
    Coeffs<T> k = make_coeffs<T>(p);
    const T* uE0a = (const T*)p->uE0a;
    const T dt = (T)p->dt;
    const size_t N = (size_t)nx * ny;
    for (size_t c = 0; c < N; ++c) { ge[c] = T(0); gs[c] = T(0); }
    for (int it = nt - 1; it >= 1; --it) {
        // Back_source (back.cu:8-37, the subtraction at :33-34): raw residual, no scaling
        for (int s = 0; s < S; ++s)
            for (int r = 0; r < nrx; ++r) {
                const int i = p->rx[((size_t)s * nrx + r) * 2], j = p->rx[((size_t)s * nrx + r) * 2 + 1];
                if (i < 0) continue;
                const size_t a = st.at(s, i, j);
                st.ez[a] = st.ez[a] - g[((size_t)s * nt + it) * nrx + r];
            }
        e_phase<T>(st, k, uE0a);
        h_phase<T>(st, k);
        // imaging (compute.py:1167-1172)
        const T* f1 = hist + (size_t)it * S * N;
        const T* f0 = hist + (size_t)(it - 1) * S * N;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                T se = T(0), ss = T(0);
                for (int s = 0; s < S; ++s) {
                    const size_t h = (size_t)s * N + (size_t)i * ny + j;
                    const T lam = st.ez[st.at(s, i, j)];
                    se += (f1[h] - f0[h]) * lam;
                    ss += (f1[h] * lam) * dt;
                }
                ge[(size_t)i * ny + j] += se;
                gs[(size_t)i * ny + j] += ss;
            }
    }
    return 0;
}

// Exact discrete adjoint of forward_impl for the functional
// J = sum_{s,t,r} w[s][t][r] traces[s][t][r].  traces[t] reads Ez of x_t, the
// state after t steps (x_0 = 0), and step t maps x_t to x_{t+1} = E(H(x_t)) +
// source.  The adjoint runs lambda_{nt-1} = R^T w_{nt-1}, lambda_{t-1} =
// S^T lambda_t + R^T w_{t-1}; the model enters step t-1 only through the E
// coefficients of x_t's Ez, so the sums
//   s1 = sum_{t>=1} sum_s lambda_t Ez(x_{t-1}),  s2 = sum_{t>=1} sum_s lambda_t Ez(x_t)
// (per cell) give the gradient (oracle.adjoint_exact forms it).  hist: the
// forward's (nt, S, nx, ny) Ez history, hist[t] = Ez of x_{t+1}.
template <typename T>
int adjoint_exact_impl(const OracleProblem* p, const T* hist, const T* w, T* s1, T* s2) {
    const int nx = p->nx, ny = p->ny, S = p->S, nt = p->nt, nrx = p->nrx;
    State<T> L(nx, ny, p->th, S);
    Coeffs<T> k = make_coeffs<T>(p);
    const size_t N = (size_t)nx * ny;
    for (size_t c = 0; c < N; ++c) { s1[c] = T(0); s2[c] = T(0); }
    auto inject = [&](int t) {
        for (int s = 0; s < S; ++s)
            for (int r = 0; r < nrx; ++r) {
                const int i = p->rx[((size_t)s * nrx + r) * 2], j = p->rx[((size_t)s * nrx + r) * 2 + 1];
                if (i < 0) continue;
                L.ez[L.at(s, i, j)] += w[((size_t)s * nt + t) * nrx + r];
            }
    };
    // Row 0 (Ez, Hx, the y-slab auxiliaries of row 0) and column 0 (Ez, Hy,
    // the x-slab auxiliaries of column 0) form closed subsystems of the
    // forward step: they are updated only by the CPML terms of their own
    // cells and feed the rest of the grid without being fed by it.  With no
    // source on them they stay exactly zero in the forward, so no J depends
    // on them; their transposed dynamics (an unstable CPML-only recursion,
    // whose adjoint the rest of the grid drives) are projected out, which
    // keeps the adjoint finite without changing the gradient.
    bool edge_src = false;
    for (int q = 0; q < S * p->nsrc; ++q)
        if (p->src[2 * q] == 0 || p->src[2 * q + 1] == 0) edge_src = true;
    auto project = [&]() {
        if (edge_src) return;
        for (int s = 0; s < S; ++s) {
            for (int j = 0; j < ny; ++j) {
                L.ez[L.at(s, 0, j)] = T(0);
                L.hx[L.at(s, 0, j)] = T(0);
            }
            for (int i = 0; i < nx; ++i) {
                L.ez[L.at(s, i, 0)] = T(0);
                L.hy[L.at(s, i, 0)] = T(0);
            }
            const int th = p->th;
            for (int q = 0; q < th; ++q) {
                L.pe_y0[((size_t)s * nx + 0) * th + q] = L.pe_ym[((size_t)s * nx + 0) * th + q] = T(0);
                L.ph_y0[((size_t)s * nx + 0) * th + q] = L.ph_ym[((size_t)s * nx + 0) * th + q] = T(0);
                L.pe_x0[((size_t)s * th + q) * ny + 0] = L.pe_xm[((size_t)s * th + q) * ny + 0] = T(0);
                L.ph_x0[((size_t)s * th + q) * ny + 0] = L.ph_xm[((size_t)s * th + q) * ny + 0] = T(0);
            }
        }
    };
    if (nt < 2) return 0;
    inject(nt - 1);
    for (int t = nt - 1; t >= 1; --t) {
        const T* xt = hist + (size_t)(t - 1) * S * N;
        const T* xp = t >= 2 ? hist + (size_t)(t - 2) * S * N : nullptr;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                T a = T(0), b = T(0);
                for (int s = 0; s < S; ++s) {
                    const size_t h = (size_t)s * N + (size_t)i * ny + j;
                    const T lam = L.ez[L.at(s, i, j)];
                    if (xp) a += lam * xp[h];
                    b += lam * xt[h];
                }
                s1[(size_t)i * ny + j] += a;
                s2[(size_t)i * ny + j] += b;
            }
        if (t >= 2) {
            e_phase_T<T>(L, k);
            h_phase_T<T>(L, k);
            project();
            inject(t - 1);
        }
    }
    return 0;
}

// One homogeneous step (no source) of a packed state, or its transpose.
// Packing: ez, hx, hy (S (nx+1) (ny+1) each), then pe_x0, pe_xm (S th ny),
// pe_y0, pe_ym (S nx th), ph_x0, ph_xm, ph_y0, ph_ym likewise.
template <typename T>
void state_io(State<T>& st, T* buf, bool load) {
    std::vector<T>* parts[11] = {&st.ez, &st.hx, &st.hy, &st.pe_x0, &st.pe_xm, &st.pe_y0, &st.pe_ym,
                                 &st.ph_x0, &st.ph_xm, &st.ph_y0, &st.ph_ym};
    for (auto* v : parts) {
        if (load) std::memcpy(v->data(), buf, v->size() * sizeof(T));
        else std::memcpy(buf, v->data(), v->size() * sizeof(T));
        buf += v->size();
    }
}
template <typename T>
int step_impl(const OracleProblem* p, const T* in, T* out, int transpose) {
    State<T> st(p->nx, p->ny, p->th, p->S);
    Coeffs<T> k = make_coeffs<T>(p);
    state_io<T>(st, const_cast<T*>(in), true);
    if (transpose) {
        e_phase_T<T>(st, k);
        h_phase_T<T>(st, k);
    } else {
        h_phase<T>(st, k);
        e_phase<T>(st, k, k.uE0);
    }
    state_io<T>(st, out, false);
    return 0;
}

}  // namespace

extern "C" {

int oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int oracle_forward(const OracleProblem* p, void* traces, void* hist) {
    if (!p || !traces) return -1;
    if (p->dtype == 0) return forward_impl<float>(p, (float*)traces, (float*)hist);
    if (p->dtype == 1) return forward_impl<double>(p, (double*)traces, (double*)hist);
    return -2;
}

int oracle_adjoint_exact(const OracleProblem* p, const void* hist, const void* w, void* s1, void* s2) {
    if (!p || !hist || !w || !s1 || !s2) return -1;
    if (p->dtype == 0) return adjoint_exact_impl<float>(p, (const float*)hist, (const float*)w, (float*)s1, (float*)s2);
    if (p->dtype == 1)
        return adjoint_exact_impl<double>(p, (const double*)hist, (const double*)w, (double*)s1, (double*)s2);
    return -2;
}

int oracle_step(const OracleProblem* p, const void* in, void* out, int transpose) {
    if (!p || !in || !out) return -1;
    if (p->dtype == 0) return step_impl<float>(p, (const float*)in, (float*)out, transpose);
    if (p->dtype == 1) return step_impl<double>(p, (const double*)in, (double*)out, transpose);
    return -2;
}

int oracle_adjoint_ref(const OracleProblem* p, const void* hist, const void* g, void* ge, void* gs) {
    if (!p || !hist || !g || !ge || !gs) return -1;
    if (p->dtype == 0) return adjoint_ref_impl<float>(p, (const float*)hist, (const float*)g, (float*)ge, (float*)gs);
    if (p->dtype == 1) return adjoint_ref_impl<double>(p, (const double*)hist, (const double*)g, (double*)ge, (double*)gs);
    return -2;
}

}  // extern "C"
