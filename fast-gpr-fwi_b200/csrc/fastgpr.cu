// libfastgpr: plan construction, workspace layout and the C ABI declared in
// include/fastgpr.h.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fastgpr.h"
#include "fdtd_kernels.cuh"
#include "fdtd_tma.cuh"
#include "fdtd_tile.cuh"
#include "fdtd_march.cuh"

using fg::Ev;
using fg::GridDev;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(FG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define FG_CUDA(call)                                   \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

struct fg_plan {
    // problem
    int nx, ny, S, nt, th, nsrc, nrx;
    float dx, dt;
    std::vector<int32_t> src, rx;
    std::vector<float> srcw, pml;
    // tiling
    int kernel, V, G, TI, NW, D;
    int P, TY, Ph, nb, nc, ngroups, ntiles, bw;
    std::vector<int> chunk_row;
    std::vector<Ev> src_ev, rx_ev, inj_ev, injh_ev;
    std::vector<int> src_off, rx_off, inj_off, injh_off;
    // workspace layout (byte offsets)
    size_t o_coef, o_state, o_psi, o_chunk, o_srcev, o_rxev, o_injev, o_injhev, o_offs, o_srcw, o_pml, o_gacc,
        o_sums, o_partial, o_norms, o_err, total;
    long long plane, pxs, pys;
    size_t state_bytes, psi_bytes;
    char* ws = nullptr;
    int64_t ws_bytes = 0;
    GridDev g;
};

namespace {

constexpr int kRedBlocks = 256;

// Classify a cell position: 1 = active, 0 = inert (zero frame or the dead
// k=1 plane of the reference layout), -1 = outside the reference's arrays.
int classify(const fg_plan* p, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i > p->nx || j > p->ny || k > 1) return -1;
    if (k == 1 || i == p->nx || j == p->ny) return 0;
    return 1;
}

void build_tiles(fg_plan* p) {
    p->P = (int)align_up((size_t)p->ny + 1, 32);
    p->TY = (int)align_up((size_t)std::max(p->th, 1), 4);
    p->Ph = (int)align_up((size_t)p->ny, 4);
    p->bw = p->kernel == 0 ? p->NW * 32 * p->V : 32 * p->V;   // register march and tiles: one warp wide
    p->nb = (p->ny + p->bw - 1) / p->bw;
    p->nc = std::max(1, (p->nx + p->TI - 1) / p->TI);
    p->ngroups = (p->S + p->G - 1) / p->G;
    p->ntiles = p->ngroups * p->nc * p->nb;
    p->chunk_row.resize(p->nc + 1);
    for (int c = 0; c <= p->nc; ++c) p->chunk_row[c] = (int)((long long)c * p->nx / p->nc);

    const int bw = p->bw;
    auto tile_events = [&](std::vector<Ev>& out, std::vector<int>& off, auto&& gen) {
        out.clear();
        off.assign(p->ntiles + 1, 0);
        for (int t = 0; t < p->ntiles; ++t) {
            const int band = t % p->nb, rest = t / p->nb, chunk = rest % p->nc, grp = rest / p->nc;
            std::vector<Ev> evs;
            gen(evs, grp, p->chunk_row[chunk], p->chunk_row[chunk + 1], band * bw, band * bw + bw);
            std::stable_sort(evs.begin(), evs.end(), [](const Ev& a, const Ev& b) {
                if (a.x != b.x) return a.x < b.x;
                if (a.y != b.y) return a.y < b.y;
                if (a.z != b.z) return a.z < b.z;
                return a.w < b.w;
            });
            out.insert(out.end(), evs.begin(), evs.end());
            off[t + 1] = (int)out.size();
        }
    };
    // sources with a non-zero waveform row
    std::vector<char> live(p->nsrc, 0);
    for (int n = 0; n < p->nsrc; ++n)
        for (int t = 0; t < p->nt; ++t)
            if (p->srcw[(size_t)n * p->nt + t] != 0.f) { live[n] = 1; break; }

    auto pos = [&](const std::vector<int32_t>& tab, int count, int s, int n, int c) {
        return tab[((size_t)s * count + n) * 3 + c];
    };
    tile_events(p->src_ev, p->src_off, [&](std::vector<Ev>& evs, int grp, int i0, int i1, int b0, int be) {
        for (int q = 0; q < p->G; ++q) {
            const int s = grp * p->G + q;
            if (s >= p->S) break;
            for (int n = 0; n < p->nsrc; ++n) {
                if (!live[n]) continue;
                const int i = pos(p->src, p->nsrc, s, n, 0), j = pos(p->src, p->nsrc, s, n, 1),
                          k = pos(p->src, p->nsrc, s, n, 2);
                if (classify(p, i, j, k) != 1) continue;
                if (i >= i0 && i < i1 && j >= b0 && j < be) evs.push_back(make_int4(i, q, j, n));
            }
        }
    });
    tile_events(p->rx_ev, p->rx_off, [&](std::vector<Ev>& evs, int grp, int i0, int i1, int b0, int be) {
        for (int q = 0; q < p->G; ++q) {
            const int s = grp * p->G + q;
            if (s >= p->S) break;
            for (int r = 0; r < p->nrx; ++r) {
                const int i = pos(p->rx, p->nrx, s, r, 0), j = pos(p->rx, p->nrx, s, r, 1),
                          k = pos(p->rx, p->nrx, s, r, 2);
                if (classify(p, i, j, k) != 1) continue;
                if (i >= i0 && i < i1 && j >= b0 && j < be) evs.push_back(make_int4(i, q, j, r));
            }
        }
    });
    // adjoint injections: rows [i0, i1] (row i1 is recomputed as a halo row)
    tile_events(p->inj_ev, p->inj_off, [&](std::vector<Ev>& evs, int grp, int i0, int i1, int b0, int be) {
        for (int q = 0; q < p->G; ++q) {
            const int s = grp * p->G + q;
            if (s >= p->S) break;
            for (int r = 0; r < p->nrx; ++r) {
                const int i = pos(p->rx, p->nrx, s, r, 0), j = pos(p->rx, p->nrx, s, r, 1),
                          k = pos(p->rx, p->nrx, s, r, 2);
                if (classify(p, i, j, k) != 1) continue;
                if (i >= i0 && i <= i1 && j >= b0 && j < be) evs.push_back(make_int4(i, q, j, r));
            }
        }
    });
    // adjoint injections on the halo column be, rows [i0, i1)
    tile_events(p->injh_ev, p->injh_off, [&](std::vector<Ev>& evs, int grp, int i0, int i1, int, int be) {
        for (int q = 0; q < p->G; ++q) {
            const int s = grp * p->G + q;
            if (s >= p->S) break;
            for (int r = 0; r < p->nrx; ++r) {
                const int i = pos(p->rx, p->nrx, s, r, 0), j = pos(p->rx, p->nrx, s, r, 1),
                          k = pos(p->rx, p->nrx, s, r, 2);
                if (classify(p, i, j, k) != 1) continue;
                if (i >= i0 && i < i1 && j == be) evs.push_back(make_int4(i, q, j, r));
            }
        }
    });
}

void layout(fg_plan* p) {
    const size_t A = 256;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o = align_up(o + std::max<size_t>(bytes, 1), A);
        return at;
    };
    p->plane = (long long)(p->nx + 1) * p->P;
    p->pxs = 2LL * p->th * p->P;
    p->pys = 2LL * (p->nx + 1) * p->TY;
    p->o_coef = take(5 * (size_t)p->plane * sizeof(float));
    p->state_bytes = 6 * (size_t)p->S * p->plane * sizeof(float);
    p->psi_bytes = 4 * (size_t)p->S * (p->pxs + p->pys) * sizeof(float);
    p->o_state = take(p->state_bytes);
    p->o_psi = take(p->psi_bytes);
    p->o_chunk = take((p->nc + 1) * sizeof(int));
    p->o_srcev = take(p->src_ev.size() * sizeof(Ev));
    p->o_rxev = take(p->rx_ev.size() * sizeof(Ev));
    p->o_injev = take(p->inj_ev.size() * sizeof(Ev));
    p->o_injhev = take(p->injh_ev.size() * sizeof(Ev));
    p->o_offs = take(4 * (size_t)(p->ntiles + 1) * sizeof(int));
    p->o_srcw = take((size_t)p->nsrc * p->nt * sizeof(float));
    p->o_pml = take(8 * (size_t)p->th * sizeof(float));
    const size_t n = (size_t)p->nx * p->ny;
    p->o_gacc = take((size_t)p->ngroups * 2 * n * sizeof(double));
    p->o_sums = take(2 * n * sizeof(double));
    p->o_partial = take(2 * kRedBlocks * sizeof(double));
    p->o_norms = take(2 * sizeof(double));
    p->o_err = take(sizeof(int) * 4);
    p->total = o;
}

void fill_grid(fg_plan* p) {
    GridDev& g = p->g;
    std::memset(&g, 0, sizeof(g));
    char* w = p->ws;
    g.nx = p->nx; g.ny = p->ny; g.P = p->P; g.th = p->th; g.TY = p->TY;
    g.S = p->S; g.nt = p->nt; g.nrx = p->nrx; g.Ph = p->Ph;
    g.d = p->dx; g.dt = p->dt;
    g.plane = p->plane; g.pxs = p->pxs; g.pys = p->pys;
    float* coef = (float*)(w + p->o_coef);
    g.ca = coef; g.cb = coef + p->plane; g.cd = coef + 2 * p->plane; g.ch = coef + 3 * p->plane;
    g.ci = coef + 4 * p->plane;
    g.pml = (const float*)(w + p->o_pml);
    float* st = (float*)(w + p->o_state);
    const long long sp = (long long)p->S * p->plane;
    g.ez[0] = st; g.ez[1] = st + sp; g.hx[0] = st + 2 * sp; g.hx[1] = st + 3 * sp;
    g.hy[0] = st + 4 * sp; g.hy[1] = st + 5 * sp;
    float* ps = (float*)(w + p->o_psi);
    const long long xs = (long long)p->S * p->pxs, ys = (long long)p->S * p->pys;
    g.pex[0] = ps; g.pex[1] = ps + xs; g.phx[0] = ps + 2 * xs; g.phx[1] = ps + 3 * xs;
    float* py = ps + 4 * xs;
    g.pey[0] = py; g.pey[1] = py + ys; g.phy[0] = py + 2 * ys; g.phy[1] = py + 3 * ys;
    g.nb = p->nb; g.nc = p->nc; g.G = p->G; g.ngroups = p->ngroups; g.ntiles = p->ntiles;
    g.chunk_row = (const int*)(w + p->o_chunk);
    g.src_ev = (const Ev*)(w + p->o_srcev);
    g.rx_ev = (const Ev*)(w + p->o_rxev);
    g.inj_ev = (const Ev*)(w + p->o_injev);
    g.injh_ev = (const Ev*)(w + p->o_injhev);
    const int* offs = (const int*)(w + p->o_offs);
    g.src_off = offs; g.rx_off = offs + (p->ntiles + 1); g.inj_off = offs + 2 * (p->ntiles + 1);
    g.injh_off = offs + 3 * (p->ntiles + 1);
    g.srcw = (const float*)(w + p->o_srcw);
    g.gacc = (double*)(w + p->o_gacc);
    g.ws_lo = w;
    g.ws_hi = w + p->total;
    g.err = (int*)(w + p->o_err);
}

template <int V, int G>
void launch_forward(const GridDev& g, int t, cudaStream_t st) {
    const int blocks = (g.ntiles + 3) / 4;
    fg::k_forward_step<V, G><<<blocks, 128, 0, st>>>(g, t);
}
template <int V, int G>
void launch_adjoint(const GridDev& g, int it, int rp, cudaStream_t st) {
    const int blocks = (g.ntiles + 3) / 4;
    fg::k_adjoint_step<V, G><<<blocks, 128, 0, st>>>(g, it, rp);
}

template <int V, int G>
cudaError_t launch_forward_tma(const GridDev& g, int t, int nw, int D, cudaStream_t st) {
    const size_t smem = fg::ring_smem_bytes(D, 5 + 6 * G, fg::ring_slot_width(nw * 32 * V, g.TY), g.th);
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(fg::k_forward_tma<V, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    });
    if (attr != cudaSuccess) return attr;
    fg::k_forward_tma<V, G><<<g.ntiles, (nw + 1) * 32, smem, st>>>(g, t, D);
    return cudaSuccess;
}
template <int V, int G>
cudaError_t launch_adjoint_tma(const GridDev& g, int it, int rp, int nw, int D, cudaStream_t st) {
    const size_t smem = fg::ring_smem_bytes(D, 5 + 8 * G, fg::ring_slot_width(nw * 32 * V, g.TY), g.th);
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(fg::k_adjoint_tma<V, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    });
    if (attr != cudaSuccess) return attr;
    fg::k_adjoint_tma<V, G><<<g.ntiles, (nw + 1) * 32, smem, st>>>(g, it, rp, D);
    return cudaSuccess;
}
template <int V>
cudaError_t launch_forward_tile(const GridDev& g, int t, int TH, int G, cudaStream_t st) {
    fg::k_forward_tile<V><<<g.ntiles, 32 * TH, fg::tile_fwd_smem(TH, V), st>>>(g, t, G);
    return cudaSuccess;
}
template <int V>
cudaError_t launch_adjoint_tile(const GridDev& g, int it, int rp, int TH, int G, cudaStream_t st) {
    fg::k_adjoint_tile<V><<<g.ntiles, 32 * TH, fg::tile_adj_smem(TH, V), st>>>(g, it, rp, G);
    return cudaSuccess;
}
template <int V>
cudaError_t launch_forward_march(const GridDev& g, int t, int TI, int G, cudaStream_t st) {
    (void)TI;
    const int blocks = (g.ntiles + fg::MARCH_WARPS - 1) / fg::MARCH_WARPS;
    fg::k_forward_march<V><<<blocks, 32 * fg::MARCH_WARPS, 0, st>>>(g, t, G);
    return cudaSuccess;
}
template <int V>
cudaError_t launch_adjoint_march(const GridDev& g, int it, int rp, int TI, int G, cudaStream_t st) {
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(fg::k_adjoint_march<V>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    });
    if (attr != cudaSuccess) return attr;
    const int blocks = (g.ntiles + fg::MARCH_WARPS - 1) / fg::MARCH_WARPS;
    fg::k_adjoint_march<V><<<blocks, 32 * fg::MARCH_WARPS, fg::march_adj_smem(TI, V), st>>>(g, it, rp, G, TI);
    return cudaSuccess;
}

using FwdTileFn = cudaError_t (*)(const GridDev&, int, int, int, cudaStream_t);
using AdjTileFn = cudaError_t (*)(const GridDev&, int, int, int, int, cudaStream_t);
FwdTileFn pick_fwd_march(int V) {
    switch (V) {
        case 1: return launch_forward_march<1>;
        case 2: return launch_forward_march<2>;
        case 4: return launch_forward_march<4>;
    }
    return nullptr;
}
AdjTileFn pick_adj_march(int V);
FwdTileFn pick_fwd_tile(int V) {
    switch (V) {
        case 1: return launch_forward_tile<1>;
        case 2: return launch_forward_tile<2>;
        case 4: return launch_forward_tile<4>;
    }
    return nullptr;
}
AdjTileFn pick_adj_march(int V) {
    switch (V) {
        case 1: return launch_adjoint_march<1>;
        case 2: return launch_adjoint_march<2>;
        case 4: return launch_adjoint_march<4>;
    }
    return nullptr;
}
AdjTileFn pick_adj_tile(int V) {
    switch (V) {
        case 1: return launch_adjoint_tile<1>;
        case 2: return launch_adjoint_tile<2>;
        case 4: return launch_adjoint_tile<4>;
    }
    return nullptr;
}

using FwdTmaFn = cudaError_t (*)(const GridDev&, int, int, int, cudaStream_t);
using AdjTmaFn = cudaError_t (*)(const GridDev&, int, int, int, int, cudaStream_t);
template <int V>
FwdTmaFn pick_fwd_tma_g(int G) {
    switch (G) {
        case 1: return launch_forward_tma<V, 1>;
        case 2: return launch_forward_tma<V, 2>;
        case 4: return launch_forward_tma<V, 4>;
    }
    return nullptr;
}
FwdTmaFn pick_fwd_tma(int V, int G) {
    switch (V) {
        case 1: return pick_fwd_tma_g<1>(G);
        case 2: return pick_fwd_tma_g<2>(G);
        case 4: return pick_fwd_tma_g<4>(G);
    }
    return nullptr;
}
template <int V>
AdjTmaFn pick_adj_tma_g(int G) {
    switch (G) {
        case 1: return launch_adjoint_tma<V, 1>;
        case 2: return launch_adjoint_tma<V, 2>;
        case 4: return launch_adjoint_tma<V, 4>;
    }
    return nullptr;
}
AdjTmaFn pick_adj_tma(int V, int G) {
    switch (V) {
        case 1: return pick_adj_tma_g<1>(G);
        case 2: return pick_adj_tma_g<2>(G);
        case 4: return pick_adj_tma_g<4>(G);
    }
    return nullptr;
}

using FwdFn = void (*)(const GridDev&, int, cudaStream_t);
using AdjFn = void (*)(const GridDev&, int, int, cudaStream_t);

template <int V>
FwdFn pick_fwd_g(int G) {
    switch (G) {
        case 1: return launch_forward<V, 1>;
        case 2: return launch_forward<V, 2>;
        case 4: return launch_forward<V, 4>;
        case 8: return launch_forward<V, 8>;
    }
    return nullptr;
}
FwdFn pick_fwd(int V, int G) {
    switch (V) {
        case 1: return pick_fwd_g<1>(G);
        case 2: return pick_fwd_g<2>(G);
        case 4: return pick_fwd_g<4>(G);
    }
    return nullptr;
}
template <int V>
AdjFn pick_adj_g(int G) {
    switch (G) {
        case 1: return launch_adjoint<V, 1>;
        case 2: return launch_adjoint<V, 2>;
        case 4: return launch_adjoint<V, 4>;
        case 8: return launch_adjoint<V, 8>;
    }
    return nullptr;
}
AdjFn pick_adj(int V, int G) {
    switch (V) {
        case 1: return pick_adj_g<1>(G);
        case 2: return pick_adj_g<2>(G);
        case 4: return pick_adj_g<4>(G);
    }
    return nullptr;
}

int coefficients(const float* er, const float* se, const float* mr, int nx, int ny, float dt, float dx, int adjoint,
                 float* out, int P, cudaStream_t st) {
    const long long n = (long long)(nx + 1) * P;
    const int threads = 256;
    const long long blocks = (n + threads - 1) / threads;
    fg::k_coefficients<<<(unsigned)blocks, threads, 0, st>>>(er, se, mr, nx, ny, dt, dx, adjoint, out, P);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

int reset_state(fg_plan* p, cudaStream_t st) {
    FG_CUDA(cudaMemsetAsync(p->ws + p->o_state, 0, p->state_bytes, st));
    FG_CUDA(cudaMemsetAsync(p->ws + p->o_psi, 0, p->psi_bytes, st));
    return FG_OK;
}

// Device scratch of fg_forward_static: one array per GPU that loads the
// library, held until the process exits.  Host code must not pass the
// symbol itself to a kernel (on the host it names a host-side shadow); the
// device address comes from cudaGetSymbolAddress, looked up once per device.
static __device__ __align__(256) unsigned char g_static_scratch[FG_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
void* g_static_ptr[kMaxDevices] = {};

int static_scratch(void** out) {
    int dev = 0;
    FG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(FG_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_ptr[dev]) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static scratch)");
        g_static_ptr[dev] = ptr;
    }
    *out = g_static_ptr[dev];
    return FG_OK;
}

}  // namespace

extern "C" {

const char* fg_last_error(void) { return g_last_error.c_str(); }

int fg_plan_check(fg_plan* p, void* stream) {
    if (!p || !p->ws) return fail(FG_ERR_INVALID, "fg_plan_check: plan has no workspace");
    cudaStream_t st = (cudaStream_t)stream;
    int code = 0;
    FG_CUDA(cudaMemcpyAsync(&code, p->ws + p->o_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    if (code == 0) return FG_OK;
    FG_CUDA(cudaMemsetAsync(p->ws + p->o_err, 0, sizeof(int), st));
    if (code == 100) return fail(FG_ERR_INVALID, "device: out-of-range access caught by the checked build");
    return fail(FG_ERR_TIMEOUT, "device: bounded wait gave up (code " + std::to_string(code) + ")");
}

int fg_plan_create(const fg_problem* prob, const fg_tuning* tune, fg_plan** out) {
    if (!prob || !out) return fail(FG_ERR_INVALID, "fg_plan_create: NULL argument");
    *out = nullptr;
    const fg_problem& q = *prob;
    if (q.nx < 2 || q.ny < 2) return fail(FG_ERR_INVALID, "grid must be at least 2x2");
    if (q.shots < 1 || q.nt < 1) return fail(FG_ERR_INVALID, "shots and nt must be >= 1");
    if (q.th < 0 || 2 * q.th > std::min(q.nx, q.ny)) return fail(FG_ERR_INVALID, "CPML thickness out of range");
    if (q.nsrc < 0 || q.nrx < 0) return fail(FG_ERR_INVALID, "negative source/receiver count");
    if ((q.nsrc > 0 && (!q.src || !q.srcw)) || (q.nrx > 0 && !q.rx)) return fail(FG_ERR_INVALID, "missing tables");
    if (q.th > 0 && !q.pml) return fail(FG_ERR_INVALID, "missing CPML coefficients");
    if (!(q.dx > 0.f) || !(q.dt > 0.f)) return fail(FG_ERR_INVALID, "dx and dt must be positive");
    fg_plan* p = new fg_plan();
    p->nx = q.nx; p->ny = q.ny; p->S = q.shots; p->nt = q.nt; p->th = q.th;
    p->nsrc = q.nsrc; p->nrx = q.nrx; p->dx = q.dx; p->dt = q.dt;
    p->src.assign(q.src, q.src + (size_t)q.shots * q.nsrc * 3);
    p->rx.assign(q.rx, q.rx + (size_t)q.shots * q.nrx * 3);
    p->srcw.assign(q.srcw, q.srcw + (size_t)q.nsrc * q.nt);
    if (q.th > 0) p->pml.assign(q.pml, q.pml + 8 * (size_t)q.th);
    for (size_t k = 0; k + 2 < p->src.size(); k += 3)
        if (classify(p, p->src[k], p->src[k + 1], p->src[k + 2]) < 0) {
            delete p;
            return fail(FG_ERR_INVALID, "source position outside the grid");
        }
    for (size_t k = 0; k + 2 < p->rx.size(); k += 3)
        if (classify(p, p->rx[k], p->rx[k + 1], p->rx[k + 2]) < 0) {
            delete p;
            return fail(FG_ERR_INVALID, "receiver position outside the grid");
        }
    p->kernel = tune ? tune->kernel : 3;
    p->V = tune && tune->cols_per_thread ? tune->cols_per_thread : (p->kernel >= 2 ? 2 : 1);
    p->G = tune && tune->shots_per_tile ? tune->shots_per_tile
                                        : (p->kernel >= 2 ? std::min(q.shots, 4) : (q.shots >= 2 ? 2 : 1));
    p->TI = tune && tune->rows_per_tile ? tune->rows_per_tile : (p->kernel == 2 ? 8 : 16);
    p->NW = tune && tune->warps_per_tile ? tune->warps_per_tile : 0;
    p->D = tune && tune->stages ? tune->stages : 4;
    if (p->kernel == 0 && p->NW == 0) {
        // default: one band covering the row when it fits in 16 warps
        p->NW = std::min(16, std::max(1, (q.ny + 32 * p->V - 1) / (32 * p->V)));
    }
    const bool ok_common = (p->V == 1 || p->V == 2 || p->V == 4) && p->TI >= 2;
    const bool ok_k0 = p->kernel == 0 && (p->G == 1 || p->G == 2 || p->G == 4) && p->NW >= 1 && p->NW <= 16 &&
                       p->D >= 3 && p->D <= 8;
    const bool ok_k1 = p->kernel == 1 && (p->G == 1 || p->G == 2 || p->G == 4 || p->G == 8);
    const bool ok_k2 = p->kernel == 2 && p->G >= 1 && p->G <= 64 && p->TI <= 16;
    const bool ok_k3 = p->kernel == 3 && p->G >= 1 && p->G <= 64 &&
                       fg::march_adj_smem(p->TI, p->V) <= 227 * 1024;
    if (!ok_common || !(ok_k0 || ok_k1 || ok_k2 || ok_k3)) {
        delete p;
        return fail(FG_ERR_INVALID, "unsupported tuning");
    }
    // The row-streaming tiles keep one x-slab auxiliary row per stage; with
    // 2*th >= nx a row lies in both x-slabs and the register march is used.
    if (p->kernel == 0 && 2 * q.th >= q.nx) {
        p->kernel = 1;
        if (p->G > 8) p->G = 8;
    }
    if (p->kernel == 0) {
        const int TY = (int)align_up((size_t)std::max(q.th, 1), 4);
        const size_t smem = fg::ring_smem_bytes(p->D, 5 + 8 * p->G, fg::ring_slot_width(p->NW * 32 * p->V, TY), q.th);
        if (smem > 227 * 1024) {
            delete p;
            return fail(FG_ERR_INVALID, "tuning needs more than 227 KB of shared memory");
        }
    }
    build_tiles(p);
    layout(p);
    *out = p;
    return FG_OK;
}

int fg_plan_destroy(fg_plan* plan) {
    delete plan;
    return FG_OK;
}

int64_t fg_plan_workspace_bytes(const fg_plan* plan) { return plan ? (int64_t)plan->total : -1; }

int32_t fg_plan_hist_pitch(const fg_plan* plan) { return plan ? plan->Ph : -1; }

int fg_plan_bind(fg_plan* p, void* workspace, int64_t bytes, void* stream) {
    if (!p) return fail(FG_ERR_INVALID, "fg_plan_bind: NULL plan");
    if (!workspace || bytes < (int64_t)p->total) return fail(FG_ERR_WORKSPACE, "workspace missing or too small");
    if (((uintptr_t)workspace) % 256) return fail(FG_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    p->ws = (char*)workspace;
    p->ws_bytes = bytes;
    fill_grid(p);
    auto up = [&](size_t off, const void* src, size_t n) -> cudaError_t {
        if (n == 0) return cudaSuccess;
        return cudaMemcpyAsync(p->ws + off, src, n, cudaMemcpyHostToDevice, st);
    };
    FG_CUDA(up(p->o_chunk, p->chunk_row.data(), p->chunk_row.size() * sizeof(int)));
    FG_CUDA(up(p->o_srcev, p->src_ev.data(), p->src_ev.size() * sizeof(Ev)));
    FG_CUDA(up(p->o_rxev, p->rx_ev.data(), p->rx_ev.size() * sizeof(Ev)));
    FG_CUDA(up(p->o_injev, p->inj_ev.data(), p->inj_ev.size() * sizeof(Ev)));
    FG_CUDA(up(p->o_injhev, p->injh_ev.data(), p->injh_ev.size() * sizeof(Ev)));
    std::vector<int> offs;
    offs.insert(offs.end(), p->src_off.begin(), p->src_off.end());
    offs.insert(offs.end(), p->rx_off.begin(), p->rx_off.end());
    offs.insert(offs.end(), p->inj_off.begin(), p->inj_off.end());
    offs.insert(offs.end(), p->injh_off.begin(), p->injh_off.end());
    FG_CUDA(up(p->o_offs, offs.data(), offs.size() * sizeof(int)));
    FG_CUDA(up(p->o_srcw, p->srcw.data(), p->srcw.size() * sizeof(float)));
    FG_CUDA(up(p->o_pml, p->pml.data(), p->pml.size() * sizeof(float)));
    FG_CUDA(cudaMemsetAsync(p->ws + p->o_err, 0, sizeof(int) * 4, st));
    // the host tables must stay valid until the copies have been consumed
    FG_CUDA(cudaStreamSynchronize(st));
    return FG_OK;
}

int fg_coefficients(const float* er, const float* se, const float* mr, int32_t nx, int32_t ny, float dt, float dx,
                    int32_t adjoint, float* out, int32_t pitch, void* stream) {
    if (!er || !se || !mr || !out) return fail(FG_ERR_INVALID, "fg_coefficients: NULL argument");
    if (nx < 1 || ny < 1 || pitch < ny + 1) return fail(FG_ERR_INVALID, "fg_coefficients: bad shape");
    return coefficients(er, se, mr, nx, ny, dt, dx, adjoint, out, pitch, (cudaStream_t)stream);
}

int fg_forward(fg_plan* p, const float* er, const float* se, const float* mr, float* traces, float* hist,
               void* stream) {
    if (!p || !er || !se || !mr || (!traces && p->nrx > 0)) return fail(FG_ERR_INVALID, "fg_forward: NULL argument");
    if (!p->ws) return fail(FG_ERR_WORKSPACE, "fg_forward: plan has no workspace");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = coefficients(er, se, mr, p->nx, p->ny, p->dt, p->dx, 0, (float*)(p->ws + p->o_coef), p->P, st);
    if (rc) return rc;
    if ((rc = reset_state(p, st))) return rc;
    if (p->nrx > 0) FG_CUDA(cudaMemsetAsync(traces, 0, (size_t)p->S * p->nt * p->nrx * sizeof(float), st));
    GridDev g = p->g;
    g.traces = traces;
    g.hist = hist;
    if (hist) {
        g.out_lo = (const char*)hist;
        g.out_hi = (const char*)(hist + (size_t)p->nt * p->S * p->nx * p->Ph);
    }
    if (p->kernel == 3) {
        FwdTileFn fn = pick_fwd_march(p->V);
        if (!fn) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        for (int t = 0; t < p->nt; ++t) FG_CUDA(fn(g, t, p->TI, p->G, st));
    } else if (p->kernel == 2) {
        FwdTileFn fn = pick_fwd_tile(p->V);
        if (!fn) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        for (int t = 0; t < p->nt; ++t) FG_CUDA(fn(g, t, p->TI, p->G, st));
    } else if (p->kernel == 0) {
        FwdTmaFn fn = pick_fwd_tma(p->V, p->G);
        if (!fn) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        for (int t = 0; t < p->nt; ++t) FG_CUDA(fn(g, t, p->NW, p->D, st));
    } else {
        FwdFn fn = pick_fwd(p->V, p->G);
        if (!fn) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        for (int t = 0; t < p->nt; ++t) fn(g, t, st);
    }
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

int fg_adjoint_reference(fg_plan* p, const float* er, const float* se, const float* mr, const float* hist,
                         const float* resid, float* grad_eps, float* grad_sig, int32_t normalize, double* norms,
                         void* stream) {
    if (!p || !er || !se || !mr || !hist || (!resid && p->nrx > 0))
        return fail(FG_ERR_INVALID, "fg_adjoint_reference: NULL argument");
    if (!p->ws) return fail(FG_ERR_WORKSPACE, "fg_adjoint_reference: plan has no workspace");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = coefficients(er, se, mr, p->nx, p->ny, p->dt, p->dx, 1, (float*)(p->ws + p->o_coef), p->P, st);
    if (rc) return rc;
    if ((rc = reset_state(p, st))) return rc;
    const size_t n = (size_t)p->nx * p->ny;
    FG_CUDA(cudaMemsetAsync(p->ws + p->o_gacc, 0, (size_t)p->ngroups * 2 * n * sizeof(double), st));
    GridDev g = p->g;
    g.hist = const_cast<float*>(hist);
    g.out_lo = (const char*)hist;
    g.out_hi = (const char*)(hist + (size_t)p->nt * p->S * p->nx * p->Ph);
    g.resid = resid;
    if (p->kernel == 3) {
        AdjTileFn fn = pick_adj_march(p->V);
        if (!fn) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        for (int it = p->nt - 1; it >= 1; --it) FG_CUDA(fn(g, it, (p->nt - 1 - it) & 1, p->TI, p->G, st));
    } else if (p->kernel == 2) {
        AdjTileFn fn = pick_adj_tile(p->V);
        if (!fn) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        for (int it = p->nt - 1; it >= 1; --it) FG_CUDA(fn(g, it, (p->nt - 1 - it) & 1, p->TI, p->G, st));
    } else if (p->kernel == 0) {
        AdjTmaFn fn = pick_adj_tma(p->V, p->G);
        if (!fn) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        for (int it = p->nt - 1; it >= 1; --it) FG_CUDA(fn(g, it, (p->nt - 1 - it) & 1, p->NW, p->D, st));
    } else {
        AdjFn fn = pick_adj(p->V, p->G);
        if (!fn) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        for (int it = p->nt - 1; it >= 1; --it) fn(g, it, (p->nt - 1 - it) & 1, st);
    }
    double* sums = (double*)(p->ws + p->o_sums);
    double* partial = (double*)(p->ws + p->o_partial);
    double* nrm = norms ? norms : (double*)(p->ws + p->o_norms);
    fg::k_grad_sum<<<kRedBlocks, 256, 0, st>>>(g.gacc, p->ngroups, (long long)n, sums, partial);
    fg::k_grad_norm<<<1, 32, 0, st>>>(partial, kRedBlocks, nrm);
    const int blocks = (int)((n + 255) / 256);
    fg::k_grad_scale<<<blocks, 256, 0, st>>>(sums, nrm, (long long)n, normalize, grad_eps, grad_sig);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

int fg_forward_static(fg_plan* p, const float* er, const float* se, const float* mr, float* traces, float* hist,
                      void* stream) {
    if (!p) return fail(FG_ERR_INVALID, "fg_forward_static: NULL plan");
    if (p->total > (size_t)FG_STATIC_SCRATCH_BYTES)
        return fail(FG_ERR_WORKSPACE, "fg_forward_static: the plan needs " + std::to_string(p->total) +
                                          " bytes of scratch, more than the static " +
                                          std::to_string((long long)FG_STATIC_SCRATCH_BYTES));
    void* scratch = nullptr;
    int rc = static_scratch(&scratch);
    if (rc) return rc;
    char* saved = p->ws;
    const int64_t saved_bytes = p->ws_bytes;
    rc = fg_plan_bind(p, scratch, (int64_t)FG_STATIC_SCRATCH_BYTES, stream);
    if (rc == FG_OK) rc = fg_forward(p, er, se, mr, traces, hist, stream);
    p->ws = saved;
    p->ws_bytes = saved_bytes;
    if (saved) fill_grid(p);
    return rc;
}

}  // extern "C"
