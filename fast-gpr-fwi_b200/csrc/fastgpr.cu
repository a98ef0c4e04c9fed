// libfastgpr: plan construction, workspace layout and the C ABI declared in
// include/fastgpr.h.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "../../include/fastgpr.h"
#include "plan.h"
#include "fdtd_setup.cuh"
#include "tv.cuh"
#include "fir.cuh"

using namespace fgk;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(FG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define FG_CUDA(call)                                       \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

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
    p->SL = p->pair ? 64 : (p->shot ? 32 : 1);
    p->CS = p->SL;
    p->BW = p->kernel == 2 ? p->WPB * p->W : (p->shot ? p->W : 32 * p->W);
    p->nb = (p->ny + p->BW - 1) / p->BW;
    // PADC leading zero columns, then columns up to nb*BW + 3 (halo column and
    // the 16-byte-aligned stage segments of the last band); rows of 16 bytes
    p->P = (int)align_up((size_t)p->nb * p->BW + 2 * fg::PADC, 4);
    p->TY = (int)align_up((size_t)std::max(p->th, 1), 4);
    p->Ph = (int)align_up((size_t)p->ny, 8);
    p->nc = std::max(1, (p->nx + p->TI - 1) / p->TI);
    p->ngroups = (p->S + p->SL - 1) / p->SL;
    p->ntiles = p->ngroups * p->nc * p->nb;
    p->chunk_row.resize(p->nc + 1);
    // tiles: chunks of exactly TI rows (the last one shorter); march: balanced chunks
    for (int c = 0; c <= p->nc; ++c)
        p->chunk_row[c] = p->kernel == 0 ? std::min(c * p->TI, p->nx) : (int)((long long)c * p->nx / p->nc);
    // events binned straight into their tiles (O(events), not O(tiles x events))
    const int bw = p->BW;
    std::vector<int> chunk_of_row(p->nx + 1, p->nc - 1);
    for (int c = 0; c < p->nc; ++c)
        for (int i = p->chunk_row[c]; i < p->chunk_row[c + 1]; ++i) chunk_of_row[i] = c;
    auto tile_id = [&](int grp, int chunk, int band) { return (grp * p->nc + chunk) * p->nb + band; };
    auto finish = [&](std::vector<std::vector<Ev>>& per, std::vector<Ev>& out, std::vector<int>& off) {
        out.clear();
        off.assign(p->ntiles + 1, 0);
        for (int t = 0; t < p->ntiles; ++t) {
            std::vector<Ev>& evs = per[t];
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
            if (p->srcw[(size_t)n * p->nt + t] != 0.f) {
                live[n] = 1;
                break;
            }
    auto pos = [&](const std::vector<int32_t>& tab, int count, int s, int n, int c) {
        return tab[((size_t)s * count + n) * 3 + c];
    };
    std::vector<std::vector<Ev>> src(p->ntiles), rxs(p->ntiles), inj(p->ntiles);
    for (int s = 0; s < p->S; ++s) {
        const int grp = s / p->SL, q = s % p->SL;
        for (int n = 0; n < p->nsrc; ++n) {
            if (!live[n]) continue;
            const int i = pos(p->src, p->nsrc, s, n, 0), j = pos(p->src, p->nsrc, s, n, 1), k = pos(p->src, p->nsrc, s, n, 2);
            if (classify(p, i, j, k) != 1) continue;
            src[tile_id(grp, chunk_of_row[i], j / bw)].push_back(make_int4(i, q, j, n));
        }
        for (int r = 0; r < p->nrx; ++r) {
            const int i = pos(p->rx, p->nrx, s, r, 0), j = pos(p->rx, p->nrx, s, r, 1), k = pos(p->rx, p->nrx, s, r, 2);
            if (classify(p, i, j, k) != 1) continue;
            const int c = chunk_of_row[i], b = j / bw;
            const Ev e = make_int4(i, q, j, r);
            rxs[tile_id(grp, c, b)].push_back(e);
            // adjoint injections: rows [i0, i1] and columns [b0, b0+bw] of a tile
            // (row i1 and column b0+bw are recomputed as halo cells), so a cell on
            // a tile's first row / first column also belongs to the tile above /
            // to the left
            inj[tile_id(grp, c, b)].push_back(e);
            const bool up = c > 0 && i == p->chunk_row[c];
            const bool left = b > 0 && j == b * bw;
            if (up) inj[tile_id(grp, c - 1, b)].push_back(e);
            if (left) inj[tile_id(grp, c, b - 1)].push_back(e);
            if (up && left) inj[tile_id(grp, c - 1, b - 1)].push_back(e);
        }
    }
    finish(src, p->src_ev, p->src_off);
    finish(rxs, p->rx_ev, p->rx_off);
    finish(inj, p->inj_ev, p->inj_off);
    // fetch order: tiles touching a CPML slab (more work per cell) first,
    // longest first -- a tile's cost is counted as one per cell plus one per
    // slab the cell lies in, ties put tiles in a y slab only first (their rows
    // cost more than x-slab rows), then (group, chunk, band) order -- and the
    // other tiles after them; with the interior split, the interior tiles (no
    // cell of the tile or of its halo in a CPML slab or on the first / last
    // rows and columns, no event) come last, from core0 on.  Longest first
    // shortens the tail of the persistent warps: 93.0 -> 90.3 us per adjoint
    // step on 440 x 340 with 64 shots.
    {
        const int th = p->th;
        auto heavy = [&](int t) {
            if (th == 0) return false;
            const int band = t % p->nb, chunk = (t / p->nb) % p->nc;
            const int i0 = p->chunk_row[chunk], i1 = p->chunk_row[chunk + 1];
            const int b0 = band * p->BW, b1 = b0 + p->BW;
            const bool xs = i0 <= th || i1 - 1 >= p->nx - th - 1;
            const bool ys = b0 <= th + 1 || b1 - 1 >= p->ny - th - 1;
            return xs || ys;
        };
        auto interior = [&](int t) {
            if (!p->split) return false;
            const int band = t % p->nb, chunk = (t / p->nb) % p->nc;
            const int i0 = p->chunk_row[chunk], i1 = p->chunk_row[chunk + 1];
            const int j0 = band * p->BW;
            const bool rows = i0 >= th + 1 && i1 <= p->nx - th - 1;
            const bool cols = j0 >= th + 1 && j0 + p->BW <= p->ny - th - 1;
            const bool quiet = p->src_off[t + 1] == p->src_off[t] && p->rx_off[t + 1] == p->rx_off[t] &&
                               p->inj_off[t + 1] == p->inj_off[t];
            return rows && cols && quiet;
        };
        // slab tiles (split plans with shot lanes): no event, and either the
        // interior's columns with rows touching an x slab (x tiles) or the
        // interior's rows with columns touching one y slab only, in the grid
        // (y tiles); they run in the slab kernel, between the general tiles
        // and the interior ones
        const bool fast = th > 0 && 2 * th < p->nx && 2 * th < p->ny;
        auto slab = [&](int t) -> int {
            if (!p->slab_on || !fast || interior(t)) return 0;
            const int band = t % p->nb, chunk = (t / p->nb) % p->nc;
            const int i0 = p->chunk_row[chunk], i1 = p->chunk_row[chunk + 1];
            const int j0 = band * p->BW, j1 = j0 + p->BW;
            const bool quiet = p->src_off[t + 1] == p->src_off[t] && p->rx_off[t + 1] == p->rx_off[t] &&
                               p->inj_off[t + 1] == p->inj_off[t];
            if (!quiet) return 0;
            const bool rows_in = i0 >= th + 1 && i1 <= p->nx - th - 1;
            const bool cols_in = j0 >= th + 1 && j1 <= p->ny - th - 1;
            if (cols_in) return 1;
            // the forward's H cells start at j0-1, the adjoint's E cells end at j0+W
            const bool one_side = !(j0 - 1 <= th && j1 >= p->ny - th);
            if (rows_in && j1 <= p->ny && one_side) return 2;
            return 0;
        };
        auto cost = [&](int t, bool* y_only) {
            const int band = t % p->nb, chunk = (t / p->nb) % p->nc;
            const int i0 = p->chunk_row[chunk], i1 = p->chunk_row[chunk + 1];
            const int b0 = band * p->BW, b1 = std::min(b0 + p->BW, p->ny);
            int c = 0;
            bool xany = false, yany = false;
            for (int i = i0; i < i1; ++i)
                for (int j = b0; j < b1; ++j) {
                    const bool xs = i <= th || i >= p->nx - th;
                    const bool ys = j <= th || j >= p->ny - th;
                    c += 1 + (xs ? 1 : 0) + (ys ? 1 : 0);
                    xany |= xs;
                    yany |= ys;
                }
            *y_only = yany && !xany;
            return c;
        };
        p->order.clear();
        {
            struct Key {
                int t, c;
                bool y;
            };
            std::vector<Key> h;
            for (int t = 0; t < p->ntiles; ++t)
                if (heavy(t) && !interior(t) && !slab(t)) {
                    Key k{t, 0, false};
                    k.c = cost(t, &k.y);
                    h.push_back(k);
                }
            std::stable_sort(h.begin(), h.end(),
                             [](const Key& a, const Key& b) { return a.c > b.c || (a.c == b.c && a.y && !b.y); });
            for (const Key& k : h) p->order.push_back(k.t);
        }
        for (int t = 0; t < p->ntiles; ++t)
            if (!heavy(t) && !interior(t) && !slab(t)) p->order.push_back(t);
        p->slab0 = (int)p->order.size();
        for (int t = 0; t < p->ntiles; ++t)
            if (slab(t) == 1) p->order.push_back(t);
        p->yslab0 = (int)p->order.size();
        for (int t = 0; t < p->ntiles; ++t)
            if (slab(t) == 2) p->order.push_back(t);
        p->core0 = (int)p->order.size();
        for (int t = 0; t < p->ntiles; ++t)
            if (interior(t)) p->order.push_back(t);
        p->tiles.resize(p->ntiles);
        for (int q = 0; q < p->ntiles; ++q) {
            const int t = p->order[q];
            const int band = t % p->nb, chunk = (t / p->nb) % p->nc, grp = t / (p->nb * p->nc);
            p->tiles[q] = make_int4(band * p->BW, p->chunk_row[chunk], grp, t);
        }
    }
}

void layout(fg_plan* p) {
    const size_t A = 256;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o = align_up(o + std::max<size_t>(bytes, 1), A);
        return at;
    };
    const long long cplane = (long long)(p->nx + 1) * p->P;
    p->plane = cplane * p->CS;
    p->pxs = 2LL * p->th * p->P * p->CS;
    p->pys = 2LL * (p->nx + 1) * p->TY * p->CS;
    p->o_coef = take(5 * (size_t)cplane * sizeof(float));
    p->state_bytes = 6 * (size_t)p->ngroups * p->plane * sizeof(float);
    p->psi_bytes = 4 * (size_t)p->ngroups * (p->pxs + p->pys) * sizeof(float);
    p->o_state = take(p->state_bytes);
    p->o_psi = take(p->psi_bytes);
    p->o_chunk = take((p->nc + 1) * sizeof(int));
    p->o_order = take((size_t)p->ntiles * sizeof(int));
    p->o_tiles = take((size_t)p->ntiles * sizeof(int4));
    p->o_ctr = take(8 * sizeof(int));
    p->o_srcev = take(p->src_ev.size() * sizeof(Ev));
    p->o_rxev = take(p->rx_ev.size() * sizeof(Ev));
    p->o_injev = take(p->inj_ev.size() * sizeof(Ev));
    p->o_offs = take(3 * (size_t)(p->ntiles + 1) * sizeof(int));
    p->o_srcw = take((size_t)p->nsrc * p->nt * sizeof(float));
    p->o_pml = take(8 * (size_t)p->th * sizeof(float));
    const size_t n = (size_t)p->nx * p->ny;
    p->o_gacc = take((size_t)p->ngroups * 2 * n * sizeof(double));
    p->o_sums = take(2 * n * sizeof(double));
    p->o_partial = take(2 * kRedBlocks * sizeof(double));
    p->o_norms = take(2 * sizeof(double));
    p->o_err = take(sizeof(int) * 4);
    p->o_rxpos = take((size_t)p->S * p->nrx * sizeof(int2));
    p->o_bar = take(4 * sizeof(unsigned));
    p->total = o;
}

void fill_grid(fg_plan* p) {
    Dev& g = p->g;
    std::memset(&g, 0, sizeof(g));
    char* w = p->ws;
    g.nx = p->nx; g.ny = p->ny; g.P = p->P; g.th = p->th; g.TY = p->TY;
    g.S = p->S; g.nt = p->nt; g.nrx = p->nrx; g.Ph = p->Ph; g.ngroups = p->ngroups;
    g.d = p->dx; g.dt = p->dt; g.dinv = p->dinv; g.div_scaled = p->div_scaled;
    g.plane = p->plane; g.pxs = p->pxs; g.pys = p->pys;
    const long long cplane = (long long)(p->nx + 1) * p->P;
    float* coef = (float*)(w + p->o_coef);
    g.ca = coef; g.cb = coef + cplane; g.cd = coef + 2 * cplane; g.ch = coef + 3 * cplane;
    g.ci = coef + 4 * cplane;
    g.pml = (const float*)(w + p->o_pml);
    float* st = (float*)(w + p->o_state);
    const long long sp = (long long)p->ngroups * p->plane;
    g.ez[0] = st; g.ez[1] = st + sp; g.hx[0] = st + 2 * sp; g.hx[1] = st + 3 * sp;
    g.hy[0] = st + 4 * sp; g.hy[1] = st + 5 * sp;
    float* ps = (float*)(w + p->o_psi);
    const long long xs = (long long)p->ngroups * p->pxs, ys = (long long)p->ngroups * p->pys;
    g.pex[0] = ps; g.pex[1] = ps + xs; g.phx[0] = ps + 2 * xs; g.phx[1] = ps + 3 * xs;
    float* py = ps + 4 * xs;
    g.pey[0] = py; g.pey[1] = py + ys; g.phy[0] = py + 2 * ys; g.phy[1] = py + 3 * ys;
    g.nb = p->nb; g.nc = p->nc; g.ntiles = p->ntiles;
    g.chunk_row = (const int*)(w + p->o_chunk);
    g.order = (const int*)(w + p->o_order);
    g.tiles = (const int4*)(w + p->o_tiles);
    g.tile_ctr = (int*)(w + p->o_ctr);
    g.fast_cpml = 2 * p->th < p->nx && 2 * p->th < p->ny;
    // shot lanes with no band whose cells (columns j0-1 .. j0+W) reach both y slabs
    g.lean = p->shot && !p->pair && g.fast_cpml;
    for (int b = 0; b < p->nb && g.lean; ++b) {
        const int j0 = b * p->BW, j1 = j0 + p->BW;
        if (p->th > 0 && j0 - 1 <= p->th && j1 >= p->ny - p->th) g.lean = 0;
    }
    g.pf = p->pf;
    g.core0 = p->core0;
    g.slab0 = p->slab0;
    g.yslab0 = p->yslab0;
    g.src_ev = (const Ev*)(w + p->o_srcev);
    g.rx_ev = (const Ev*)(w + p->o_rxev);
    g.inj_ev = (const Ev*)(w + p->o_injev);
    const int* offs = (const int*)(w + p->o_offs);
    g.src_off = offs; g.rx_off = offs + (p->ntiles + 1); g.inj_off = offs + 2 * (p->ntiles + 1);
    g.srcw = (const float*)(w + p->o_srcw);
    g.gacc = (double*)(w + p->o_gacc);
    g.ws_lo = w;
    g.ws_hi = w + p->total;
    g.err = (int*)(w + p->o_err);
}

int coefficients(const float* er, const float* se, const float* mr, int nx, int ny, float dt, float dx, int adjoint,
                 float* out, int P, int col0, cudaStream_t st) {
    const long long n = (long long)(nx + 1) * P;
    const int threads = 256;
    const long long blocks = (n + threads - 1) / threads;
    fg::k_coefficients<<<(unsigned)blocks, threads, 0, st>>>(er, se, mr, nx, ny, dt, dx, adjoint, out, P, col0);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

// Zero fields, auxiliaries and the tile counters before a solve.
int reset_state(fg_plan* p, cudaStream_t st) {
    FG_CUDA(cudaMemsetAsync(p->ws + p->o_state, 0, p->state_bytes, st));
    FG_CUDA(cudaMemsetAsync(p->ws + p->o_psi, 0, p->psi_bytes, st));
    FG_CUDA(cudaMemsetAsync(p->ws + p->o_ctr, 0, 8 * sizeof(int), st));
    return FG_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    });
    return fn;
}

// A float32 tensor map over `base`: dims[0] fastest, strides in bytes of
// dims 1.., box in elements; out-of-range elements of a box read as zero.
int encode_map(CUtensorMap* m, const void* base, int rank, const uint64_t* dims, const uint64_t* strides,
               const uint32_t* box) {
    auto fn = tensor_map_encoder();
    if (!fn) return fail(FG_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    cuuint64_t d[5], st[4];
    cuuint32_t b[5], es[5];
    for (int k = 0; k < rank; ++k) {
        d[k] = dims[k];
        b[k] = box[k];
        es[k] = 1;
        if (k + 1 < rank) st[k] = strides[k];
    }
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (cuuint32_t)rank, const_cast<void*>(base), d, st, b, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(FG_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return FG_OK;
}

// State box of `cells` columns and `rows` rows over all six field buffers
// (Ez, Hx, Hy x parity), one group.
int encode_state_map(const fg_plan* p, CUtensorMap* m, int cells, int rows) {
    const void* base = p->ws + p->o_state;
    const uint64_t f4 = sizeof(float);
    if (p->shot) {
        const uint64_t dims[5] = {32, (uint64_t)p->P, (uint64_t)p->nx + 1, (uint64_t)p->ngroups, 6};
        const uint64_t st[4] = {32 * f4, (uint64_t)p->P * 32 * f4, (uint64_t)p->plane * f4,
                                (uint64_t)p->ngroups * p->plane * f4};
        const uint32_t box[5] = {32, (uint32_t)cells, (uint32_t)rows, 1, 1};
        return encode_map(m, base, 5, dims, st, box);
    }
    const uint64_t dims[4] = {(uint64_t)p->P, (uint64_t)p->nx + 1, (uint64_t)p->ngroups, 6};
    const uint64_t st[3] = {(uint64_t)p->P * f4, (uint64_t)p->plane * f4, (uint64_t)p->ngroups * p->plane * f4};
    const uint32_t box[4] = {(uint32_t)cells, (uint32_t)rows, 1, 1};
    return encode_map(m, base, 4, dims, st, box);
}

int encode_tile_maps(fg_plan* p) {
    const int R = p->TI, W = p->W;
    const int BW = p->BW, NW = BW + 8;
    const bool sh = p->shot;
    int rc = FG_OK;
    if ((rc = encode_state_map(p, &p->tm_fez, sh ? W + 2 : NW, R + 2))) return rc;
    if ((rc = encode_state_map(p, &p->tm_fhx, sh ? W + 1 : NW, R))) return rc;
    if ((rc = encode_state_map(p, &p->tm_fhy, sh ? W : NW, R + 1))) return rc;
    if ((rc = encode_state_map(p, &p->tm_aez, sh ? W + 1 : NW, R + 1))) return rc;
    if ((rc = encode_state_map(p, &p->tm_ahx, sh ? W + 2 : NW, R + 1))) return rc;
    if ((rc = encode_state_map(p, &p->tm_ahy, sh ? W + 1 : NW, R + 2))) return rc;
    const uint64_t f4 = sizeof(float);
    const uint64_t dims[3] = {(uint64_t)p->P, (uint64_t)p->nx + 1, 5};
    const uint64_t st[2] = {(uint64_t)p->P * f4, (uint64_t)(p->nx + 1) * p->P * f4};
    const uint32_t box[3] = {(uint32_t)(BW + 8), (uint32_t)R + 1, 5};
    return encode_map(&p->tm_co, p->ws + p->o_coef, 3, dims, st, box);
}

// Box over the Ez history: W (shot lanes, all 32 slots) or BW (column lanes)
// columns of R rows of one (step, group).
int encode_hist_map(const fg_plan* p, CUtensorMap* m, const float* hist, int nsteps) {
    const uint64_t f4 = sizeof(float);
    const uint64_t steps = (uint64_t)nsteps * p->ngroups;
    if (p->shot) {
        const uint64_t dims[4] = {32, (uint64_t)p->Ph, (uint64_t)p->nx, steps};
        const uint64_t st[3] = {32 * f4, (uint64_t)p->Ph * 32 * f4, (uint64_t)p->nx * p->Ph * 32 * f4};
        const uint32_t box[4] = {32, (uint32_t)p->W, (uint32_t)p->TI, 1};
        return encode_map(m, hist, 4, dims, st, box);
    }
    const uint64_t dims[3] = {(uint64_t)p->Ph, (uint64_t)p->nx, steps};
    const uint64_t st[2] = {(uint64_t)p->Ph * f4, (uint64_t)p->nx * p->Ph * f4};
    const uint32_t box[3] = {(uint32_t)p->BW, (uint32_t)p->TI, 1};
    return encode_map(m, hist, 3, dims, st, box);
}

// Device scratch of fg_forward_static: one array per GPU that loads the
// library, held until the process exits.  Host code must not pass the
// symbol itself to a kernel (on the host it names a host-side shadow); the
// device address comes from cudaGetSymbolAddress, looked up once per device.
static __device__ __align__(256) unsigned char g_static_scratch[FG_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
void* g_static_ptr[kMaxDevices] = {};
// which plan's tables the array of each device holds (0: none), and the
// division checks of that bind
struct StaticOwner {
    uint64_t plan = 0;
    float dinv = 0.f;
    int div_scaled = 0;
};
StaticOwner g_static_owner[kMaxDevices];
std::atomic<uint64_t> g_next_plan_id{1};

int static_scratch(void** out, int* device) {
    int dev = 0;
    FG_CUDA(cudaGetDevice(&dev));
    *device = dev;
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

// ---------------------------------------------------------------------------
// Total-variation regulariser
// ---------------------------------------------------------------------------
namespace {
constexpr int kTvMaxBlocks = 4096;
struct TvLayout {
    size_t arr, partial, pmax, words, total;
    TvLayout(int M, int N) {
        const size_t A = 256, cells = (size_t)(M + 2) * (N + 2);
        arr = align_up(cells * sizeof(float), A);
        partial = 7 * arr;
        pmax = partial + align_up(2 * kTvMaxBlocks * sizeof(double), A);
        words = pmax + align_up(kTvMaxBlocks * sizeof(float), A);
        total = words + A;
    }
};
}  // namespace

int fg_fir_causal(const float* x, int64_t batch, int32_t T, int32_t R, const float* taps, int32_t k, float* out,
                  void* stream) {
    if (batch < 0 || T < 1 || R < 1) return fail(FG_ERR_INVALID, "fg_fir_causal: bad shape");
    if (k < 1 || k > fg::FIR_MAX_TAPS) return fail(FG_ERR_INVALID, "fg_fir_causal: taps must number 1.." +
                                                                       std::to_string(fg::FIR_MAX_TAPS));
    if (k - 1 >= T) return fail(FG_ERR_INVALID, "fg_fir_causal: the reflect padding (taps - 1) must be shorter "
                                                "than the series");
    if (batch == 0) return FG_OK;
    if (!x || !out || !taps) return fail(FG_ERR_INVALID, "fg_fir_causal: NULL argument");
    const size_t bytes = (size_t)batch * T * R * sizeof(float);
    if ((const char*)out < (const char*)x + bytes && (const char*)x < (const char*)out + bytes)
        return fail(FG_ERR_INVALID, "fg_fir_causal: out overlaps x");
    int dev = 0, sms = 0;
    FG_CUDA(cudaGetDevice(&dev));
    FG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long long n = batch * (long long)T * R;
    const long long blocks = std::max<long long>(1, std::min<long long>((n + fg::FIR_THREADS - 1) / fg::FIR_THREADS,
                                                                        (long long)sms * 8));
    fg::k_fir_causal<<<(unsigned)blocks, fg::FIR_THREADS, 0, (cudaStream_t)stream>>>(x, batch, T, R, taps, k, out);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

int64_t fg_tv_workspace_bytes(int32_t M, int32_t N) {
    if (M < 1 || N < 1) return -1;
    return (int64_t)TvLayout(M, N).total;
}

int fg_total_variation(const float* data, int32_t M, int32_t N, double lamda, double rho, int32_t num_iter,
                       double tol, float* out, void* workspace, int64_t bytes, int32_t* iters, void* stream) {
    if (!data || !out) return fail(FG_ERR_INVALID, "fg_total_variation: NULL argument");
    if (M < 1 || N < 1 || num_iter < 0) return fail(FG_ERR_INVALID, "fg_total_variation: bad shape or iteration count");
    if (!(rho != 0.0)) return fail(FG_ERR_INVALID, "fg_total_variation: rho must be non-zero");
    const TvLayout L(M, N);
    if (!workspace || bytes < (int64_t)L.total) return fail(FG_ERR_WORKSPACE, "fg_total_variation: workspace too small");
    if (((uintptr_t)workspace) % 256) return fail(FG_ERR_WORKSPACE, "fg_total_variation: workspace not 256-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0, sms = 0, per_sm = 0, coop = 0;
    FG_CUDA(cudaGetDevice(&dev));
    FG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    FG_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) return fail(FG_ERR_CUDA, "fg_total_variation: device without cooperative launch");
    FG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fg::k_total_variation, fg::TV_THREADS, 0));
    const long long cells = (long long)(M + 2) * (N + 2);
    // one CTA per SM at most (cheap barriers), fewer for small models
    long long blocks = std::min<long long>((cells + fg::TV_THREADS * 4 - 1) / (fg::TV_THREADS * 4), sms);
    blocks = std::max<long long>(1, std::min<long long>(blocks, (long long)per_sm * sms));
    blocks = std::min<long long>(blocks, kTvMaxBlocks);
    char* w = (char*)workspace;
    fg::TvArgs a;
    a.data = data;
    a.out = out;
    a.M = M;
    a.N = N;
    // scalars as float32 tensor arithmetic sees them: products in double, then rounded
    a.lam = (float)lamda;
    a.lr = (float)(lamda * rho);
    a.rho = (float)rho;
    a.inv_rho = (float)(1.0 / rho);
    a.den = (float)(1.0 + 4.0 * lamda * rho);
    a.num_iter = num_iter;
    a.tol = (double)(float)tol;
    float* arr[7];
    for (int k = 0; k < 7; ++k) arr[k] = (float*)(w + k * L.arr);
    a.x0 = arr[0]; a.x1 = arr[1]; a.y = arr[2]; a.zx = arr[3]; a.zy = arr[4]; a.ux = arr[5]; a.uy = arr[6];
    a.partial = (double*)(w + L.partial);
    a.pmax = (float*)(w + L.pmax);
    a.bar = (unsigned*)(w + L.words);
    a.err = (int*)(w + L.words + 8);
    a.iters = (int*)(w + L.words + 12);
    FG_CUDA(cudaMemsetAsync(w + L.words, 0, 16, st));
    void* args[] = {&a};
    FG_CUDA(cudaLaunchCooperativeKernel((const void*)fg::k_total_variation, dim3((unsigned)blocks),
                                        dim3(fg::TV_THREADS), args, 0, st));
    if (!iters) return FG_OK;   // enqueue only (capturable): the status words stay in the workspace
    int words[2] = {0, 0};
    FG_CUDA(cudaMemcpyAsync(words, w + L.words + 8, sizeof(words), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    if (words[0] != 0) return fail(FG_ERR_TIMEOUT, "fg_total_variation: a grid barrier gave up");
    *iters = words[1];
    return FG_OK;
}

int fg_plan_check(fg_plan* p, void* stream) {
    if (!p || !p->ws) return fail(FG_ERR_INVALID, "fg_plan_check: plan has no workspace");
    cudaStream_t st = (cudaStream_t)stream;
    fg_plan* plans[2] = {p, p->adj};
    int code[2] = {0, 0};
    for (int k = 0; k < 2; ++k)
        if (plans[k] && plans[k]->ws)
            FG_CUDA(cudaMemcpyAsync(&code[k], plans[k]->ws + plans[k]->o_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    int c = 0;
    for (int k = 0; k < 2; ++k)
        if (code[k]) {
            FG_CUDA(cudaMemsetAsync(plans[k]->ws + plans[k]->o_err, 0, sizeof(int), st));
            if (!c) c = code[k];
        }
    if (c == 0) return FG_OK;
    if (c == 100) return fail(FG_ERR_INVALID, "device: out-of-range access caught by the checked build");
    return fail(FG_ERR_TIMEOUT, "device: bounded wait gave up (code " + std::to_string(c) + ")");
}

// One plan: the problem's tables and one launch shape.
static int create_one(const fg_problem* prob, const fg_tuning* tune, fg_plan** out) {
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
    p->id = g_next_plan_id.fetch_add(1);
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
    const int lanes = tune ? tune->lanes : 0;
    if (lanes < 0 || lanes > 3) {
        delete p;
        return fail(FG_ERR_INVALID, "unsupported tuning: lanes must be 0, 1, 2 or 3");
    }
    p->pair = lanes == 3;
    p->shot = p->pair || lanes == 1 || (lanes == 0 && q.shots >= 8);
    // defaults: the fastest measured shapes on the 440 x 340 benchmark grid --
    // lane march (4 cells x 4 rows) for shot lanes, tile pipeline (2 cells x 4
    // rows) for column lanes
    const bool tuned_kernel = tune && (tune->kernel || tune->stages || tune->rows_per_tile || tune->cells_per_thread);
    // the whole time loop in one persistent launch (fdtd_multi.cuh) only when
    // asked for: measured on the 140 x 100 one-shot and 240 x 160 13-shot
    // grids it is no faster than a launch per step (a step's time is the
    // serial latency of a warp's tile, which the launch does not change)
    const int persistent = tune ? tune->persistent : 0;
    if (persistent < -1 || persistent > 1) {
        delete p;
        return fail(FG_ERR_INVALID, "unsupported tuning: persistent must be -1, 0 or 1");
    }
    p->kernel = tuned_kernel ? tune->kernel : ((p->shot || persistent == 1) ? 1 : 0);
    if (p->kernel < 0 || p->kernel > 2) {
        delete p;
        return fail(FG_ERR_INVALID, "unsupported tuning: kernel must be 0 (tiles), 1 (lane march) or 2 (band pipeline)");
    }
    p->W = tune && tune->cells_per_thread ? tune->cells_per_thread : (p->shot ? 4 : 2);
    // rows per tile: 4, but 2 for the shot-lane lane march on steps below
    // 1.2e5 cells x shot groups, where the general kernel holds only a few
    // hundred tiles, one per warp, and a tile's serial latency is the step's
    // (measured, us per forward step with 2 / 4 rows: 100 x 80, 8 shots 11.6 /
    // 18.1; 240 x 160, 13 shots 14.2 / 16.7; 296 x 296, 32 shots 22.5 / 27.5;
    // 440 x 340, 32 shots 36.9 / 34.8)
    const bool small_step = (long long)q.nx * q.ny * ((q.shots + 31) / 32) < 120000;
    p->TI = tune && tune->rows_per_tile
                ? tune->rows_per_tile
                : (p->kernel == 2 ? 32
                                  : (p->kernel == 1 && p->shot && !p->pair && !(tune && tune->stages) &&
                                             persistent != 1 && small_step
                                         ? 2
                                         : 4));
    p->WPB = tune && tune->warps_per_block ? tune->warps_per_block : (p->kernel == 0 ? std::min(p->TI, 4) : 4);
    p->D = tune ? tune->stages : 0;
    if (p->kernel == 0 && p->pair) {
        delete p;
        return fail(FG_ERR_INVALID, "unsupported tuning: shot pairs (lanes 3) take the lane march (kernel 1)");
    }
    if (p->kernel == 2) {
        if (p->D == 0) p->D = 6;   // ring stages of the band pipeline
        if (!p->shot || p->pair) {
            delete p;
            return fail(FG_ERR_INVALID, "unsupported tuning: the band pipeline (kernel 2) takes shot lanes");
        }
        if (!pick_fwd_band(p->W, p->WPB) || p->TI < 1 || p->D < 2 || p->D > 16) {
            delete p;
            return fail(FG_ERR_INVALID, "unsupported tuning: the band pipeline takes (cells_per_thread, "
                                        "warps_per_block) in (2,4) (2,8) (4,2) (4,4), "
                                        "rows_per_tile >= 1 and stages 2..16");
        }
        if (std::max(band_smem(p->W, p->WPB, p->th, p->D, false), band_smem(p->W, p->WPB, p->th, p->D, true)) >
            227 * 1024) {
            delete p;
            return fail(FG_ERR_INVALID, "unsupported tuning: the band pipeline's stages need more than 227 KB of "
                                        "shared memory");
        }
    } else if (p->kernel == 0) {
        if (p->D == 0) p->D = 3;   // pipeline stages of the tile kernels
        const bool okw = p->shot ? (p->W == 4 || p->W == 8) : (p->W == 2 || p->W == 4);
        if (!okw || !(p->TI == 2 || p->TI == 4 || p->TI == 8 || p->TI == 16) || p->D < 2 || p->D > fg::MAX_STAGES ||
            !(p->WPB == 1 || p->WPB == 2 || p->WPB == 4 || p->WPB == 8) || p->TI % p->WPB != 0) {
            delete p;
            return fail(FG_ERR_INVALID, "unsupported tuning: tiles take cells_per_thread 4/8 (shot lanes) or 2/4 "
                                        "(column lanes), rows_per_tile 2/4/8/16 split evenly over warps_per_block "
                                        "1/2/4/8 consumer warps, and stages 0 or 2..4");
        }
    } else {
        if (!(p->W == 2 || p->W == 4 || p->W == 8) || p->TI < 1 || !(p->WPB == 1 || p->WPB == 2 || p->WPB == 4) ||
            p->D < 0 || p->D == 1 || p->D > 8) {
            delete p;
            return fail(FG_ERR_INVALID, "unsupported tuning: cells_per_thread 2/4/8, rows_per_tile >= 1, "
                                        "warps_per_block 1/2/4, stages 0 or 2..8");
        }
        if (p->pair && (p->D != 0 || p->W > 4)) {
            delete p;
            return fail(FG_ERR_INVALID, "unsupported tuning: shot pairs take the lane march with cells_per_thread 2 "
                                        "or 4 and no stages");
        }
        // shot-lane stages copy coefficient rows from column j0-4: 16-byte aligned only for W >= 4
        if (p->D > 0 && p->shot && p->W < 4) {
            delete p;
            return fail(FG_ERR_INVALID, "unsupported tuning: shot lanes with stages need cells_per_thread 4 or 8");
        }
    }
    const int pf = tune ? tune->prefetch : 0;
    if (pf < -1 || pf > 2) {
        delete p;
        return fail(FG_ERR_INVALID, "unsupported tuning: prefetch must be -1, 0, 1 or 2");
    }
    // the next-tile prefetch serves the shot-lane lane march with direct loads;
    // the band pipeline prefetches the CPML auxiliaries of the rows it streams
    p->pf = ((p->kernel == 1 && p->shot && !p->pair && p->D == 0) || p->kernel == 2) ? (pf == 0 ? 1 : std::max(pf, 0))
                                                                                      : 0;
    // interior tiles in their own lean kernel (shot-lane lane march with direct loads)
    const int interior = tune ? tune->interior : 0;
    if (interior < -1 || interior > 8) {
        delete p;
        return fail(FG_ERR_INVALID, "unsupported tuning: interior must be -1 .. 8");
    }
    // by default wherever a step pays for the extra launches: at least 12,000
    // cells x shot groups (measured, us per forward / adjoint step with the
    // split against without: 140 x 100, 16 shots 15.3 / 24.5 against 19.5 /
    // 25.9; 440 x 340, 32 shots 34.5 / 60.2 against 48.4 / 73.9; 100 x 80,
    // 8 shots 19.3 against 18.0 forward), and not in a persistent plan, whose
    // one launch takes every tile
    const long long work = (long long)p->nx * p->ny * ((p->S + 31) / 32);
    p->split = p->kernel == 1 && p->shot && !p->pair && p->D == 0 && pick_fwd_core(p->W) &&
               (interior > 0 || (interior == 0 && work >= 12000 && persistent != 1));
    // measured on the 64-shot 440 x 340 benchmark grid: the general kernel is
    // fastest beside the interior kernel with 3 blocks per SM
    p->split_bpsm = interior > 0 ? interior : 3;
    const int slab = tune ? tune->slab : 0;
    if (slab < -1 || slab > 8) {
        delete p;
        return fail(FG_ERR_INVALID, "unsupported tuning: slab must be -1 .. 8");
    }
    // measured on the 64-shot 440 x 340 benchmark grid (us per step): the
    // forward's slab kernel at 2 blocks per SM beside the others 68.1 against
    // 75.3 without it (1: 88.9, 3: 77.7, as many as fit: 83.9); the
    // adjoint's (8 cells per thread) 109.3 against 98.5 without it, so
    // fg_plan_create turns it on for the adjoint plan on small steps only
    p->slab_on = p->split && slab != -1;
    p->slab_bpsm = slab > 0 ? slab : 2;
    // beside the interior kernel the general kernel's next-tile prefetch only
    // competes for bandwidth (measured on that grid: forward 74.0 against
    // 78.1 us, adjoint 99.2 against 101.9 us without it): off unless asked for
    if (p->split && pf == 0) p->pf = 0;
    p->persist = p->kernel == 1 && p->D == 0 && !p->pair && !p->split && persistent == 1;
    if (p->kernel == 1 && fg::prof_bytes(p->th) + plan_ring_smem(p) > 227 * 1024) {
        delete p;
        return fail(FG_ERR_INVALID, "unsupported tuning: the ring needs more than 227 KB of shared memory");
    }
    build_tiles(p);
    layout(p);
    if (p->kernel == 0 && plan_tile_smem(p) > 227 * 1024) {
        delete p;
        return fail(FG_ERR_INVALID, "unsupported tuning: a tile needs more than 227 KB of shared memory");
    }
    *out = p;
    return FG_OK;
}

int fg_plan_create(const fg_problem* prob, const fg_tuning* tune, fg_plan** out) {
    fg_plan* p = nullptr;
    int rc = create_one(prob, tune, &p);
    if (rc) return rc;
    // the adjoint's launch shape: the forward's when the caller gave one and no
    // adj_* field, else adj_* with defaults (shot lanes: lane march with 8
    // cells per thread over 4 rows -- the fastest measured adjoint on the
    // 440 x 340 benchmark grid, 119 us against 139 us for the tile pipeline)
    const bool tuned = tune && (tune->kernel || tune->stages || tune->rows_per_tile || tune->cells_per_thread);
    const int ak = tune ? tune->adj_kernel : 0;
    if (ak < 0 || ak > 3) {
        delete p;
        return fail(FG_ERR_INVALID,
                    "unsupported tuning: adj_kernel must be 0, 1 (tiles), 2 (lane march) or 3 (band pipeline)");
    }
    fg_tuning at = {};
    at.lanes = p->pair ? 3 : (p->shot ? 1 : 2);
    at.cells_per_thread = p->W;
    if (ak == 0 && (tuned || !p->shot || p->pair)) {
        at.kernel = p->kernel;
        at.rows_per_tile = p->TI;
        at.warps_per_block = p->WPB;
        at.stages = p->D;
    } else if (ak == 0) {
        // 8 cells per thread where the interior split runs (the 440 x 340
        // 64-shot grid), 4 on smaller steps (measured on 240 x 160, 13 shots:
        // 110 against 130 ms per adjoint)
        const long long work = (long long)prob->nx * prob->ny * ((prob->shots + 31) / 32);
        at.kernel = 1;
        at.cells_per_thread = work >= 200000 ? 8 : 4;
        at.rows_per_tile = tune && tune->adj_rows_per_tile ? tune->adj_rows_per_tile : 4;
        at.warps_per_block = tune && tune->adj_warps_per_block ? tune->adj_warps_per_block : 4;
        at.stages = tune && tune->adj_stages ? tune->adj_stages : 0;
    } else {
        at.kernel = ak == 3 ? 2 : (ak == 2 ? 1 : 0);
        at.rows_per_tile = tune && tune->adj_rows_per_tile ? tune->adj_rows_per_tile
                                                           : (at.kernel == 0 ? 8 : (at.kernel == 2 ? 32 : 4));
        at.warps_per_block = tune && tune->adj_warps_per_block ? tune->adj_warps_per_block
                                                               : (at.kernel == 0 ? std::min(at.rows_per_tile, 4) : 4);
        at.stages = tune && tune->adj_stages ? tune->adj_stages : (at.kernel == 0 ? 2 : (at.kernel == 2 ? 6 : 0));
        if (at.kernel == 2 && !(tune && tune->adj_cells_per_thread)) at.cells_per_thread = 4;
    }
    if (tune && tune->adj_cells_per_thread) at.cells_per_thread = tune->adj_cells_per_thread;
    at.prefetch = tune ? tune->prefetch : 0;
    at.interior = tune ? tune->interior : 0;
    at.persistent = tune ? tune->persistent : 0;
    // the adjoint's slab kernel (4 cells per thread) on small steps, where the
    // general kernel's CPML tiles are most of the work; measured, us per
    // adjoint step with 2 / 1 / 0 slab blocks per SM: 140 x 100, 16 shots
    // 18.2 / 18.2 / 24.5; 280 x 200, 13 shots 19.9 / 21.5 / 28.1; 296 x 296,
    // 32 shots 41.7 / 38.3 / 41.3; 440 x 340, 32 shots 78.2 / 63.0 / 60.2
    if (tune && tune->slab) {
        at.slab = tune->slab;
    } else {
        const long long work = (long long)prob->nx * prob->ny * ((prob->shots + 31) / 32);
        at.slab = work < 50000 ? 2 : (work < 120000 ? 1 : -1);
    }
    fg_plan* a = nullptr;
    rc = create_one(prob, &at, &a);
    if (rc) {
        delete p;
        return rc;
    }
    // the adjoint's general kernel beside its interior kernel: 3 blocks per SM by default (as many as its
    // 168 registers let one SM hold; a fourth block only starts as the others leave)
    if (!(tune && tune->interior)) a->split_bpsm = 3;
    p->adj = a;
    *out = p;
    return FG_OK;
}

int fg_plan_destroy(fg_plan* plan) {
    delete plan;
    return FG_OK;
}

namespace {
size_t own_bytes(const fg_plan* p) { return align_up(p->total, 256); }
}  // namespace

int64_t fg_plan_workspace_bytes(const fg_plan* plan) {
    if (!plan) return -1;
    return (int64_t)(own_bytes(plan) + (plan->adj ? plan->adj->total : 0));
}

int fg_plan_shape(const fg_plan* plan, int32_t* out) {
    if (!plan || !out) return fail(FG_ERR_INVALID, "fg_plan_shape: NULL argument");
    const fg_plan* ps[2] = {plan, plan->adj ? plan->adj : plan};
    for (int k = 0; k < 2; ++k) {
        const fg_plan* p = ps[k];
        int32_t* o = out + 9 * k;
        o[0] = p->kernel;
        o[1] = p->pair ? 3 : (p->shot ? 1 : 2);
        o[2] = p->W;
        o[3] = p->TI;
        o[4] = p->WPB;
        o[5] = p->D;
        o[6] = p->split ? 1 : 0;
        o[7] = p->slab_on ? p->slab_bpsm : 0;
        o[8] = p->persist ? 1 : 0;
    }
    return FG_OK;
}

int fg_plan_hist_shape(const fg_plan* p, int64_t shape[5]) {
    if (!p || !shape) return fail(FG_ERR_INVALID, "fg_plan_hist_shape: NULL argument");
    shape[0] = p->nt;
    shape[1] = p->ngroups;
    shape[2] = p->nx;
    shape[3] = p->Ph;
    shape[4] = p->CS;
    return FG_OK;
}

// The division checks depend only on the divisor (and the device's
// arithmetic), so each (device, divisor) is checked once per process.
//   dinv:   RN(1/d) when div_d may use its reciprocal step (every significand
//           of one binade matches __fdiv_rn), else 0
//   scaled: div_d_scaled matches __fdiv_rn for every |x| < 2^31
struct DivCheck { float dinv; int scaled; };
static int div_check(float d, cudaStream_t st, int* bad, DivCheck* out) {
    static std::mutex mu;
    static std::vector<std::pair<std::pair<int, unsigned>, DivCheck>> cache;
    int dev = 0;
    FG_CUDA(cudaGetDevice(&dev));
    unsigned bits;
    std::memcpy(&bits, &d, 4);
    {
        std::lock_guard<std::mutex> lk(mu);
        for (auto& e : cache)
            if (e.first.first == dev && e.first.second == bits) {
                *out = e.second;
                return FG_OK;
            }
    }
    const float dinv = 1.0f / d;
    DivCheck c{0.f, 0};
    if (d >= 0x1p-30f && d <= 0x1p30f && std::fabs((double)d * (double)dinv - 1.0) < 0x1p-25) {
        int nbad[2] = {-1, -1};
        int sms = 0;
        FG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        fg::k_div_check<<<512, 256, 0, st>>>(d, dinv, bad);
        FG_CUDA(cudaGetLastError());
        fg::k_div_check_scaled<<<sms * 8, 256, 0, st>>>(d, dinv, bad + 1);
        FG_CUDA(cudaGetLastError());
        FG_CUDA(cudaMemcpyAsync(nbad, bad, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
        FG_CUDA(cudaStreamSynchronize(st));
        if (nbad[0] == 0) {
            c.dinv = dinv;
            c.scaled = nbad[1] == 0;
        }
    }
    std::lock_guard<std::mutex> lk(mu);
    cache.push_back({{dev, bits}, c});
    *out = c;
    return FG_OK;
}

static int bind_one(fg_plan* p, void* workspace, int64_t bytes, void* stream) {
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
    FG_CUDA(up(p->o_order, p->order.data(), p->order.size() * sizeof(int)));
    FG_CUDA(up(p->o_tiles, p->tiles.data(), p->tiles.size() * sizeof(int4)));
    FG_CUDA(up(p->o_srcev, p->src_ev.data(), p->src_ev.size() * sizeof(Ev)));
    FG_CUDA(up(p->o_rxev, p->rx_ev.data(), p->rx_ev.size() * sizeof(Ev)));
    FG_CUDA(up(p->o_injev, p->inj_ev.data(), p->inj_ev.size() * sizeof(Ev)));
    std::vector<int> offs;
    offs.insert(offs.end(), p->src_off.begin(), p->src_off.end());
    offs.insert(offs.end(), p->rx_off.begin(), p->rx_off.end());
    offs.insert(offs.end(), p->inj_off.begin(), p->inj_off.end());
    FG_CUDA(up(p->o_offs, offs.data(), offs.size() * sizeof(int)));
    FG_CUDA(up(p->o_srcw, p->srcw.data(), p->srcw.size() * sizeof(float)));
    // receiver cells per shot for the exact adjoint's injection, (-1, -1) when inert
    std::vector<int2> rxpos((size_t)p->S * p->nrx);
    for (size_t k = 0; k < rxpos.size(); ++k) {
        const int i = p->rx[3 * k], j = p->rx[3 * k + 1], kk = p->rx[3 * k + 2];
        rxpos[k] = classify(p, i, j, kk) == 1 ? make_int2(i, j) : make_int2(-1, -1);
    }
    FG_CUDA(up(p->o_rxpos, rxpos.data(), rxpos.size() * sizeof(int2)));
    FG_CUDA(up(p->o_pml, p->pml.data(), p->pml.size() * sizeof(float)));
    FG_CUDA(cudaMemsetAsync(p->ws + p->o_err, 0, sizeof(int) * 4, st));
    // division by the cell size: the reciprocal step of div_d is enabled when
    // it returns __fdiv_rn's bits for every significand (one binade decides all)
    // The scaled step of the shot-lane CPML rows is enabled when it returns
    // __fdiv_rn's bits for every |x| < 2^31.
    {
        DivCheck c;
        const int rc = div_check(p->dx, st, (int*)(p->ws + p->o_err) + 2, &c);
        if (rc) return rc;
        p->dinv = c.dinv;
        p->div_scaled = c.scaled;
    }
    p->g.dinv = p->dinv;
    p->g.div_scaled = p->div_scaled;
    if (p->kernel == 0) {
        const int rc = encode_tile_maps(p);
        if (rc) return rc;
    }
    // the host tables must stay valid until the copies have been consumed
    FG_CUDA(cudaStreamSynchronize(st));
    return FG_OK;
}

int fg_plan_bind(fg_plan* p, void* workspace, int64_t bytes, void* stream) {
    if (!p) return fail(FG_ERR_INVALID, "fg_plan_bind: NULL plan");
    if (bytes < fg_plan_workspace_bytes(p)) return fail(FG_ERR_WORKSPACE, "workspace missing or too small");
    int rc = bind_one(p, workspace, (int64_t)own_bytes(p), stream);
    if (rc == FG_OK && p->adj)
        rc = bind_one(p->adj, (char*)workspace + own_bytes(p), bytes - (int64_t)own_bytes(p), stream);
    return rc;
}

int fg_plan_set_profile(fg_plan* p, const float* pml, void* stream) {
    if (!p) return fail(FG_ERR_INVALID, "fg_plan_set_profile: NULL plan");
    if (p->th == 0) return FG_OK;
    if (!pml) return fail(FG_ERR_INVALID, "fg_plan_set_profile: NULL profile");
    cudaStream_t st = (cudaStream_t)stream;
    fg_plan* plans[2] = {p, p->adj};
    for (fg_plan* q : plans) {
        if (!q) continue;
        q->pml.assign(pml, pml + 8 * (size_t)q->th);
        // the allocation-free entry point re-uploads the tables of a plan it has not seen
        q->id = g_next_plan_id.fetch_add(1);
        if (q->ws)
            FG_CUDA(cudaMemcpyAsync(q->ws + q->o_pml, q->pml.data(), q->pml.size() * sizeof(float),
                                    cudaMemcpyHostToDevice, st));
    }
    return FG_OK;
}

int fg_coefficients(const float* er, const float* se, const float* mr, int32_t nx, int32_t ny, float dt, float dx,
                    int32_t adjoint, float* out, int32_t pitch, void* stream) {
    if (!er || !se || !mr || !out) return fail(FG_ERR_INVALID, "fg_coefficients: NULL argument");
    if (nx < 1 || ny < 1 || pitch < ny + 1) return fail(FG_ERR_INVALID, "fg_coefficients: bad shape");
    return coefficients(er, se, mr, nx, ny, dt, dx, adjoint, out, pitch, 0, (cudaStream_t)stream);
}

}  // extern "C"

namespace {

// Blocks of the general kernel's persistent launch when the interior tiles
// run beside it: split_bpsm per SM (fewer than it could hold, so that the
// interior kernel's blocks fit beside it), at most one warp per tile.
cudaError_t split_blocks(const fg_plan* p, int* blocks) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const int need = (p->slab0 + p->WPB - 1) / p->WPB;
    *blocks = std::max(1, std::min(need, p->split_bpsm * sms));
    return cudaSuccess;
}

// One persistent launch over the models plans[0..n) with descriptors devs:
// forward steps [t0, t1) / adjoint rounds [k0, k1) (round k runs iteration
// nt - 1 - k of each model).  The barrier words are the first plan's.
cudaError_t multi_devs(fg_plan* const* plans, const Dev* devs, int n, fg::MultiDevs* M, int* want, cudaStream_t st) {
    M->n = n;
    int most = 1;
    for (int m = 0; m < n; ++m) {
        M->d[m] = devs[m];
        most = std::max(most, plans[m]->ntiles);
    }
    M->bar = (unsigned*)(plans[0]->ws + plans[0]->o_bar);
    M->err = devs[0].err;
    *want = (most + 3) / 4;
    return cudaMemsetAsync(M->bar, 0, sizeof(unsigned), st);
}
cudaError_t multi_fwd(fg_plan* const* plans, const Dev* devs, int n, int t0, int t1, cudaStream_t st) {
    fg::MultiDevs M;
    int want = 1;
    cudaError_t e = multi_devs(plans, devs, n, &M, &want, st);
    if (e != cudaSuccess) return e;
    if (n == 1) return launch_fwd_persist(devs[0], plans[0]->shot, plans[0]->W, M.bar, want, t0, t1, st);
    return launch_fwd_multi(M, plans[0]->shot, plans[0]->W, want, t0, t1, st);
}
cudaError_t multi_adj(fg_plan* const* plans, const Dev* devs, int n, int k0, int k1, cudaStream_t st) {
    fg::MultiDevs M;
    int want = 1;
    cudaError_t e = multi_devs(plans, devs, n, &M, &want, st);
    if (e != cudaSuccess) return e;
    if (n == 1) return launch_adj_persist(devs[0], plans[0]->shot, plans[0]->W, M.bar, want, k0, k1, st);
    return launch_adj_multi(M, plans[0]->shot, plans[0]->W, want, k0, k1, st);
}

// Forward steps [t0, t1) of plan p with descriptor g.
int fwd_steps(fg_plan* p, const Dev& g, int t0, int t1, cudaStream_t st) {
    if (p->kernel == 0) {
        FwdTileFn tfn = pick_fwd_tile(p->shot, p->W);
        if (!tfn) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        for (int t = t0; t < t1; ++t) FG_CUDA(tfn(p, g, t, st));
    } else if (p->kernel == 2) {
        FwdFn fn = pick_fwd_band(p->W, p->WPB);
        if (!fn) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        for (int t = t0; t < t1; ++t) FG_CUDA(fn(g, t, p->WPB, p->D, &p->fwd_blocks, st));
    } else if (p->persist) {
        FG_CUDA(multi_fwd(&p, &g, 1, t0, t1, st));
    } else if (p->split) {
        // the general lane march on the tiles before slab0, the slab kernel on
        // [slab0, core0), the interior kernel on the rest; each behind the one
        // before with programmatic dependent launch
        FwdFn fn = pick_fwd(p->shot, p->W), fs = pick_fwd_slab(p->W), fc = pick_fwd_core(p->W);
        if (!fn || !fs || !fc) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        Dev gb = g;
        gb.ntiles = p->slab0;
        if (p->slab0 > 0 && p->fwd_blocks == 0) FG_CUDA(split_blocks(p, &p->fwd_blocks));
        const bool gen = p->slab0 > 0, slab = p->core0 > p->slab0, core = p->core0 < p->ntiles;
        for (int t = t0; t < t1; ++t) {
            if (gen) FG_CUDA(fn(gb, t, p->WPB, p->D, &p->fwd_blocks, st));
            if (slab) FG_CUDA(fs(g, t, p->slab_bpsm, gen, &p->fwd_slab_blocks, st));
            if (core) FG_CUDA(fc(g, t, 4, gen || slab, &p->fwd_core_blocks, st));
        }
    } else {
        FwdFn fn = p->pair ? pick_fwd2(p->W) : pick_fwd(p->shot, p->W);
        if (!fn) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        for (int t = t0; t < t1; ++t) FG_CUDA(fn(g, t, p->WPB, p->D, &p->fwd_blocks, st));
    }
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

// Adjoint iterations it = hi, hi-1, .., lo (>= 1) of plan a; g.hist holds steps
// from g.hist_t0 on, nsteps of them.
int adj_steps(fg_plan* a, const Dev& g, int hi, int lo, int nsteps, cudaStream_t st) {
    if (a->kernel == 0) {
        AdjTileFn tfn = pick_adj_tile(a->shot, a->W);
        if (!tfn) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        CUtensorMap tmh;
        const int rc = encode_hist_map(a, &tmh, g.hist, nsteps);
        if (rc) return rc;
        for (int it = hi; it >= lo; --it) FG_CUDA(tfn(a, g, tmh, it, (a->nt - 1 - it) & 1, st));
    } else if (a->kernel == 2) {
        AdjFn fn = pick_adj_band(a->W, a->WPB);
        if (!fn) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        for (int it = hi; it >= lo; --it) FG_CUDA(fn(g, it, (a->nt - 1 - it) & 1, a->WPB, a->D, &a->adj_blocks, st));
    } else if (a->persist) {
        FG_CUDA(multi_adj(&a, &g, 1, a->nt - 1 - hi, a->nt - lo, st));
    } else if (a->split) {
        AdjFn fn = pick_adj(a->shot, a->W), fs = pick_adj_slab(a->W), fc = pick_adj_core(a->W);
        if (!fn || !fs || !fc) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        Dev gb = g;
        gb.ntiles = a->slab0;
        if (a->slab0 > 0 && a->adj_blocks == 0) FG_CUDA(split_blocks(a, &a->adj_blocks));
        const bool gen = a->slab0 > 0, slab = a->core0 > a->slab0, core = a->core0 < a->ntiles;
        for (int it = hi; it >= lo; --it) {
            const int rp = (a->nt - 1 - it) & 1;
            if (gen) FG_CUDA(fn(gb, it, rp, a->WPB, a->D, &a->adj_blocks, st));
            if (slab) FG_CUDA(fs(g, it, rp, a->slab_bpsm, gen, &a->adj_slab_blocks, st));
            if (core) FG_CUDA(fc(g, it, rp, 4, gen || slab, &a->adj_core_blocks, st));
        }
    } else {
        AdjFn fn = a->pair ? pick_adj2(a->W) : pick_adj(a->shot, a->W);
        if (!fn) return fail(FG_ERR_INVALID, "no kernel for this tuning");
        for (int it = hi; it >= lo; --it) FG_CUDA(fn(g, it, (a->nt - 1 - it) & 1, a->WPB, a->D, &a->adj_blocks, st));
    }
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

// Start of an adjoint solve on plan a: adjoint coefficients, zero state and accumulators.
int adj_begin(fg_plan* a, const float* er, const float* se, const float* mr, cudaStream_t st) {
    int rc = coefficients(er, se, mr, a->nx, a->ny, a->dt, a->dx, 1, (float*)(a->ws + a->o_coef), a->P, fg::PADC, st);
    if (rc) return rc;
    if ((rc = reset_state(a, st))) return rc;
    const size_t n = (size_t)a->nx * a->ny;
    FG_CUDA(cudaMemsetAsync(a->ws + a->o_gacc, 0, (size_t)a->ngroups * 2 * n * sizeof(double), st));
    return FG_OK;
}

// End of an adjoint solve: the last imaging term (g.hist must hold step 0),
// the group sum, the norms and the scaled gradients.
int adj_finish(fg_plan* a, const Dev& g, float* grad_eps, float* grad_sig, int normalize, double* norms,
               cudaStream_t st) {
    if (a->nt >= 2) {
        // the adjoint Ez after the last step (it = 1) is in the buffer that launch wrote
        const float* ez_final = g.ez[((a->nt - 2) & 1) ^ 1];
        const long long cells = (long long)a->ngroups * a->nx * a->ny;
        const int tb = (int)((cells + 255) / 256);
        if (a->pair) fg::k_imaging_tail<64><<<tb, 256, 0, st>>>(g, ez_final);
        else if (a->shot) fg::k_imaging_tail<32><<<tb, 256, 0, st>>>(g, ez_final);
        else fg::k_imaging_tail<1><<<tb, 256, 0, st>>>(g, ez_final);
    }
    const size_t n = (size_t)a->nx * a->ny;
    double* sums = (double*)(a->ws + a->o_sums);
    double* partial = (double*)(a->ws + a->o_partial);
    double* nrm = norms ? norms : (double*)(a->ws + a->o_norms);
    fg::k_grad_sum<<<kRedBlocks, 256, 0, st>>>(g.gacc, a->ngroups, (long long)n, sums, partial);
    fg::k_grad_norm<<<1, 32, 0, st>>>(partial, kRedBlocks, nrm);
    const int blocks = (int)((n + 255) / 256);
    fg::k_grad_scale<<<blocks, 256, 0, st>>>(sums, nrm, (long long)n, normalize, grad_eps, grad_sig);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

size_t hist_step_floats(const fg_plan* p) { return (size_t)p->ngroups * p->nx * p->Ph * p->CS; }

// One checkpoint: the state of one parity (Ez, Hx, Hy of every group, then
// the four CPML auxiliary arrays).
size_t checkpoint_floats(const fg_plan* p) {
    return 3 * (size_t)p->ngroups * p->plane + 2 * (size_t)p->ngroups * (p->pxs + p->pys);
}

// Copy the state of parity `par` to (save) or from (restore) a checkpoint.
int checkpoint_copy(fg_plan* p, int par, float* ck, bool save, cudaStream_t st) {
    const Dev& g = p->g;
    const size_t fp = (size_t)p->ngroups * p->plane, fx = (size_t)p->ngroups * p->pxs, fy = (size_t)p->ngroups * p->pys;
    float* parts[7] = {g.ez[par], g.hx[par], g.hy[par], g.pex[par], g.phx[par], g.pey[par], g.phy[par]};
    const size_t len[7] = {fp, fp, fp, fx, fx, fy, fy};
    for (int k = 0; k < 7; ++k) {
        if (len[k] == 0) continue;
        if (save) FG_CUDA(cudaMemcpyAsync(ck, parts[k], len[k] * sizeof(float), cudaMemcpyDeviceToDevice, st));
        else FG_CUDA(cudaMemcpyAsync(parts[k], ck, len[k] * sizeof(float), cudaMemcpyDeviceToDevice, st));
        ck += len[k];
    }
    return FG_OK;
}

int checkpoint_args(const fg_plan* p, int interval, int64_t bytes, const void* ck, const char* who) {
    if (interval < 1) return fail(FG_ERR_INVALID, std::string(who) + ": interval must be >= 1");
    const int64_t need = fg_plan_checkpoint_bytes(p, interval);
    if (need > 0 && (!ck || bytes < need))
        return fail(FG_ERR_WORKSPACE, std::string(who) + ": checkpoint buffer missing or too small");
    if (((uintptr_t)ck) % 16) return fail(FG_ERR_INVALID, std::string(who) + ": checkpoint buffer not 16-byte aligned");
    return FG_OK;
}

}  // namespace

extern "C" {

int fg_forward(fg_plan* p, const float* er, const float* se, const float* mr, float* traces, float* hist,
               void* stream) {
    if (!p || !er || !se || !mr || (!traces && p->nrx > 0)) return fail(FG_ERR_INVALID, "fg_forward: NULL argument");
    if (!p->ws) return fail(FG_ERR_WORKSPACE, "fg_forward: plan has no workspace");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = coefficients(er, se, mr, p->nx, p->ny, p->dt, p->dx, 0, (float*)(p->ws + p->o_coef), p->P, fg::PADC, st);
    if (rc) return rc;
    if ((rc = reset_state(p, st))) return rc;
    if (p->nrx > 0) FG_CUDA(cudaMemsetAsync(traces, 0, (size_t)p->S * p->nt * p->nrx * sizeof(float), st));
    Dev g = p->g;
    g.traces = traces;
    g.hist = hist;
    if (hist) {
        g.out_lo = (const char*)hist;
        g.out_hi = (const char*)(hist + (size_t)p->nt * hist_step_floats(p));
    }
    return fwd_steps(p, g, 0, p->nt, st);
}

static int adjoint_full(fg_plan* p, const float* er, const float* se, const float* mr, const float* hist,
                        const float* resid, const float* obs, float obs_scale, float* grad_eps, float* grad_sig,
                        int32_t normalize, double* norms, void* stream, const char* who) {
    if (!p || !er || !se || !mr || !hist || (!resid && p->nrx > 0))
        return fail(FG_ERR_INVALID, std::string(who) + ": NULL argument");
    fg_plan* a = p->adj ? p->adj : p;
    if (!a->ws) return fail(FG_ERR_WORKSPACE, std::string(who) + ": plan has no workspace");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = adj_begin(a, er, se, mr, st);
    if (rc) return rc;
    Dev g = a->g;
    g.hist = const_cast<float*>(hist);
    g.out_lo = (const char*)hist;
    g.out_hi = (const char*)(hist + (size_t)a->nt * hist_step_floats(a));
    g.resid = resid;
    g.obs = obs;
    g.obs_scale = obs_scale;
    if ((rc = adj_steps(a, g, a->nt - 1, 1, a->nt, st))) return rc;
    return adj_finish(a, g, grad_eps, grad_sig, normalize, norms, st);
}

int fg_adjoint_reference(fg_plan* p, const float* er, const float* se, const float* mr, const float* hist,
                         const float* resid, float* grad_eps, float* grad_sig, int32_t normalize, double* norms,
                         void* stream) {
    return adjoint_full(p, er, se, mr, hist, resid, nullptr, 0.f, grad_eps, grad_sig, normalize, norms, stream,
                        "fg_adjoint_reference");
}

int fg_adjoint_reference_l1(fg_plan* p, const float* er, const float* se, const float* mr, const float* hist,
                            const float* traces, const float* observed, float scale, float* grad_eps,
                            float* grad_sig, int32_t normalize, double* norms, void* stream) {
    if (p && p->nrx > 0 && !observed) return fail(FG_ERR_INVALID, "fg_adjoint_reference_l1: NULL observed traces");
    return adjoint_full(p, er, se, mr, hist, traces, observed, scale, grad_eps, grad_sig, normalize, norms, stream,
                        "fg_adjoint_reference_l1");
}

int fg_adjoint_exact(fg_plan* p, const float* er, const float* se, const float* mr, const float* hist,
                     const float* weights, float* grad_eps, float* grad_sig, void* stream) {
    if (!p || !er || !se || !mr || !hist || (!weights && p->nrx > 0))
        return fail(FG_ERR_INVALID, "fg_adjoint_exact: NULL argument");
    fg_plan* a = p->adj ? p->adj : p;
    if (!a->ws) return fail(FG_ERR_WORKSPACE, "fg_adjoint_exact: plan has no workspace");
    cudaStream_t st = (cudaStream_t)stream;
    // the forward's coefficients (Ucget): the adjoint of the forward operator itself
    int rc = coefficients(er, se, mr, a->nx, a->ny, a->dt, a->dx, 0, (float*)(a->ws + a->o_coef), a->P, fg::PADC, st);
    if (rc) return rc;
    if ((rc = reset_state(a, st))) return rc;
    const size_t n = (size_t)a->nx * a->ny;
    FG_CUDA(cudaMemsetAsync(a->ws + a->o_gacc, 0, (size_t)a->ngroups * 2 * n * sizeof(double), st));
    Dev g = a->g;
    g.hist = const_cast<float*>(hist);
    g.out_lo = (const char*)hist;
    g.out_hi = (const char*)(hist + (size_t)a->nt * hist_step_floats(a));
    const int2* rxpos = (const int2*)(a->ws + a->o_rxpos);
    const int nt = a->nt;
    // row 0 and column 0 stay zero in the forward unless a source lies on them
    int proj = 1;
    for (size_t k = 0; k + 2 < a->src.size(); k += 3)
        if (classify(a, a->src[k], a->src[k + 1], a->src[k + 2]) == 1 && (a->src[k] == 0 || a->src[k + 1] == 0))
            proj = 0;
    if (nt >= 2) {
        // lambda_{nt-1} = R^T w_{nt-1} in parity 0; iteration it reads parity (nt-1-it) & 1
        if (a->nrx > 0) FG_CUDA(launch_inject_exact(g, rxpos, weights, nt - 1, 0, a->CS, st));
        for (int it = nt - 1; it >= 1; --it) {
            const int rp = (nt - 1 - it) & 1;
            FG_CUDA(launch_adj_exact(g, it, rp, a->CS, proj, st));
            if (it >= 2 && a->nrx > 0) FG_CUDA(launch_inject_exact(g, rxpos, weights, it - 1, rp ^ 1, a->CS, st));
        }
    }
    double* sums = (double*)(a->ws + a->o_sums);
    double* partial = (double*)(a->ws + a->o_partial);
    fg::k_grad_sum<<<kRedBlocks, 256, 0, st>>>(g.gacc, a->ngroups, (long long)n, sums, partial);
    FG_CUDA(cudaGetLastError());
    const double e0 = (double)8.8541878128e-12f;   // the float constant of uc.cu:8
    FG_CUDA(launch_grad_exact(sums, er, se, a->nx, a->ny, e0 / (double)a->dt, grad_eps, grad_sig, st));
    return FG_OK;
}

namespace {
// The checks a batch of plans must pass: bound, persistent lane march, one
// kernel shape for all (the launch is one kernel), at most FG_BATCH_MAX.
int batch_args(fg_plan* const* plans, int32_t n, bool adjoint, const char* who) {
    if (!plans || n < 1 || n > FG_BATCH_MAX)
        return fail(FG_ERR_INVALID, std::string(who) + ": 1 to " + std::to_string(FG_BATCH_MAX) + " plans");
    for (int m = 0; m < n; ++m) {
        const fg_plan* p = plans[m];
        if (!p) return fail(FG_ERR_INVALID, std::string(who) + ": NULL plan");
        const fg_plan* q = adjoint ? (p->adj ? p->adj : p) : p;
        const fg_plan* q0 = adjoint ? (plans[0]->adj ? plans[0]->adj : plans[0]) : plans[0];
        if (!q->ws) return fail(FG_ERR_WORKSPACE, std::string(who) + ": plan has no workspace");
        if (!q->persist)
            return fail(FG_ERR_INVALID, std::string(who) + ": plan " + std::to_string(m) +
                                            " is not a persistent lane-march plan (tuning persistent)");
        if (q->shot != q0->shot || q->W != q0->W)
            return fail(FG_ERR_INVALID, std::string(who) + ": the plans differ in lanes or cells_per_thread");
    }
    return FG_OK;
}
}  // namespace

int fg_forward_batch(fg_plan* const* plans, int32_t n, const float* const* er, const float* const* se,
                     const float* const* mr, float* const* traces, float* const* hist, void* stream) {
    int rc = batch_args(plans, n, false, "fg_forward_batch");
    if (rc) return rc;
    if (!er || !se || !mr || !traces || !hist) return fail(FG_ERR_INVALID, "fg_forward_batch: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    Dev devs[FG_BATCH_MAX];
    int nt = 0;
    for (int m = 0; m < n; ++m) {
        fg_plan* p = plans[m];
        if (!er[m] || !se[m] || !mr[m] || (!traces[m] && p->nrx > 0))
            return fail(FG_ERR_INVALID, "fg_forward_batch: NULL argument");
        if ((rc = coefficients(er[m], se[m], mr[m], p->nx, p->ny, p->dt, p->dx, 0, (float*)(p->ws + p->o_coef), p->P,
                               fg::PADC, st)))
            return rc;
        if ((rc = reset_state(p, st))) return rc;
        if (p->nrx > 0) FG_CUDA(cudaMemsetAsync(traces[m], 0, (size_t)p->S * p->nt * p->nrx * sizeof(float), st));
        devs[m] = p->g;
        devs[m].traces = traces[m];
        devs[m].hist = hist[m];
        if (hist[m]) {
            devs[m].out_lo = (const char*)hist[m];
            devs[m].out_hi = (const char*)(hist[m] + (size_t)p->nt * hist_step_floats(p));
        }
        nt = std::max(nt, p->nt);
    }
    FG_CUDA(multi_fwd(plans, devs, n, 0, nt, st));
    return FG_OK;
}

int fg_adjoint_reference_batch(fg_plan* const* plans, int32_t n, const float* const* er, const float* const* se,
                               const float* const* mr, const float* const* hist, const float* const* resid,
                               float* const* grad_eps, float* const* grad_sig, int32_t normalize, void* stream) {
    int rc = batch_args(plans, n, true, "fg_adjoint_reference_batch");
    if (rc) return rc;
    if (!er || !se || !mr || !hist || !resid || !grad_eps || !grad_sig)
        return fail(FG_ERR_INVALID, "fg_adjoint_reference_batch: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    fg_plan* as[FG_BATCH_MAX];
    Dev devs[FG_BATCH_MAX];
    int rounds = 0;
    for (int m = 0; m < n; ++m) {
        fg_plan* a = plans[m]->adj ? plans[m]->adj : plans[m];
        if (!er[m] || !se[m] || !mr[m] || !hist[m] || (!resid[m] && a->nrx > 0))
            return fail(FG_ERR_INVALID, "fg_adjoint_reference_batch: NULL argument");
        if ((rc = adj_begin(a, er[m], se[m], mr[m], st))) return rc;
        as[m] = a;
        devs[m] = a->g;
        devs[m].hist = const_cast<float*>(hist[m]);
        devs[m].out_lo = (const char*)hist[m];
        devs[m].out_hi = (const char*)(hist[m] + (size_t)a->nt * hist_step_floats(a));
        devs[m].resid = resid[m];
        rounds = std::max(rounds, a->nt - 1);
    }
    if (rounds > 0) FG_CUDA(multi_adj(as, devs, n, 0, rounds, st));
    for (int m = 0; m < n; ++m)
        if ((rc = adj_finish(as[m], devs[m], grad_eps[m], grad_sig[m], normalize, nullptr, st))) return rc;
    return FG_OK;
}

int64_t fg_plan_checkpoint_bytes(const fg_plan* p, int32_t interval) {
    if (!p || interval < 1) return -1;
    const int64_t segments = (p->nt + interval - 1) / interval;
    return (segments - 1) * (int64_t)(checkpoint_floats(p) * sizeof(float));
}

int fg_forward_checkpointed(fg_plan* p, const float* er, const float* se, const float* mr, float* traces, void* ckpt,
                            int64_t ckpt_bytes, int32_t interval, void* stream) {
    if (!p || !er || !se || !mr || (!traces && p->nrx > 0))
        return fail(FG_ERR_INVALID, "fg_forward_checkpointed: NULL argument");
    if (!p->ws) return fail(FG_ERR_WORKSPACE, "fg_forward_checkpointed: plan has no workspace");
    int rc = checkpoint_args(p, interval, ckpt_bytes, ckpt, "fg_forward_checkpointed");
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if ((rc = coefficients(er, se, mr, p->nx, p->ny, p->dt, p->dx, 0, (float*)(p->ws + p->o_coef), p->P, fg::PADC, st)))
        return rc;
    if ((rc = reset_state(p, st))) return rc;
    if (p->nrx > 0) FG_CUDA(cudaMemsetAsync(traces, 0, (size_t)p->S * p->nt * p->nrx * sizeof(float), st));
    Dev g = p->g;
    g.traces = traces;
    const size_t cf = checkpoint_floats(p);
    for (int s0 = 0; s0 < p->nt; s0 += interval) {
        // checkpoint c >= 1 holds the state at the start of step c * interval
        if (s0 > 0 && (rc = checkpoint_copy(p, s0 & 1, (float*)ckpt + (size_t)(s0 / interval - 1) * cf, true, st)))
            return rc;
        if ((rc = fwd_steps(p, g, s0, std::min(s0 + interval, p->nt), st))) return rc;
    }
    return FG_OK;
}

int fg_adjoint_reference_checkpointed(fg_plan* p, const float* er, const float* se, const float* mr, const void* ckpt,
                                      int64_t ckpt_bytes, int32_t interval, float* segment, const float* resid,
                                      float* grad_eps, float* grad_sig, int32_t normalize, double* norms,
                                      void* stream) {
    if (!p || !er || !se || !mr || !segment || (!resid && p->nrx > 0))
        return fail(FG_ERR_INVALID, "fg_adjoint_reference_checkpointed: NULL argument");
    if (!p->adj) return fail(FG_ERR_INVALID, "fg_adjoint_reference_checkpointed: plan without an adjoint plan");
    fg_plan* a = p->adj;
    if (!p->ws || !a->ws) return fail(FG_ERR_WORKSPACE, "fg_adjoint_reference_checkpointed: plan has no workspace");
    int rc = checkpoint_args(p, interval, ckpt_bytes, ckpt, "fg_adjoint_reference_checkpointed");
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // forward recompute on this plan (Ucget coefficients), adjoint on its adjoint plan
    if ((rc = coefficients(er, se, mr, p->nx, p->ny, p->dt, p->dx, 0, (float*)(p->ws + p->o_coef), p->P, fg::PADC, st)))
        return rc;
    if ((rc = adj_begin(a, er, se, mr, st))) return rc;
    const size_t cf = checkpoint_floats(p), hs = hist_step_floats(p);
    Dev gf = p->g;
    gf.traces = nullptr;
    gf.hist = segment;
    gf.out_lo = (const char*)segment;
    gf.out_hi = (const char*)(segment + (size_t)interval * hs);
    Dev ga = a->g;
    ga.hist = segment;
    ga.out_lo = gf.out_lo;
    ga.out_hi = gf.out_hi;
    ga.resid = resid;
    const int segments = (p->nt + interval - 1) / interval;
    for (int c = segments - 1; c >= 0; --c) {
        const int s0 = c * interval, s1 = std::min(s0 + interval, p->nt);
        // the forward state at the start of step s0, then its history over [s0, s1)
        if (c == 0) {
            if ((rc = reset_state(p, st))) return rc;
        } else {
            if ((rc = checkpoint_copy(p, s0 & 1, (float*)ckpt + (size_t)(c - 1) * cf, false, st))) return rc;
            FG_CUDA(cudaMemsetAsync(p->ws + p->o_ctr, 0, 8 * sizeof(int), st));
        }
        gf.hist_t0 = s0;
        if ((rc = fwd_steps(p, gf, s0, s1, st))) return rc;
        ga.hist_t0 = s0;
        const int lo = std::max(s0, 1);
        if (s1 - 1 >= lo && (rc = adj_steps(a, ga, s1 - 1, lo, s1 - s0, st))) return rc;
    }
    return adj_finish(a, ga, grad_eps, grad_sig, normalize, norms, st);
}

int fg_forward_static(fg_plan* p, const float* er, const float* se, const float* mr, float* traces, float* hist,
                      void* stream) {
    if (!p) return fail(FG_ERR_INVALID, "fg_forward_static: NULL plan");
    if (p->total > (size_t)FG_STATIC_SCRATCH_BYTES)
        return fail(FG_ERR_WORKSPACE, "fg_forward_static: the plan needs " + std::to_string(p->total) +
                                          " bytes of scratch, more than the static " +
                                          std::to_string((long long)FG_STATIC_SCRATCH_BYTES));
    void* scratch = nullptr;
    int dev = 0;
    int rc = static_scratch(&scratch, &dev);
    if (rc) return rc;
    char* saved = p->ws;
    const int64_t saved_bytes = p->ws_bytes;
    const float saved_dinv = p->dinv;
    const int saved_scaled = p->div_scaled;
    // the tables are uploaded (with a wait for the stream) only when the array
    // does not hold this plan's already; the field state is cleared by the solve
    bool filled;
    {
        std::lock_guard<std::mutex> lock(g_static_mu);
        filled = g_static_owner[dev].plan == p->id;
        if (filled) {
            p->dinv = g_static_owner[dev].dinv;
            p->div_scaled = g_static_owner[dev].div_scaled;
        }
    }
    if (filled) {
        p->ws = (char*)scratch;
        p->ws_bytes = FG_STATIC_SCRATCH_BYTES;
        fill_grid(p);
        if (p->kernel == 0) rc = encode_tile_maps(p);
    } else {
        {
            std::lock_guard<std::mutex> lock(g_static_mu);
            g_static_owner[dev].plan = 0;
        }
        rc = bind_one(p, scratch, (int64_t)FG_STATIC_SCRATCH_BYTES, stream);
        if (rc == FG_OK) {
            std::lock_guard<std::mutex> lock(g_static_mu);
            g_static_owner[dev] = StaticOwner{p->id, p->dinv, p->div_scaled};
        }
    }
    if (rc == FG_OK) rc = fg_forward(p, er, se, mr, traces, hist, stream);
    p->ws = saved;
    p->ws_bytes = saved_bytes;
    p->dinv = saved_dinv;
    p->div_scaled = saved_scaled;
    if (saved) {
        fill_grid(p);
        // the tile kernels' tensor maps address the workspace too
        if (p->kernel == 0) {
            const int mrc = encode_tile_maps(p);
            if (rc == FG_OK) rc = mrc;
        }
    }
    return rc;
}

}  // extern "C"
