// Band-pipeline time-step kernels (shot lanes): one launch per time step;
// persistent CTAs of C consumer warps and one producer warp.
//
// Tile = (shot group, row chunk [i0, i1), column band [b0, b0 + C*W)).  The
// consumer warps of a CTA march down the rows of the tile together, warp k
// owning the W cells b0 + k*W .. b0 + k*W + W-1 of the band, lane l being
// shot slot l of the group (32 shots of the same cells, so a cell is one
// 128-byte line).  As in the lane march (fdtd_lanes.cuh) each warp carries
// the previous row in registers and recomputes its one-cell halo, so warps
// never wait on each other and every cell is read once and written once per
// step.  What differs is the operand delivery: lane 0 of the producer warp
// streams, row by row, every operand the band needs -- the old Ez/Hx/Hy row
// segments of the whole band with their halo cells, the coefficient rows and
// (adjoint) the stored forward Ez row -- into a ring of D shared-memory
// stages with one cp.async.bulk copy per segment, completing on the stage's
// "full" mbarrier.  A row segment of a band is contiguous in the shot-lane
// layout, so a copy is a single 1-D bulk transfer; bytes in flight cost no
// registers and the consumers issue no global loads for the fields.  The
// consumers copy their operands out of the stage, release it (one arrival per
// warp on its "empty" mbarrier) and compute; the new state, the CPML
// auxiliaries and the history are stored straight to global memory.  The
// producer also prefetches the CPML auxiliaries of each row it issues into
// L2 (the consumers load them directly).
//
// Tiles come from the launch's tile counter (CPML-heavy tiles first in the
// fetch order); the producer takes them, and each tile opens with a head
// stage whose header carries the tile and its event ranges to the consumers
// (the tile's first rows and its halo row).  A header with b0 < 0 ends the
// launch.  Every wait is bounded (2 s): a stage that never lands or a stage
// that is never released sets the device error word and the CTA's stop flag,
// every wait then returns at once, the producer waits (bounded) for the copies
// it issued, and the CTA leaves; later launches of the solve return at once.
//
// Forward step t (src/compute.py:574-712) and reference-mode adjoint step
// (src/compute.py:1048-1172): per row, the same arithmetic as the lane march
// (fwd_row, adj_row), hence the reference's bits.
#pragma once

#include "fdtd_common.cuh"
#include "fdtd_lanes.cuh"
#include "fdtd_shot.cuh"
#include "fdtd_tile.cuh"

namespace fg {

// Stage geometry (floats; a cell segment holds 32 floats per cell).
template <int W, int C>
struct BandGeom {
    static constexpr int BC = C * W;   // cells of a band
    static constexpr int HDR = 32;     // header: int4 (b0, i0, i1, group) + int4 event ranges
    // forward row i: Ez row i+1 from b0-1 (BC+2 cells), Hx row i from b0-1
    // (BC+1), Hy row i from b0 (BC); uE0 and uE1 of row i from b0 (BC
    // floats each), uH1 of row i from b0-4 (BC+4)
    static constexpr int F_EZ = HDR;
    static constexpr int F_HX = F_EZ + (BC + 2) * 32;
    static constexpr int F_HY = F_HX + (BC + 1) * 32;
    static constexpr int F_CA = F_HY + BC * 32;
    static constexpr int F_CB = F_CA + BC;
    static constexpr int F_CH = F_CB + BC;
    static constexpr int F_END = F_CH + BC + 4;
    // forward head of a tile: Ez row i0 from b0-1 (BC+2), Ez and Hy of row
    // i0-1 from b0 (BC each), uH1 of row i0-1 from b0-4 (BC+4)
    static constexpr int H_EZ = HDR;
    static constexpr int H_EU = H_EZ + (BC + 2) * 32;
    static constexpr int H_HY = H_EU + BC * 32;
    static constexpr int H_CH = H_HY + BC * 32;
    static constexpr int H_END = H_CH + BC + 4;
    // adjoint iteration i (E of row r = i+1, H of row i): Ez row r from b0
    // (BC+1), Hx row r from b0-1 (BC+2), Hy row r from b0 (BC+1), forward Ez of
    // row i from b0 (BC), [head: Hy row i0-1 from b0 (BC+1)], uE0 and uE1 of
    // row r from b0 (BC+4 floats each), uH1 of row i from b0 (BC)
    static constexpr int A_EZ = HDR;
    static constexpr int A_HX = A_EZ + (BC + 1) * 32;
    static constexpr int A_HY = A_HX + (BC + 2) * 32;
    static constexpr int A_HS = A_HY + (BC + 1) * 32;
    static constexpr int A_HU = A_HS + BC * 32;
    static constexpr int A_CA = A_HU + (BC + 1) * 32;
    static constexpr int A_CB = A_CA + BC + 4;
    static constexpr int A_CH = A_CB + BC + 4;
    static constexpr int A_END = A_CH + BC;
    static constexpr int FWD = ((F_END > H_END ? F_END : H_END) + 31) / 32 * 32;
    static constexpr int ADJ = (A_END + 31) / 32 * 32;
};

// Resident CTAs per SM the register budget is sized for (about 128
// registers per thread with C = 4).
template <int C>
constexpr int band_min_blocks() { return C <= 2 ? 5 : (C <= 4 ? 3 : 2); }

// Whole-CTA layout (bytes): CPML profile, the full and empty barriers, the
// stop flag, then D stages.
struct BandSmem {
    size_t prof, bars, flag, stages, stage, total;
    __host__ __device__ BandSmem(int th, int D, int stage_floats) {
        prof = 0;
        bars = ((size_t)8 * th * sizeof(float) + 127) / 128 * 128;
        flag = bars + ((size_t)16 * D + 15) / 16 * 16;
        stages = (flag + 16 + 127) / 128 * 128;
        stage = (size_t)stage_floats * sizeof(float);
        total = stages + (size_t)D * stage;
    }
};

struct BandHead {
    int4 tile;   // b0 (< 0: no more tiles), i0, i1, group
    int4 ev;     // forward: sources [x, y), receivers [z, w); adjoint: injections [x, y)
};

// N consecutive floats of a stage (a coefficient run, the same for every
// lane); p is 16-byte aligned when N is a multiple of 4, 8-byte when of 2.
template <int N>
__device__ __forceinline__ void lds_run(float* x, const float* p) {
    if constexpr (N % 4 == 0) {
#pragma unroll
        for (int k = 0; k < N; k += 4) {
            const float4 v = *reinterpret_cast<const float4*>(p + k);
            x[k] = v.x; x[k + 1] = v.y; x[k + 2] = v.z; x[k + 3] = v.w;
        }
    } else if constexpr (N % 2 == 0) {
#pragma unroll
        for (int k = 0; k < N; k += 2) {
            const float2 v = *reinterpret_cast<const float2*>(p + k);
            x[k] = v.x; x[k + 1] = v.y;
        }
    } else {
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = p[k];
    }
}

// Next tile of the launch for the producer: (b0, i0, i1, group) and the
// tile id, or b0 = -1 when the launch's tiles are gone.
__device__ __forceinline__ int4 band_next_tile(const Dev& g, int* ctr, int& id) {
    const int pos = atomicAdd(ctr, 1);
    if (pos >= g.ntiles) return make_int4(-1, 0, 0, 0);
    const int4 T = __ldg(g.tiles + pos);   // b0, i0, group, id
    id = T.w;
    const int chunk = (T.w / g.nb) % g.nc;
    return make_int4(T.x, T.y, __ldg(g.chunk_row + chunk + 1), T.z);
}

// Producer state of one CTA (lane 0 of the producer warp).
struct BandProducer {
    uint64_t *full, *empty;
    volatile int* stop;
    int D;
    uint32_t qi = 0;   // stages issued
    // Claim the next stage slot (waiting until its consumers released it);
    // false when the CTA stops.
    __device__ __forceinline__ bool claim(const Dev& g, int& slot) {
        slot = (int)(qi % (uint32_t)D);
        if (qi >= (uint32_t)D && !wait_or_stop(g, empty + slot, (qi / D + 1) & 1u, stop)) return false;
        return true;
    }
    // Wait (bounded) for the copies of the last D issued stages before the CTA retires.
    __device__ __forceinline__ void drain() {
        const uint32_t lo = qi > (uint32_t)D ? qi - D : 0u;
        for (uint32_t m = lo; m < qi; ++m) wait_stage(full + m % D, (m / D) & 1u);
    }
};

// ---------------------------------------------------------------------------
// Forward step
// ---------------------------------------------------------------------------
template <int W, int C>
__device__ __forceinline__ void band_fwd_producer(const Dev& g, BandProducer& pr, unsigned char* stages,
                                                  size_t stage_bytes, int* ctr, int rp) {
    using G = BandGeom<W, C>;
    const long long rowS = (long long)g.P * 32;
    for (;;) {
        int id = 0;
        const int4 T = band_next_tile(g, ctr, id);
        int slot;
        if (!pr.claim(g, slot)) return;
        float* st = reinterpret_cast<float*>(stages + (size_t)slot * stage_bytes);
        BandHead* h = reinterpret_cast<BandHead*>(st);
        uint64_t* bar = pr.full + slot;
        h->tile = T;
        if (T.x < 0) {
            mbar_expect_tx(bar, 0);
            ++pr.qi;
            return;
        }
        const int b0 = T.x, i0 = T.y, i1 = T.z, grp = T.w;
        h->ev = make_int4(__ldg(g.src_off + id), __ldg(g.src_off + id + 1), __ldg(g.rx_off + id),
                          __ldg(g.rx_off + id + 1));
        const long long go = (long long)grp * g.plane;
        const float* ez = g.ez[rp] + go + (long long)(b0 - 1 + PADC) * 32;   // cell (0, b0-1)
        const float* hx = g.hx[rp] + go + (long long)(b0 - 1 + PADC) * 32;
        const float* hy = g.hy[rp] + go + (long long)(b0 + PADC) * 32;        // cell (0, b0)
        // head: Ez row i0 from b0-1; Ez and Hy of row i0-1 from b0; uH1 of row i0-1 from b0-4
        issue_stage(g, bar, [&](auto&& f) {
            f(st + G::H_EZ, ez + i0 * rowS, (G::BC + 2) * 128);
            if (i0 >= 1) {
                f(st + G::H_EU, ez + (i0 - 1) * rowS + 32, G::BC * 128);
                f(st + G::H_HY, hy + (i0 - 1) * rowS, G::BC * 128);
                f(st + G::H_CH, g.ch + (long long)(i0 - 1) * g.P + b0 - 4 + PADC, (G::BC + 4) * 4);
            }
        });
        if (g.pf && g.th > 0) prefetch_tile_psi<32>(g, grp, rp, i0 - 1, i0, b0 - 1, b0 + G::BC);
        ++pr.qi;
        for (int i = i0; i < i1; ++i) {
            if (!pr.claim(g, slot)) return;
            st = reinterpret_cast<float*>(stages + (size_t)slot * stage_bytes);
            bar = pr.full + slot;
            const long long crow = (long long)i * g.P + b0 + PADC;
            issue_stage(g, bar, [&](auto&& f) {
                f(st + G::F_EZ, ez + (i + 1) * rowS, (G::BC + 2) * 128);
                f(st + G::F_HX, hx + i * rowS, (G::BC + 1) * 128);
                f(st + G::F_HY, hy + i * rowS, G::BC * 128);
                f(st + G::F_CA, g.ca + crow, G::BC * 4);
                f(st + G::F_CB, g.cb + crow, G::BC * 4);
                f(st + G::F_CH, g.ch + crow - 4, (G::BC + 4) * 4);
            });
            if (g.pf && g.th > 0) prefetch_tile_psi<32>(g, grp, rp, i, i, b0 - 1, b0 + G::BC);
            ++pr.qi;
        }
    }
}

template <int W, int C>
__global__ void __launch_bounds__(32 * (C + 1), band_min_blocks<C>()) k_fwd_band(const Dev g, const int t, const int D) {
    using G = BandGeom<W, C>;
    extern __shared__ __align__(128) unsigned char smem[];
    const BandSmem L(g.th, D, G::FWD);
    float* R = reinterpret_cast<float*>(smem + L.prof);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.bars);
    uint64_t* empty = full + D;
    volatile int* flags = reinterpret_cast<volatile int*>(smem + L.flag);
    unsigned char* stages = smem + L.stages;
    if (abort_launch(g, flags)) return;
    if (threadIdx.x == 0) {
        flags[1] = 0;
        for (int s = 0; s < D; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, C);
        }
        fence_mbar_init();
        if (blockIdx.x == 0) g.tile_ctr[(t + 1) & 1] = 0;   // the next launch's counter
    }
    for (int k = threadIdx.x; k < 8 * g.th; k += blockDim.x) R[k] = __ldg(g.pml + k);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rp = t & 1, wp = rp ^ 1;
    if (warp == C) {
        if (lane == 0) {
            BandProducer pr;
            pr.full = full;
            pr.empty = empty;
            pr.stop = flags + 1;
            pr.D = D;
            band_fwd_producer<W, C>(g, pr, stages, L.stage, g.tile_ctr + (t & 1), rp);
            pr.drain();
        }
        return;
    }
    const int nx = g.nx, ny = g.ny, th = g.th;
    const long long hrow = (long long)g.Ph * 32;
    const int l = lane, cw = warp * W;   // this warp's first cell within the band
    int s = 0;
    uint32_t par = 0;
    auto next = [&]() {
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + s);
        if (++s == D) {
            s = 0;
            par ^= 1u;
        }
    };
    for (;;) {
        if (!wait_or_stop(g, full + s, par, flags + 1)) return;
        const float* st = reinterpret_cast<const float*>(stages + (size_t)s * L.stage);
        const BandHead hd = *reinterpret_cast<const BandHead*>(st);
        if (hd.tile.x < 0) return;
        const int b0 = hd.tile.x, i0 = hd.tile.y, i1 = hd.tile.z, grp = hd.tile.w;
        const int j0 = b0 + cw;
        const int slot = l, sh = grp * 32 + l;
        // the CPML geometry (rd, wr, by) is rebuilt where a row needs it, so
        // it holds no registers across the march
        const bool bcore = j0 >= th + 1 && j0 + W <= ny - th;
        int sc = hd.ev.x, rc = hd.ev.z;
        const int se = hd.ev.y, re = hd.ev.w;
        // Ez_old of row i0, columns j0-1 .. j0+W; new Hy of the row above the chunk
        float ezc[W + 2], hyu[W];
#pragma unroll
        for (int k = 0; k < W + 2; ++k) ezc[k] = st[G::H_EZ + (cw + k) * 32 + l];
#pragma unroll
        for (int w = 0; w < W; ++w) hyu[w] = 0.f;
        // warps whose cells lie beyond the grid (the last band) only release stages
        const bool live = j0 < ny;
        if (live && i0 >= 1) {
            const int ih = i0 - 1;
            float ea[W], chu[W], dz[W];
#pragma unroll
            for (int w = 0; w < W; ++w) {
                ea[w] = st[G::H_EU + (cw + w) * 32 + l];
                hyu[w] = st[G::H_HY + (cw + w) * 32 + l];
                chu[w] = st[G::H_CH + 4 + cw + w];
            }
            next();
#pragma unroll
            for (int w = 0; w < W; ++w) dz[w] = __fsub_rn(ezc[w + 1], ea[w]);
            const PsiG rd = psi_group(g, rp, grp);
            const BandY by = band_fwd<W>(g, j0);
            if (by.lean) {
                fwd_hy_halo_shot<W>(g, R, by, ih, j0, l, hyu, dz, chu, rd);
            } else if (g.fast_cpml) {
                hy_cells<W, 32, false>(g, R, ih, j0, l, hyu, dz, chu, rd, rd);
            } else {
                float ha[W];
#pragma unroll
                for (int w = 0; w < W; ++w) ha[w] = hyu[w];
#pragma unroll
                for (int w = 0; w < W; ++w)
                    if (j0 + w < ny) hyu[w] = hy_cell<32, false>(g, R, ih, j0 + w, l, ha[w], dz[w], chu[w], rd, rd);
            }
        } else {
            next();
        }
        // interior rows of an interior band take the lean path: the update of
        // fwd_core and stores through row pointers advanced row by row
        const bool wcore = live && bcore;
        const long long rowS = (long long)g.P * 32;
        const long long o0 = (long long)grp * g.plane + ((long long)i0 * g.P + j0 + PADC) * 32 + l;
        float* pe = g.ez[wp] + o0;
        float* px = g.hx[wp] + o0;
        float* py = g.hy[wp] + o0;
        float* ph = g.hist ? g.hist + (((long long)(t - g.hist_t0) * g.ngroups + grp) * nx + i0) * hrow +
                                 (long long)j0 * 32 + l
                           : nullptr;
        for (int i = i0; i < i1; ++i) {
            if (!wait_or_stop(g, full + s, par, flags + 1)) return;
            st = reinterpret_cast<const float*>(stages + (size_t)s * L.stage);
            FwdIn<W> B;
            const float* sz = st + G::F_EZ + cw * 32 + l;
#pragma unroll
            for (int k = 0; k < W + 2; ++k) B.en[k] = sz[k * 32];
#pragma unroll
            for (int k = 0; k <= W; ++k) B.hxo[k] = sz[G::F_HX - G::F_EZ + k * 32];
#pragma unroll
            for (int w = 0; w < W; ++w) B.hyo[w] = sz[G::F_HY - G::F_EZ + w * 32];
            lds_run<W>(B.ca, st + G::F_CA + cw);
            lds_run<W>(B.cb, st + G::F_CB + cw);
            B.ch[0] = st[G::F_CH + 3 + cw];
            lds_run<W>(B.ch + 1, st + G::F_CH + 4 + cw);
            next();
            if (wcore && i >= th + 1 && i <= nx - th - 1) {
                float hxn[W + 1], hyn[W], ezn[W];
                fwd_core<W>(B, ezc, hyu, hxn, hyn, ezn);
                fwd_sources<W>(g, i, t, j0, slot, ezn, sc, se);
                st_cells<W, 32>(g, pe, ezn);
                st_cells<W, 32>(g, px, hxn + 1);
                st_cells<W, 32>(g, py, hyn);
                if (ph) st_cells<W, 32, true>(g, ph, ezn);
                fwd_receivers<W>(g, i, t, j0, slot, sh, ezn, rc, re);
#pragma unroll
                for (int k = 0; k < W + 2; ++k) ezc[k] = B.en[k];
#pragma unroll
                for (int w = 0; w < W; ++w) hyu[w] = hyn[w];
            } else if (live) {
                const long long go = (long long)grp * g.plane;
                float* hs = g.hist ? g.hist + (((long long)(t - g.hist_t0) * g.ngroups + grp) * nx) * hrow +
                                         (long long)j0 * 32 + l
                                   : nullptr;
                fwd_row<W, 32>(g, R, band_fwd<W>(g, j0), B, ezc, hyu, i, t, j0, l, slot, sh, bcore, g.ez[wp] + go,
                               g.hx[wp] + go, g.hy[wp] + go, hs, hrow, psi_group(g, rp, grp), psi_group(g, wp, grp), sc,
                               se, rc, re);
            }
            pe += rowS;
            px += rowS;
            py += rowS;
            if (ph) ph += hrow;
        }
    }
}

// ---------------------------------------------------------------------------
// Reference-mode adjoint step
// ---------------------------------------------------------------------------
template <int W, int C>
__device__ __forceinline__ void band_adj_producer(const Dev& g, BandProducer& pr, unsigned char* stages,
                                                  size_t stage_bytes, int* ctr, int rp, int it) {
    using G = BandGeom<W, C>;
    const long long rowS = (long long)g.P * 32;
    const int nx = g.nx;
    for (;;) {
        int id = 0;
        const int4 T = band_next_tile(g, ctr, id);
        int slot;
        if (!pr.claim(g, slot)) return;
        float* st = reinterpret_cast<float*>(stages + (size_t)slot * stage_bytes);
        BandHead* h = reinterpret_cast<BandHead*>(st);
        uint64_t* bar = pr.full + slot;
        h->tile = T;
        if (T.x < 0) {
            mbar_expect_tx(bar, 0);
            ++pr.qi;
            return;
        }
        const int b0 = T.x, i0 = T.y, i1 = T.z, grp = T.w;
        h->ev = make_int4(__ldg(g.inj_off + id), __ldg(g.inj_off + id + 1), 0, 0);
        const long long go = (long long)grp * g.plane;
        const float* ez = g.ez[rp] + go + (long long)(b0 + PADC) * 32;        // cell (0, b0)
        const float* hx = g.hx[rp] + go + (long long)(b0 - 1 + PADC) * 32;    // cell (0, b0-1)
        const float* hy = g.hy[rp] + go + (long long)(b0 + PADC) * 32;
        const float* hs = g.hist + (((long long)(it - g.hist_t0) * g.ngroups + grp) * nx * g.Ph + b0) * 32;
        const uint32_t hbytes = b0 < g.Ph ? (uint32_t)min(G::BC, g.Ph - b0) * 128 : 0u;
        // E operands of row r (none for the frame row r = nx)
        auto e_row = [&](auto&& f, float* s2, int r) {
            if (r >= nx) return;
            const long long crow = (long long)r * g.P + b0 + PADC;
            f(s2 + G::A_EZ, ez + r * rowS, (G::BC + 1) * 128);
            f(s2 + G::A_HX, hx + r * rowS, (G::BC + 2) * 128);
            f(s2 + G::A_HY, hy + r * rowS, (G::BC + 1) * 128);
            f(s2 + G::A_CA, g.ca + crow, (G::BC + 4) * 4);
            f(s2 + G::A_CB, g.cb + crow, (G::BC + 4) * 4);
        };
        // head: E operands of row i0 and Hy of row i0-1
        issue_stage(g, bar, [&](auto&& f) {
            e_row(f, st, i0);
            if (i0 >= 1) f(st + G::A_HU, hy + (i0 - 1) * rowS, (G::BC + 1) * 128);
        });
        if (g.pf && g.th > 0) prefetch_tile_psi<32>(g, grp, rp, i0, i0, b0, b0 + G::BC);
        ++pr.qi;
        for (int i = i0; i < i1; ++i) {
            if (!pr.claim(g, slot)) return;
            st = reinterpret_cast<float*>(stages + (size_t)slot * stage_bytes);
            bar = pr.full + slot;
            issue_stage(g, bar, [&](auto&& f) {
                e_row(f, st, i + 1);
                f(st + G::A_HS, hs + (long long)i * g.Ph * 32, hbytes);
                f(st + G::A_CH, g.ch + (long long)i * g.P + b0 + PADC, G::BC * 4);
            });
            if (g.pf && g.th > 0) prefetch_tile_psi<32>(g, grp, rp, i + 1, i + 1, b0, b0 + G::BC);
            ++pr.qi;
        }
    }
}

// E operands of row r for this warp's cells j0 .. j0+W (stage layout A_*).
template <int W, int C>
__device__ __forceinline__ void band_adj_e_in(const float* st, int cw, int l, AdjEIn<W>& A) {
    using G = BandGeom<W, C>;
    const float* sz = st + G::A_EZ + cw * 32 + l;
#pragma unroll
    for (int k = 0; k <= W; ++k) {
        A.ez[k] = sz[k * 32];
        A.hyo[k] = sz[G::A_HY - G::A_EZ + k * 32];
    }
#pragma unroll
    for (int k = 0; k < W + 2; ++k) A.hxo[k] = sz[G::A_HX - G::A_EZ + k * 32];
    lds_run<W>(A.ca, st + G::A_CA + cw);
    lds_run<W>(A.cb, st + G::A_CB + cw);
    A.ca[W] = st[G::A_CA + cw + W];
    A.cb[W] = st[G::A_CB + cw + W];
}

template <int W, int C>
__global__ void __launch_bounds__(32 * (C + 1), band_min_blocks<C>()) k_adj_band(const Dev g, const int it, const int rp, const int D) {
    using G = BandGeom<W, C>;
    extern __shared__ __align__(128) unsigned char smem[];
    const BandSmem L(g.th, D, G::ADJ);
    float* R = reinterpret_cast<float*>(smem + L.prof);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.bars);
    uint64_t* empty = full + D;
    volatile int* flags = reinterpret_cast<volatile int*>(smem + L.flag);
    unsigned char* stages = smem + L.stages;
    if (abort_launch(g, flags)) return;
    if (threadIdx.x == 0) {
        flags[1] = 0;
        for (int s = 0; s < D; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, C);
        }
        fence_mbar_init();
        if (blockIdx.x == 0) g.tile_ctr[rp ^ 1] = 0;   // the next launch's counter
    }
    for (int k = threadIdx.x; k < 8 * g.th; k += blockDim.x) R[k] = __ldg(g.pml + k);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wp = rp ^ 1;
    if (warp == C) {
        if (lane == 0) {
            BandProducer pr;
            pr.full = full;
            pr.empty = empty;
            pr.stop = flags + 1;
            pr.D = D;
            band_adj_producer<W, C>(g, pr, stages, L.stage, g.tile_ctr + rp, rp, it);
            pr.drain();
        }
        return;
    }
    const int nx = g.nx, ny = g.ny, th = g.th;
    const int l = lane, cw = warp * W;
    int s = 0;
    uint32_t par = 0;
    auto next = [&]() {
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + s);
        if (++s == D) {
            s = 0;
            par ^= 1u;
        }
    };
    for (;;) {
        if (!wait_or_stop(g, full + s, par, flags + 1)) return;
        const float* st = reinterpret_cast<const float*>(stages + (size_t)s * L.stage);
        const BandHead hd = *reinterpret_cast<const BandHead*>(st);
        if (hd.tile.x < 0) return;
        const int b0 = hd.tile.x, i0 = hd.tile.y, i1 = hd.tile.z, grp = hd.tile.w;
        const int j0 = b0 + cw, slot = l, sh = grp * 32 + l;
        // the CPML geometry (rd, wr, by) is rebuilt where a row needs it, so
        // it holds no registers across the march
        // E at columns j0 .. j0+W (incl. the halo) and H at j0 .. j0+W-1 are interior cells
        const bool bcore = j0 >= th + 1 && j0 + W <= ny - th - 1;
        int ic = hd.ev.x;
        const int ie = hd.ev.y;
        const long long resid_o = ((long long)sh * g.nt + it) * g.nrx;
        const bool hist_ok = j0 < g.Ph;
        // warps whose cells lie beyond the grid (the last band) only release stages
        const bool live = j0 < ny;

        // new E of row i0 (own), with the old H of rows i0-1 and i0; eoc keeps
        // the old Ez of the row (before the residual injection)
        float ezc[W + 1], hxc[W + 2], hyc[W + 1], eoc[W];
        {
            float hyu[W + 1];
            AdjEIn<W> A;
            band_adj_e_in<W, C>(st, cw, l, A);
#pragma unroll
            for (int k = 0; k <= W; ++k) hyu[k] = i0 >= 1 ? st[G::A_HU + (cw + k) * 32 + l] : 0.f;
            next();
#pragma unroll
            for (int w = 0; w < W; ++w) eoc[w] = A.ez[w];
            if (live)
                adj_e_row<W, 32>(g, R, band_adj<W>(g, j0), A, i0, j0, l, slot,
                                 bcore && i0 >= th + 1 && i0 <= nx - th - 1, true, hyu, ezc, resid_o, ic, ie,
                                 psi_group(g, rp, grp), psi_group(g, wp, grp));
#pragma unroll
            for (int k = 0; k < W + 2; ++k) hxc[k] = A.hxo[k];
#pragma unroll
            for (int k = 0; k <= W; ++k) hyc[k] = A.hyo[k];
        }
        // interior rows of an interior band take the lean path (E of row i+1
        // and H of row i both away from the CPML and the frame): the updates
        // of adj_e_core / adj_h_core, stores and accumulators through row
        // pointers advanced row by row
        const bool wcore = live && bcore;
        const long long rowS = (long long)g.P * 32;
        const long long o0 = (long long)grp * g.plane + ((long long)i0 * g.P + j0 + PADC) * 32 + l;
        float* pe = g.ez[wp] + o0;
        float* px = g.hx[wp] + o0;
        float* py = g.hy[wp] + o0;
        double* ge_row = g.gacc + (long long)grp * 2 * ((long long)nx * ny) + (long long)i0 * ny + j0;
        double* gs_row = ge_row + (long long)nx * ny;
        for (int i = i0; i < i1; ++i) {
            if (!wait_or_stop(g, full + s, par, flags + 1)) return;
            st = reinterpret_cast<const float*>(stages + (size_t)s * L.stage);
            AdjEIn<W> A;
            float ch[W], f1[W];
            if (i + 1 < nx) band_adj_e_in<W, C>(st, cw, l, A);
            lds_run<W>(ch, st + G::A_CH + cw);
            const float* sh1 = st + G::A_HS + cw * 32 + l;
#pragma unroll
            for (int w = 0; w < W; ++w) f1[w] = hist_ok ? sh1[w * 32] : 0.f;
            next();
            if (wcore && i >= th + 1 && i + 1 <= nx - th - 1) {
                float eor[W], ezr[W + 1], hx[W], hy[W];
#pragma unroll
                for (int w = 0; w < W; ++w) eor[w] = A.ez[w];
                adj_inject<W>(g, A.ez, i + 1, j0, slot, resid_o, ic, ie);
                adj_e_core<W>(A, hyc, ezr);
                adj_h_core<W>(ch, ezc, ezr, hxc, hyc, hx, hy);
                adj_image<W, true>(g, f1, ezc, eoc, ge_row, gs_row, j0, lane);
                st_cells<W, 32>(g, pe, ezc);
                st_cells<W, 32>(g, px, hx);
                st_cells<W, 32>(g, py, hy);
#pragma unroll
                for (int k = 0; k <= W; ++k) {
                    ezc[k] = ezr[k];
                    hyc[k] = A.hyo[k];
                }
#pragma unroll
                for (int w = 0; w < W; ++w) eoc[w] = eor[w];
#pragma unroll
                for (int k = 0; k < W + 2; ++k) hxc[k] = A.hxo[k];
            } else if (live) {
                const long long go = (long long)grp * g.plane;
                double* gae = g.gacc + (long long)grp * 2 * ((long long)nx * ny);
                adj_row<W, true>(g, R, band_adj<W>(g, j0), A, ch, f1, ezc, hxc, hyc, eoc, i, i1, j0, l, slot, lane,
                                 bcore, resid_o, ic, ie, psi_group(g, rp, grp), psi_group(g, wp, grp), g.ez[wp] + go,
                                 g.hx[wp] + go, g.hy[wp] + go, gae, gae + (long long)nx * ny);
            }
            pe += rowS;
            px += rowS;
            py += rowS;
            ge_row += ny;
            gs_row += ny;
        }
    }
}

}  // namespace fg
