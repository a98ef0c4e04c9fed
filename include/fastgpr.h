/*
 * fastgpr.h -- C ABI of the B200 TMz FDTD library (libfastgpr.so).
 *
 * One shared library replaces the six the reference builds from
 * src/lib/*.cu and binds through ctypes (src/__init__.py:30-221).  Where the
 * reference launches 12 kernels and 10 device-wide synchronisations per time
 * step from Python, this ABI takes a whole solve per call:
 *
 *   fg_coefficients       replaces Ucget / Ucgeta          (src/lib/uc.cu:48, :94)
 *   fg_forward            replaces, per time step, launch_store_outputs
 *                         (sourcereceiver.cu:40), h_fields_updates
 *                         (fields_updates_gpu.cu:80), order1_* H
 *                         (pml_updates_h.cu:84-661), e_fields_updates
 *                         (fields_updates_gpu.cu:35), order1_* E
 *                         (pml_updates_e.cu:80-633), update_hertzian_dipole
 *                         (sourcereceiver.cu:89) and the Ez history copy
 *                         (src/compute.py:712) -- the loop of compute.py:574-712
 *   fg_adjoint_reference  replaces back_source (back.cu:39), the reversed
 *                         update launches and the imaging/normalisation torch
 *                         ops -- the loop of compute.py:1048-1180
 *
 * Conventions
 *   - All array arguments are device pointers unless marked HOST.
 *   - Every call is queued on the given stream (cudaStream_t passed as
 *     void*; NULL = legacy default stream) and returns an FG_* status.  The
 *     solves return without waiting; the calls that wait for their stream are
 *     fg_plan_bind (the plan's tables must stay valid until uploaded),
 *     fg_total_variation with iters != NULL (it returns the iteration count),
 *     fg_plan_check and
 *     fg_forward_static when it uploads a plan's tables (see there); the first
 *     bind of a cell size on a device also runs its division check and waits
 *     for it.  fg_last_error() gives the message of the most recent failure
 *     on the calling thread.
 *   - The caller owns every buffer.  A plan owns only host-side tables; its
 *     device scratch (fields, CPML auxiliaries, event tables, gradient
 *     accumulators) lives in a caller-allocated workspace of
 *     fg_plan_workspace_bytes() bytes bound with fg_plan_bind().
 *   - Distinct plans may be used concurrently from different threads; one
 *     plan must not run two solves at once (they share its workspace).
 */
#ifndef FASTGPR_H
#define FASTGPR_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FG_OK 0
#define FG_ERR_INVALID 1     /* bad argument, shape or position */
#define FG_ERR_CUDA 2        /* a CUDA runtime call failed */
#define FG_ERR_WORKSPACE 3   /* workspace missing or too small */
#define FG_ERR_TIMEOUT 4     /* a bounded device-side wait gave up */

/* Geometry of one model solved for `shots` shots (the reference's `step`
 * batch).  Mirrors FDTDGrid after initialization() (src/compute.py:726-872). */
typedef struct fg_problem {
    int32_t nx, ny;        /* compute grid: reference G.nx (axis 0), G.ny (axis 1) */
    int32_t shots;         /* G.step */
    int32_t nt;            /* G.iterations */
    int32_t th;            /* CPML cells on each side, 0 = no CPML (G.pmlthick) */
    float dx;              /* cell size (dx == dy), float32 as the kernels see it */
    float dt;              /* time step, float32 */
    int32_t nsrc, nrx;     /* sources / receivers per shot */
    const int32_t* src;    /* HOST (shots, nsrc, 3) cell indices (i, j, k), G.source */
    const int32_t* rx;     /* HOST (shots, nrx, 3) cell indices, G.receiver */
    const float* srcw;     /* HOST (nsrc, nt) waveform times dl/(dx dy dz) */
    const float* pml;      /* HOST (8, th) ERA ERB ERE ERF HRA HRB HRE HRF, or NULL if th == 0 */
} fg_problem;

/* Launch shape (all zero or NULL = defaults chosen from the problem).  A tile
 * is (shot group, row chunk, column band); each thread owns `cells_per_thread`
 * consecutive columns of one shot. */
typedef struct fg_tuning {
    int32_t lanes;             /* 0 = choose (shot lanes when shots >= 8), 1 = shot lanes: the 32
                                  lanes of a warp are 32 shots of the same cells, 2 = column
                                  lanes: one shot per warp, lanes own consecutive columns,
                                  3 = shot pairs: 64 shots of the same cells, two per lane
                                  (lane march only, cells_per_thread 2 or 4, no stages) */
    int32_t cells_per_thread;  /* 2, 4 or 8 (default 4 with shot lanes, 2 with column lanes) */
    int32_t rows_per_tile;     /* rows of one tile, >= 1 (default 4; 2 for the shot-lane
                                  lane march below 1.2e5 cells x shot groups) */
    int32_t warps_per_block;   /* 1, 2 or 4 (default 4) */
    int32_t stages;            /* lane march: 0 = operands loaded into registers row by row;
                                  2..8 = a ring of this many rows per warp in shared memory,
                                  filled ahead by bulk copies (shot lanes need cells_per_thread >= 4) */
    int32_t kernel;            /* 0 = tensor-map tile pipeline: persistent CTAs of rows_per_tile
                                  (2/4/8) consumer warps and one producer warp that fetches tiles
                                  by cp.async.bulk.tensor into `stages` (2..4, default 3)
                                  shared-memory stages; cells_per_thread 4/8 (shot lanes) or 2/4
                                  (column lanes); 1 = lane march (persistent warps).  With no
                                  kernel, stages, rows or cells given, shot lanes take the lane
                                  march and column lanes the tile pipeline. */
    /* The adjoint runs on a plan of its own (own state and accumulators); its
     * launch shape: adj_kernel 0 = the forward's shape when the fields above
     * name one, else the default adjoint shape (shot lanes: lane march with
     * 8 cells per thread over 4 rows -- 4 cells when nx * ny * shot groups is
     * below 2e5; column lanes: the forward's);
     * 1 = tile pipeline, 2 = lane march, shaped by the three fields below
     * (0 = their defaults).  lanes is shared; adj_cells_per_thread (0 = the
     * forward's cells_per_thread) sets the adjoint's own.  The Ez history
     * layout does not depend on cells_per_thread, so the two may differ. */
    int32_t adj_kernel;
    int32_t adj_rows_per_tile;
    int32_t adj_warps_per_block;
    int32_t adj_stages;
    int32_t adj_cells_per_thread;
    /* Lane march with shot lanes and no stages (forward and adjoint): each
     * warp prefetches into L2 the rows of the tile it will take next, so the
     * loads of that tile find their lines in L2 instead of waiting for HBM.
     * 0 = default (1; off where the interior split runs, beside which it
     * only competes for bandwidth), -1 = off, 1 = when the warp starts its
     * current tile, 2 = at the current tile's middle row. */
    int32_t prefetch;
    /* Lane march with shot lanes and no stages: the interior tiles (no CPML
     * cell in the tile or its halo, no source, receiver or injection) run in
     * a lean kernel of their own, side by side with the general kernel on the
     * other tiles.  -1 = off; 0 = default (on when nx * ny * shot groups is
     * at least 12,000 -- smaller steps do not pay for the extra launches --
     * and persistent is not 1, with the general kernel at 3 blocks per SM);
     * 1..8 = on, the general kernel with that many blocks per SM. */
    int32_t interior;
    /* Lane march without stages or shot pairs: the whole time loop of a
     * solve in one persistent cooperative launch, the steps separated by a
     * grid barrier, instead of one launch per step; needed by the batch calls
     * below.  0 or -1 = off (default), 1 = on (the lane march also for column
     * lanes when no kernel is given).  A step then costs the serial latency
     * of one warp's tile plus about 2.4 us of barrier, so on small grids it
     * is no faster than a launch per step; several models in one launch
     * (fg_forward_batch) fill the GPU better than one. */
    int32_t persistent;
    /* With the interior split: the slab tiles (in one CPML slab, no event)
     * run in a lean kernel of their own between the general and the interior
     * kernel.  -1 = off (they stay in the general kernel); 0 = default (the
     * forward's on with at most 2 blocks per SM; the adjoint's with at most
     * 2 blocks per SM when nx * ny * shot groups is below 50,000, 1 below
     * 120,000, off above); 1..8 = on for both, at most that many blocks per
     * SM. */
    int32_t slab;
} fg_tuning;

typedef struct fg_plan fg_plan;

/* Build a plan (host tables only).  Positions with k != 0, i == nx or
 * j == ny address the reference's dead plane / zero frame and are kept as
 * inert (traces read 0, injections are dropped); negative or larger indices
 * are rejected with FG_ERR_INVALID. */
int fg_plan_create(const fg_problem* prob, const fg_tuning* tune, fg_plan** out);
int fg_plan_destroy(fg_plan* plan);
/* Shape of the Ez history buffer fg_forward writes and fg_adjoint_reference
 * reads: shape = {nt, groups, nx, pitch, slots}, float32, last index fastest.
 * Ez after step t of shot s at cell (i, j) is element
 * [t][s / slots][i][j][s % slots]; columns j >= ny and slots of shots >= the
 * solve's count are padding.  The buffer holds the product of the five
 * extents in floats. */
int fg_plan_hist_shape(const fg_plan* plan, int64_t shape[5]);
/* Device scratch a plan needs (its own and its adjoint plan's), in bytes
 * (>= 0), or -1 on a NULL plan. */
int64_t fg_plan_workspace_bytes(const fg_plan* plan);
/* The launch shape a plan chose (host-side, no device work): FG_SHAPE_FIELDS
 * int32 values, the forward's nine and then the adjoint's nine, each
 *   kernel (0 tile pipeline, 1 lane march, 2 band pipeline), lanes (1 shot
 *   lanes, 2 column lanes, 3 shot pairs), cells_per_thread, rows_per_tile,
 *   warps_per_block, stages, interior split (1 = the interior tiles run in
 *   their own kernel), slab kernel (its blocks per SM, 0 = off),
 *   persistent launch (1 = the whole time loop in one launch). */
#define FG_SHAPE_FIELDS 18
int fg_plan_shape(const fg_plan* plan, int32_t* out);
/* Attach a workspace (256-byte aligned device memory of at least
 * fg_plan_workspace_bytes bytes) and upload the plan's tables into it. */
int fg_plan_bind(fg_plan* plan, void* workspace, int64_t bytes, void* stream);

/* Per-cell update coefficients, the reference's Ucget (adjoint == 0) or
 * Ucgeta (adjoint != 0) (src/lib/uc.cu:11-45, :60-91).  er, se, mr: (nx, ny)
 * float32 row-major.  out: 5 planes of (nx+1, pitch) float32 -- uE0, uE1,
 * uE4, uH1, uH4 -- zero on the i == nx / j >= ny frame. */
int fg_coefficients(const float* er, const float* se, const float* mr, int32_t nx, int32_t ny,
                    float dt, float dx, int32_t adjoint, float* out, int32_t pitch, void* stream);

/* Forward solve (compute.py:574-712).  er, se, mr: (nx, ny) float32.
 * traces: (shots, nt, nrx) float32, Ez at each receiver at the start of each
 * step.  hist: Ez after each step in the layout of fg_plan_hist_shape, or
 * NULL. */
int fg_forward(fg_plan* plan, const float* er, const float* se, const float* mr,
               float* traces, float* hist, void* stream);

/* Reference-mode adjoint (compute.py:1048-1180): the forward operator run in
 * reverse time with Ucgeta's uE0, the raw residual injected at the receivers,
 * and the imaging sums g_eps = sum_t,s (Ez[t]-Ez[t-1]) lambda and
 * g_sig = sum_t,s Ez[t] lambda dt.  resid: (shots, nt, nrx) float32; hist
 * from fg_forward.  grad_eps / grad_sig: (nx, ny) float32 outputs, either may
 * be NULL.  normalize != 0 divides each by its L2 norm as the reference does;
 * norms (HOST-visible is not required: device double[2]) receives the two L2
 * norms when not NULL. */
int fg_adjoint_reference(fg_plan* plan, const float* er, const float* se, const float* mr,
                         const float* hist, const float* resid, float* grad_eps, float* grad_sig,
                         int32_t normalize, double* norms, void* stream);

/* fg_adjoint_reference for the L1 misfit of the multiscale inversion
 * (example.ipynb's L1Loss feeding back.cu): instead of a residual tensor,
 * the synthetic traces (fg_forward's) and the observed ones, both
 * (shots, nt, nrx) float32; the value injected at receiver r of shot s at
 * step t is scale * sign(traces - observed) with sign(0) = 0, formed inside
 * the adjoint step -- the gradient of scale * sum |traces - observed|
 * (scale = 1 / (shots * nt * nrx), rounded to float32, for the mean). */
int fg_adjoint_reference_l1(fg_plan* plan, const float* er, const float* se, const float* mr, const float* hist,
                            const float* traces, const float* observed, float scale, float* grad_eps,
                            float* grad_sig, int32_t normalize, double* norms, void* stream);

/* Exact discrete adjoint of fg_forward: the gradient of
 * J = sum_{s,t,r} weights[s][t][r] * traces[s][t][r] with respect to the
 * relative permittivity and the conductivity of every cell, for traces as
 * fg_forward returns them (the CPML profile held fixed).  No counterpart in
 * the reference, whose gradient (compute.py:1020-1180, back.cu:8-37) runs the
 * forward operator in reverse time with Ucgeta's coefficients and the raw
 * residual, and so is not the derivative of anything: this call transposes
 * every step of the forward loop (H and E leapfrog, both CPML phases), runs
 * the transposed steps from the last step back to the first with the weights
 * injected at the receivers, and forms dJ/d eps_r and dJ/d sigma from the
 * derivatives of Ucget's E coefficients.  er, se, mr and hist as for
 * fg_adjoint_reference (hist from fg_forward); weights: (shots, nt, nrx)
 * float32 (a loss's gradient with respect to the traces); grad_eps /
 * grad_sig: (nx, ny) float32, either may be NULL.  Not normalised.  Runs on
 * the plan's adjoint state (like fg_adjoint_reference). */
int fg_adjoint_exact(fg_plan* plan, const float* er, const float* se, const float* mr, const float* hist,
                     const float* weights, float* grad_eps, float* grad_sig, void* stream);

/* Replace the CPML profile of a plan (and of its adjoint plan) -- the 8*th
 * floats of fg_problem.pml, HOST -- keeping its tables, workspace and launch
 * shape.  The profile is the only part of a plan that depends on the model
 * (HORIPML averages the first row of eps_r, src/compute.py:267-313), so an
 * inversion whose model changes keeps its plan, buffers and captured CUDA
 * graphs.  A bound plan's copy in the workspace is updated on `stream`
 * (pageable-memory copy: pml may be reused when the call returns). */
int fg_plan_set_profile(fg_plan* p, const float* pml, void* stream);

/* Several models in one launch: no counterpart in the reference, which
 * solves one model per call.  fg_forward_batch runs fg_forward for plans[0..n)
 * -- models of any grid, shot count and step count -- with every time step of
 * all of them in one persistent launch (the warps take each model's tiles of
 * a step in turn, a grid barrier separates the steps, a model whose steps
 * are done sits out); fg_adjoint_reference_batch does the same for
 * fg_adjoint_reference (each model's gradient normalised on its own when
 * normalize != 0).  Every plan must be bound, use the persistent lane march
 * (fg_tuning.persistent = 1) and share
 * lanes and cells_per_thread; at most FG_BATCH_MAX plans.  The arrays hold one
 * pointer per model with the meaning of the single-model calls.  Results
 * equal the single-model calls' bit for bit. */
#define FG_BATCH_MAX 8
int fg_forward_batch(fg_plan* const* plans, int32_t n, const float* const* er, const float* const* se,
                     const float* const* mr, float* const* traces, float* const* hist, void* stream);
int fg_adjoint_reference_batch(fg_plan* const* plans, int32_t n, const float* const* er, const float* const* se,
                               const float* const* mr, const float* const* hist, const float* const* resid,
                               float* const* grad_eps, float* const* grad_sig, int32_t normalize, void* stream);

/* Checkpointed solve, for histories that do not fit in device memory (the
 * reference keeps the whole Ez history, src/compute.py:553, which limits it
 * to nt * shots * nx * ny * 4 bytes of HBM).  fg_forward_checkpointed runs the
 * forward solve and saves the state (fields and CPML auxiliaries) at the
 * start of every `interval`-th step instead of the history;
 * fg_adjoint_reference_checkpointed then walks the segments backwards:
 * it restores a segment's checkpoint, recomputes that segment's Ez history
 * into `segment` (interval steps in the layout of fg_plan_hist_shape, i.e.
 * interval * groups * nx * pitch * slots floats) and runs the segment's
 * adjoint steps.  One extra forward solve of work; traces, gradients and
 * norms are bit-identical to fg_forward + fg_adjoint_reference.  ckpt: device
 * memory of fg_plan_checkpoint_bytes(plan, interval) bytes (may be 0 when
 * interval >= nt), 16-byte aligned.  The adjoint call uses the plan's
 * forward state as scratch, so the two calls of one solve must not overlap
 * with other solves on the same plan. */
int64_t fg_plan_checkpoint_bytes(const fg_plan* plan, int32_t interval);
int fg_forward_checkpointed(fg_plan* plan, const float* er, const float* se, const float* mr, float* traces,
                            void* ckpt, int64_t ckpt_bytes, int32_t interval, void* stream);
int fg_adjoint_reference_checkpointed(fg_plan* plan, const float* er, const float* se, const float* mr,
                                      const void* ckpt, int64_t ckpt_bytes, int32_t interval, float* segment,
                                      const float* resid, float* grad_eps, float* grad_sig, int32_t normalize,
                                      double* norms, void* stream);

/* Forward solve that allocates no device memory: no counterpart in the
 * reference (whose launchers take buffers allocated by torch).
 *
 * For callers that cannot call cudaMalloc: cudaMalloc and cudaFree may
 * synchronise the whole device, which a host loop driving other streams in
 * real time cannot afford, and some host applications hand all device memory
 * to their own pool up front, leaving nothing for a library to allocate.
 * Such a caller still allocates the inputs and outputs (er, se, mr, traces,
 * hist, exactly as for fg_forward) and builds the plan with fg_plan_create,
 * which touches host memory only; this call then runs fg_forward with the
 * plan's device scratch placed in one array of FG_STATIC_SCRATCH_BYTES that
 * the library holds in device memory of every GPU that loads it, until the
 * process exits.  The plan's own workspace binding (fg_plan_bind), if any,
 * is left as it was.
 *
 *   - A plan whose forward scratch exceeds FG_STATIC_SCRATCH_BYTES is
 *     rejected with FG_ERR_WORKSPACE before any device work.  That is the
 *     forward plan's own share of fg_plan_workspace_bytes (which also counts
 *     the adjoint plan's scratch), so a plan whose workspace bytes exceed the
 *     array may still fit.
 *   - The first call on a device looks up the array's device address (with
 *     that device current) and keeps it; make that first call before any
 *     stream capture.
 *   - When the array of the device does not hold this plan's tables (the
 *     plan's first call there, or another plan called in between), the call
 *     uploads them and waits for `stream` (as fg_plan_bind does); otherwise
 *     it only queues the solve.
 *   - Every call on a device shares the one array and the array keeps what
 *     the last call left in it; each call clears the field state it needs.
 *     Calls whose work overlaps on the GPU (other streams, other threads)
 *     race on the array: serialise them.
 *   - Device-side error words of the checked build land in the array, not in
 *     the plan's workspace, so fg_plan_check does not see them. */
#define FG_STATIC_SCRATCH_BYTES (32LL * 1024 * 1024)
int fg_forward_static(fg_plan* plan, const float* er, const float* se, const float* mr,
                      float* traces, float* hist, void* stream);

/* Causal FIR filter of the multiscale inversion (reference
 * src/multiscale.py:19-53, apply_filter): x is (batch, T, R) float32 with
 * the time axis T in the middle and R innermost -- the layout of the traces
 * fg_forward returns, (shots, nt, nrx); a single series is batch = R = 1.
 * Each series is reflect-padded by k-1 samples on the left and
 * cross-correlated with the k taps:
 *   out[b][t][r] = sum_m taps[m] * x[b][|t + m - (k-1)|][r].
 * taps: device float32[k], 1 <= k <= 8192 and k - 1 < T; out must not
 * overlap x.  Float32 sum over m in order with fused multiply-adds. */
int fg_fir_causal(const float* x, int64_t batch, int32_t T, int32_t R, const float* taps, int32_t k, float* out,
                  void* stream);

/* Total-variation denoising of an (M, N) float32 model (reference
 * src/tv.py:135-217, the regulariser of the default gradient,
 * src/compute.py:916-933): ADMM on the model scaled by 1/(max + 1e-6) with a
 * one-cell zero border, at most num_iter iterations, stopping when the
 * update's L2 norm drops below tol; out = the result times max(data).  Each
 * iteration repeats the float32 arithmetic of the reference's tensor
 * operations; the convergence norm is summed in float64.  data, out and
 * workspace are device memory (workspace: fg_tv_workspace_bytes(M, N) bytes,
 * 256-byte aligned, not overlapping data or out).  One cooperative launch on
 * `stream`; with iters != NULL the call then waits for `stream`, *iters
 * (host) receives the iteration count, and FG_ERR_TIMEOUT is returned if a
 * device-side barrier gave up.  With iters == NULL the call only enqueues
 * (it may be captured in a CUDA graph) and reports neither. */
int64_t fg_tv_workspace_bytes(int32_t M, int32_t N);
int fg_total_variation(const float* data, int32_t M, int32_t N, double lamda, double rho, int32_t num_iter,
                       double tol, float* out, void* workspace, int64_t bytes, int32_t* iters, void* stream);

/* Wait for the plan's work on `stream`, then read and clear the device-side
 * error word its kernels set (an out-of-range access caught by the checked
 * build, or a bounded wait that gave up).  Returns FG_OK, FG_ERR_TIMEOUT or
 * FG_ERR_INVALID.  This is the only call that synchronises. */
int fg_plan_check(fg_plan* plan, void* stream);

/* Message of the last failing call on this thread ("" if none). */
const char* fg_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* FASTGPR_H */
