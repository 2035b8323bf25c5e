/*
 * dtb.h - C ABI of libdtb.so, a B200 (sm_100a) backend for the explicit Euler path of
 * DiplodocusTransport.jl.
 *
 * The ABI is what a Julia `ccall` binds: plain pointers and sizes, 0 on success, an error
 * code otherwise, never a C++ exception. Host arrays are owned by the caller and are only
 * read or written during the call; the library copies everything it keeps into device
 * memory it owns and frees in dtb_destroy. Calls on one context must be serialised by
 * the caller; separate contexts may be used from separate threads.
 *
 * Each entry point names the reference interface it replaces (paths are relative to
 * the DiplodocusTransport.jl project).
 */
#ifndef DTB_H
#define DTB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DTB_ABI_VERSION 1

/* status codes */
#define DTB_OK 0
#define DTB_EINVAL 1   /* bad argument or inconsistent sizes */
#define DTB_ENOMEM 2   /* device allocation failed or the HBM budget is exceeded */
#define DTB_ECUDA 3    /* a CUDA runtime call failed (see dtb_last_error) */
#define DTB_ETIMEOUT 4 /* a bounded device-side wait gave up; the context stays usable */
#define DTB_ESTATE 5   /* call out of order (e.g. a step before any operator was uploaded) */
#define DTB_ENODEV 6   /* no usable CUDA device */
#define DTB_ENOTFOUND 7 /* unknown slot / request id */

/* state precision (Main.Precision, SteppingStructs.jl:36-38) */
#define DTB_F64 0       /* Float64 state and operators */
#define DTB_F32 1       /* Float32 state and operators (the reference's CUDA precision, Backends.jl:12) */
#define DTB_MIXED 2     /* batched: G, the loss rows and E as BF16 hi+lo with per-row scales (FP32
                           accumulation on the tensor cores), f in FP32, FP64 compensated update
                           and moments */

/* dtb_opts.flags */
#define DTB_FLAG_SYMPLECTIC 1  /* ForwardSymplecticEulerStruct (SteppingStructs.jl:104-229):
                                  momentum update, then space update (SteppingMethods.jl:120-243) */
#define DTB_FLAG_NO_AUTOTUNE 2 /* batched contexts: plan the gain GEMM by a fixed rule instead of
                                  timing the candidate plans on the device at commit */

/* flux parts (FluxMatricesStruct.X_Flux / P_Flux, StructsAndDictionaries.jl:346-347) */
#define DTB_FLUX_X 0
#define DTB_FLUX_P 1

/* element type tags for uploads */
#define DTB_DTYPE_F64 0
#define DTB_DTYPE_F32 1

#define DTB_MAX_SPECIES 16

typedef struct dtb_ctx dtb_ctx;

/* Grid description: the part of PhaseSpaceStruct (StructsAndDictionaries.jl:290) the step reads. */
typedef struct dtb_dims {
    int32_t n_species;                       /* length(name_list) */
    int32_t n_space;                         /* x_num * y_num * z_num */
    int64_t species_size[DTB_MAX_SPECIES];   /* px_num * py_num * pz_num per species */
} dtb_dims;

typedef struct dtb_opts {
    int32_t precision;     /* DTB_F64, DTB_F32 or DTB_MIXED */
    int32_t device;        /* CUDA device ordinal */
    void* stream;          /* cudaStream_t to run on, or NULL for a library-owned stream */
    int32_t index_base;    /* base of sparse indices the caller passes: 1 (Julia) or 0 */
    int32_t graph_steps;   /* steps per captured CUDA graph (at most 1024). 0: the default, for
                              plain contexts 64 when the step records of 64 steps fit in 8 MB
                              (grids up to about 175,000 states) and 16 above; 16 for batched ones */
    double dt0;            /* TimeStruct.dt0 (StructsAndDictionaries.jl:55) */
    int32_t batch;         /* instances per context; 1 for the plain method */
    int32_t flags;         /* reserved, 0 */
} dtb_opts;

/* Per-step diagnostics of the functor (SteppingMethods.jl:48-94). */
typedef struct dtb_step_diag {
    double cr;        /* Cr = -min(df ./ f), NaN mapped to Inf; 0 when sum(f) == 0 */
    double cr_bin;    /* Verbose == 3 only: binary part */
    double cr_emi;    /* Verbose == 3 only: emission part */
    double cr_flux;   /* Verbose == 3 only: flux part */
    double sum_df;    /* sum(df) after scaling (FP64 accumulation) */
    double sum_f;     /* sum(f) before the update */
    int32_t finite;   /* isfinite(sum(df)) */
    int32_t pad;
} dtb_step_diag;

/* ---- version / device (host only) ---- */
int32_t dtb_abi_version(void);
const char* dtb_last_error(void);                 /* thread-local message of the last failure */
int32_t dtb_device_count(int32_t* n);

/* ---- construction: ForwardEulerStruct(PhaseSpace, Initial, Injection, BinM, EmiM, FluxM)
 *      (SteppingStructs.jl:33-100) ---- */
int32_t dtb_create(const dtb_dims* dims, const dtb_opts* opts, dtb_ctx** out);
int32_t dtb_destroy(dtb_ctx* ctx);

/* F_Flux += M for a CSC matrix n x n (X_Flux + P_Flux, SteppingStructs.jl:60,68).
 * colptr has n+1 entries; indices use opts.index_base. Call once per matrix to add. */
int32_t dtb_add_flux_csc(dtb_ctx* ctx, int64_t n, const int64_t* colptr, const int64_t* rowval,
                         const double* nzval);

/* Adds X_Flux (part DTB_FLUX_X) or P_Flux (DTB_FLUX_P). The explicit Euler method sums both
 * into F; the symplectic method (DTB_FLAG_SYMPLECTIC) keeps X apart for its space update
 * (SteppingStructs.jl:170-171,188-189). */
int32_t dtb_add_flux_csc_part(dtb_ctx* ctx, int32_t part, int64_t n, const int64_t* colptr,
                              const int64_t* rowval, const double* nzval);

/* Reference-layout M_Bin (n_mom^2 x n_mom, column-major, BuildBinaryMatrices.jl:54) replaces
 * BinM.M_Bin (SteppingStructs.jl:58,66). It is decomposed on upload into gain blocks and
 * loss rows, exactly (no thresholding). */
int32_t dtb_upload_mbin_ref(dtb_ctx* ctx, const double* M_Bin, int64_t n_mom);

/* Blocked gain: df[a] += Vol * sum_{b in in1, c in in2} G[a][b][c] f_b f_c.
 * G is row-major [N_out][N_in1][N_in2] (c fastest); `on_device` != 0 means G is a device
 * pointer (same dtype as the context precision, N_in2 a multiple of 8 and in1 <= in2).
 * Calls for the same (out, in1, in2) add. This is the block GainMatrix_to_M_Bin!
 * (BuildBinaryMatrices.jl:114-204) scatters into M_Bin. */
int32_t dtb_add_gain_block(dtb_ctx* ctx, int32_t out_sp, int32_t in1_sp, int32_t in2_sp,
                           const void* G, int32_t dtype, int32_t on_device);

/* Blocked loss: df[a] -= Vol * f_a * sum_{c in other} L[a][c] f_c; L row-major [N_sp][N_other].
 * The block LossMatrix_to_M_Bin! (BuildBinaryMatrices.jl:206-284) scatters into M_Bin. */
int32_t dtb_add_loss_block(dtb_ctx* ctx, int32_t sp, int32_t other_sp, const double* L);

/* Reference dense M_Emi (n x n column-major, EmissionMatricesStruct, SteppingStructs.jl:59,67);
 * stored as its nonzero (cell, species) blocks. */
int32_t dtb_upload_emi_ref(dtb_ctx* ctx, const double* M_Emi, int64_t n);

/* A dense row-major piece of M_Emi at (row0, col0). Pieces add. */
int32_t dtb_add_emi_block(dtb_ctx* ctx, int64_t row0, int64_t nrows, int64_t col0, int64_t ncols,
                          const double* E);

/* Ap_Flux (diagonal, n), Vol (n_space), Initial (n), Injection (n)
 * (SteppingStructs.jl:53-55,61-64). invAp = 1 ./ Ap is formed in the state precision. */
int32_t dtb_upload_vectors(dtb_ctx* ctx, const double* Ap, const double* Vol,
                           const double* f_init, const double* inj);

/* M_Bin as a sparse matrix (BuildBinaryMatrices.jl:44-52, Bin_sparse = true): CSC of the
 * n_mom^2 x n_mom matrix (colptr n_mom + 1 entries, indices with opts.index_base; duplicate
 * entries are summed like sparse(I, J, V)). Decomposed like dtb_upload_mbin_ref, but the gain
 * part stays sparse: the kernel streams only the nonzero b-rows of each output row, each run
 * of consecutive b-rows trimmed to the c-span of its nonzeros. */
int32_t dtb_upload_mbin_csc(dtb_ctx* ctx, int64_t n_mom, const int64_t* colptr, const int64_t* rowval,
                            const double* nzval);

/* BinM.Domain (StructsAndDictionaries.jl:320, read at SteppingMethods.jl:355-369): the binary
 * term is applied only in the space cells whose 0-based off_space is listed; n < 0 or a NULL
 * list means `nothing` (every cell). Cells outside the domain get a zero binary term, which is
 * what the reference's skipped cells hold for a finite M_Bin. Before dtb_commit. */
int32_t dtb_set_bin_domain(dtb_ctx* ctx, const int64_t* off_space, int64_t n);

/* Builds the device layouts. Called implicitly by the first step; calling it early moves
 * the upload cost out of the first step. */
int32_t dtb_commit(dtb_ctx* ctx);

/* ---- stepping ---- */

/* The ForwardEuler functor (SteppingMethods.jl:12-107): truncates dt at t_stop, advances f
 * by one step. Writes the (possibly truncated) dt and the save flag; when verbose is 1, 2 or
 * 3 also writes the diagnostics (one device->host sync, like the reference's reductions). */
int32_t dtb_step(dtb_ctx* ctx, double t_start, double t_stop, double dt, int32_t verbose,
                 double* dt_out, int32_t* save_out, dtb_step_diag* diag_out);

/* The functor of SteppingMethods.jl:12-107 on a state kept in host memory, as the reference's
 * CPU backend keeps method.f: f_in (n_state values; NULL keeps the device state) is uploaded,
 * the step of dtb_step runs, and the new state is written to f_out (may equal f_in), all with
 * one wait for the whole round trip (dtb_set_f + dtb_step + dtb_get_f make three). Page-locked
 * arrays avoid the driver's staging copies. The diagnostics are written to diag_out when it is
 * not NULL. */
int32_t dtb_step_io(dtb_ctx* ctx, const double* f_in, double* f_out, double t_start, double t_stop,
                    double dt, int32_t verbose, double* dt_out, int32_t* save_out,
                    dtb_step_diag* diag_out);

/* Captures, instantiates and uploads the CUDA graphs that dtb_run (Verbose = 0) or, for a
 * batched context, dtb_batch_run replay, without running a step (commits first if needed).
 * Optional: without it the first run long enough for a graph captures it. A caller that times
 * its steps calls it once beforehand so no capture falls inside the timed steps. No
 * counterpart in the reference (its Julia loop has no graphs). */
int32_t dtb_prepare(dtb_ctx* ctx);

/* nsteps steps with the given dt/dt0 values, replayed from captured CUDA graphs.
 * diag_hist (nullable) receives one dtb_step_diag per step. */
int32_t dtb_run(dtb_ctx* ctx, const double* dt_scales, int64_t nsteps, int32_t verbose,
                dtb_step_diag* diag_hist);

/* Solve (Solver.jl:1-64): resets f to Initial, steps to every t_save[i] and writes f there
 * (f_out: n_save x n, row i = state at t_save[i]). Steps whose Cr exceeds 1 are reported on
 * stdout like the reference when verbose == 1. n_steps_out (nullable) gets the step count. */
int32_t dtb_solve(dtb_ctx* ctx, double dt_initial, const double* t_save, int64_t n_save,
                  int32_t verbose, double* f_out, int64_t* n_steps_out);

/* Step schedule of Solve, host only: per save interval the number of steps, and the
 * dt/dt0 of every step (capacity cap; n_total_out gets the total count). `precision`
 * selects how dt0 is rounded (Float32(dt0) for DTB_F32, SteppingStructs.jl:44). */
/* Solve with the save points pipelined behind the stepping (Solver.jl:1-64; the copies of
 * Solver.jl:40-43 made asynchronous) and the OutputStruct's moments computed on the device:
 * the whole schedule is enqueued without a host round trip per interval; at each save point
 * f is copied into a device ring slot that a second stream moves to pinned memory while the
 * next interval steps. f_out: n_save x n (or NULL); w: n_mom energy weights (or NULL for no
 * moments); number, energy: n_save x n_space x n_species, FP64 sums over each species slice
 * (DistributionMoments.jl:33,145,162). dtb_solve is this call with no moments. */
int32_t dtb_solve_ex(dtb_ctx* ctx, double dt_initial, const double* t_save, int64_t n_save,
                     int32_t verbose, double* f_out, const double* w, double* number,
                     double* energy, int64_t* n_steps);

int32_t dtb_solve_schedule(double dt_initial, const double* t_save, int64_t n_save, double dt0,
                           int32_t precision, int64_t* steps_per_interval, double* dt_scales,
                           int64_t cap, int64_t* n_total_out);

/* f (length n, as Float64) copy out / in; reset to Initial (Solver.jl:22). */
int32_t dtb_get_f(dtb_ctx* ctx, double* f);
int32_t dtb_set_f(dtb_ctx* ctx, const double* f);
int32_t dtb_reset(dtb_ctx* ctx);

/* Per (cell, species) number sum(f) and energy sum(f * w) in FP64 on the device
 * (DistributionMoments.jl:33,145,162); w is the per-state energy weight of one cell
 * (n_mom). Outputs are n_space x n_species, row-major. */
int32_t dtb_moments(dtb_ctx* ctx, const double* w, double* number, double* energy);

/* Device bytes held by the context; the stream it runs on; wait for its work. */
int32_t dtb_device_bytes(dtb_ctx* ctx, int64_t* bytes);
int32_t dtb_get_stream(dtb_ctx* ctx, void** stream);
int32_t dtb_sync(dtb_ctx* ctx);

/* Kernel launches issued per step by dtb_run (for launch accounting); the diagnostics
 * reduction adds one launch per sequence of steps (a graph replay, or up to a graph's length
 * of steps run outside one). */
int32_t dtb_launches_per_step(dtb_ctx* ctx, int32_t* n);
/* Kernel launches the context's step functions (dtb_step, dtb_step_io, dtb_run, dtb_solve) have
 * issued so far, kernels replayed in graphs included. No counterpart in the reference. */
int32_t dtb_launch_count(dtb_ctx* ctx, int64_t* n);

/* Failure-detection self-test: launches one block that waits, with a limit of limit_s
 * seconds (at most 2), on an mbarrier phase nothing completes, i.e. the give-up path of every
 * pipeline wait of the library. Returns DTB_ETIMEOUT and leaves the context usable. */
int32_t dtb_selftest_bounded_wait(dtb_ctx* ctx, double limit_s);

/* Dominant-kernel timing over the last dtb_run: average gain-kernel duration in ms measured
 * with CUDA events on the context stream, and its algorithmic bytes per launch. */
int32_t dtb_gain_kernel_stats(dtb_ctx* ctx, double* avg_ms, double* bytes_per_launch);
int32_t dtb_set_profiling(dtb_ctx* ctx, int32_t on);

/* ---- batched instances (precision DTB_MIXED, opts.batch = number of slots) ----
 * Many independent solves of one grid share the operators uploaded with the calls above;
 * each slot holds one instance (its own f, dt/dt0 and step count). The gain contraction of
 * all slots is one tensor-core GEMM per input pair with G stored as BF16 hi + lo with a
 * power-of-two scale per row (three MMAs: hi*hi + hi*lo + lo*hi, FP32 accumulation), f in
 * FP32 with a power-of-two scale per (slot, species) inside the GEMM operand, and the update
 * f += df of SteppingMethods.jl:97-101 accumulated in FP64 with a compensation term. A slot
 * holds dims.n_space cells (n_state = n_space * n_mom values): every (cell, slot) pair is a
 * column of the gain GEMM (update_Big_Bin!'s loop over cells, SteppingMethods.jl:360-386),
 * each cell with its Vol and BinM.Domain, the flux coupling the cells. */

/* Starts a solve in `slot`: f = f0 (n_state values), dt_scale = dt/dt0, n_steps steps from the
 * current batched step. A slot that finished (or was never admitted) does not step. */
int32_t dtb_batch_admit(dtb_ctx* ctx, int32_t slot, const double* f0, double dt_scale, int64_t n_steps);

/* nsteps batched steps of every slot that still has steps left, replayed from captured CUDA
 * graphs. Returns once the steps are enqueued on the context's stream; a device-side error of
 * these steps (a bounded wait that gave up) is reported by the next call that reads results
 * (dtb_batch_get_f, dtb_batch_get_f_all, dtb_batch_slot_info, dtb_batch_moments) or by dtb_sync.
 * With profiling on (dtb_batch_set_profiling) the call waits for the steps and checks them. */
int32_t dtb_batch_run(dtb_ctx* ctx, int64_t nsteps);

/* The slot's current f (FP32 state plus its compensation term, as Float64). */
int32_t dtb_batch_get_f(dtb_ctx* ctx, int32_t slot, double* f);

/* Steps taken and left, the largest Cr = -min(df ./ f) seen over the slot's steps, and
 * whether every df was finite (SteppingMethods.jl:48-94 reduced over the run). */
int32_t dtb_batch_slot_info(dtb_ctx* ctx, int32_t slot, int64_t* steps_done, int64_t* steps_left,
                            double* cr_max, int32_t* finite);

/* The whole batch's state in or out: f is [batch][n_state] Float64 (slot-major). set_f_all
 * replaces every slot's f (steps left and dt are kept); get_f_all reads every slot's f. */
int32_t dtb_batch_set_f_all(dtb_ctx* ctx, const double* f);
int32_t dtb_batch_get_f_all(dtb_ctx* ctx, double* f);

/* The host round trip of a caller that steps from host memory, in one call and one wait:
 * dtb_batch_set_f_all(f_in) (skipped when f_in is NULL), dtb_batch_run(nsteps), then
 * dtb_batch_get_f_all(f_out) (skipped when f_out is NULL). f_in and f_out may be the same
 * array. Device errors of the steps are reported by this call. */
int32_t dtb_batch_run_io(dtb_ctx* ctx, const double* f_in, int64_t nsteps, double* f_out);

/* FP64 number sum(f) and energy sum(f * w) of every slot, space cell and species, on the device
 * (DistributionMoments.jl:33,145,162); w is the per-state energy weight (n_mom). Outputs are
 * batch x n_space x n_species, slot-major. */
int32_t dtb_batch_moments(dtb_ctx* ctx, const double* w, double* number, double* energy);

/* Stops a slot (it no longer steps). */
int32_t dtb_batch_release(dtb_ctx* ctx, int32_t slot);

/* Number of slots and the batched steps taken so far. */
int32_t dtb_batch_capacity(dtb_ctx* ctx, int32_t* capacity, int64_t* step);

/* Times the gain GEMM launches of each step with CUDA events while on (direct launches). */
int32_t dtb_batch_set_profiling(dtb_ctx* ctx, int32_t on);

/* Average gain-GEMM time per step over the profiled steps, its algorithmic FLOPs (three MMAs)
 * and operator bytes per step, and the kernel launches per batched step. */
int32_t dtb_batch_gemm_stats(dtb_ctx* ctx, double* avg_ms, double* flops_per_step, double* bytes_per_step,
                             int32_t* launches_per_step);

/* Gain-GEMM autotuning. At commit a batched context times, for each gain group (the gain
 * blocks of one input pair), the candidate plans on the device with CUDA events: the column
 * tile width (64, 128 or 256 instances), one SM per tile or an SM pair sharing 256 x 256 MMAs
 * (cta_group::2, when the group's 128-row tiles pair up) and the K splits that fill the device,
 * and keeps the fastest. A plan is chosen once per shape and process, so contexts of one shape
 * run the same plan (and round alike). dtb_set_tune_cache names a text file that seeds the
 * plans and records every measured one, one line per shape:
 *   sm<SMs>:M<rows>:N1<n1>:n2<n2>:cols<columns>:cells<cells> <pair 0|1> <bn> <splits> <us>
 * NULL forgets the plans chosen so far and stops recording. Process-wide; replaces the
 * per-stage tile choices of a hand-tuned build (no reference counterpart: the reference's
 * mul! calls, SteppingMethods.jl:372-373, leave this to MKL / cuBLAS). */
int32_t dtb_set_tune_cache(const char* path);

/* The plan a committed batched context runs for gain group `group` (DTB_ENOTFOUND past the
 * last group): SM pairs or not, column tile width, K splits, and the measured time of one
 * GEMM with it in microseconds (0 when the plan came from the cache or the fixed rule). */
int32_t dtb_batch_gemm_plan(dtb_ctx* ctx, int32_t group, int32_t* pair, int32_t* bn, int32_t* n_splits,
                            double* tuned_us);

/* ---- serving: continuous batching of solve requests ----
 * A server owns a host thread that admits queued requests into free slots of their grid's
 * batched context, launches chunks of batched steps on every grid with running requests (the
 * grids' chunks overlap on the device, each on its context's stream), reads back finished
 * requests and frees their slots. Requests of one grid share the operators; requests that
 * arrive while others run join at the next admission point. */
typedef struct dtb_server dtb_server;

typedef struct dtb_serve_opts {
    int64_t hbm_budget_bytes;  /* device bytes all registered grids may hold (0: no limit) */
    int32_t max_chunk_steps;   /* most batched steps between admission points (0: 256) */
    int32_t flags;             /* reserved, 0 */
    double chunk_ms;           /* target device time of one chunk of a grid (0: 20 ms) */
} dtb_serve_opts;

typedef struct dtb_request_stats {
    double t_submit, t_admit, t_done;  /* seconds since dtb_serve_start */
    int64_t steps;
    double cr_max;                     /* largest Cr seen over the request's steps */
    int32_t finite;                    /* every df was finite */
    int32_t grid;
} dtb_request_stats;

typedef struct dtb_serve_stats {
    int64_t completed, instance_steps, batched_steps, queued, running, device_bytes;
    double busy_s, elapsed_s;
} dtb_serve_stats;

int32_t dtb_serve_create(const dtb_serve_opts* opts, dtb_server** out);
/* Registers a committed batched context as a grid (its device bytes count against the HBM
 * budget: DTB_ENOMEM when they do not fit). The server drives the context from its thread; the
 * caller must not use it directly until dtb_serve_destroy, and destroys it afterwards. */
int32_t dtb_serve_add_grid(dtb_server* srv, dtb_ctx* batched_ctx, int32_t* grid_id);
int32_t dtb_serve_start(dtb_server* srv);
/* Queues a solve (f0 copied; dt_scale = dt/dt0; n_steps steps). Thread-safe. */
int32_t dtb_serve_submit(dtb_server* srv, int32_t grid_id, const double* f0, double dt_scale, int64_t n_steps,
                         int64_t* request_id);
/* Waits for a request (timeout in seconds, <= 0: no limit; DTB_ETIMEOUT when it runs out) and
 * copies its final f and timings. */
int32_t dtb_serve_wait(dtb_server* srv, int64_t request_id, double timeout_s, double* f_out,
                       dtb_request_stats* stats);
/* Cancels a request (no counterpart in the reference, whose Solve runs one request to its end):
 * a queued request leaves the queue at once, a running one frees its slot at its grid's next chunk
 * boundary; dtb_serve_wait then returns DTB_ESTATE for it. Thread-safe; a request already done is
 * left as it is. */
int32_t dtb_serve_cancel(dtb_server* srv, int64_t request_id);
int32_t dtb_serve_get_stats(dtb_server* srv, dtb_serve_stats* stats);
/* Stops the loop thread (running requests are abandoned) and frees the server. */
int32_t dtb_serve_destroy(dtb_server* srv);

/* ---- kernel-level entry ---- */

/* out[a] = sum_b f1[b] sum_c G[a][b][c] f2[c] for one dense gain block in the caller's device
 * memory: the two products of update_Big_Bin! (SteppingMethods.jl:372-373) for one
 * (output, input-1, input-2) species block. G is row-major [n_out][n1][n2] with n2 a
 * multiple of 8 and 16-byte aligned; f1 (n1), f2 (n2) are device vectors of the same dtype;
 * out (n_out doubles) is a device vector. Runs asynchronously on `stream` (NULL: the legacy
 * default stream) on the current device. Its scratch (work table, per-unit partial sums and a
 * copy of f1|f2) is allocated on the first call on a device, grown when a larger block needs
 * more, and kept until the process exits. Calls on one device are serialised on the host.
 * DTB_EINVAL when G is not 16-byte aligned, out not 8-byte aligned or f1, f2 not aligned to
 * their element size. The call only enqueues work: a bounded device wait that gives up leaves
 * `out` incomplete and is reported by dtb_gain_contract_status. */
int32_t dtb_gain_contract(int32_t dtype, const void* G, int64_t n_out, int64_t n1, int64_t n2,
                          const void* f1, const void* f2, double* out, void* stream);

/* Device-side status of the kernel-level entries (no counterpart in the reference, whose
 * mul! calls report nothing): synchronises `stream`, then reads and clears the kernel error
 * flags of dtb_gain_contract and dtb_gain_contract_noalloc on the current device. Each call of
 * those entries clears its flag first, so the status covers the latest call of each entry on
 * this device. DTB_ETIMEOUT when a bounded wait gave up (that call's `out` is incomplete),
 * DTB_OK otherwise. */
int32_t dtb_gain_contract_status(void* stream);

/* Test hook (no counterpart in the reference): runs a kernel whose bounded wait on a flag that
 * nothing sets gives up after limit_s seconds (0 < limit_s <= 2) and raises the timeout flag of
 * dtb_gain_contract (noalloc = 0) or dtb_gain_contract_noalloc (noalloc = 1) on the current
 * device, through the give-up path of the contraction's waits; DTB_ESTATE when that entry has
 * not run on the device yet. */
int32_t dtb_selftest_gain_contract_timeout(int32_t noalloc, double limit_s, void* stream);

/* dtb_gain_contract for callers that cannot call cudaMalloc; it has no counterpart in the
 * reference. A host application that gives all device memory to its own pool allocator (a
 * Julia session whose CUDA.jl pool owns the device heap, a serving process that reserved its
 * HBM budget up front) or a latency-critical loop that cannot afford an allocator call uses
 * this entry point: it allocates nothing. Same arguments and result as dtb_gain_contract; the
 * scratch is a static device array of about 1.4 MB in libdtb.so, held by every GPU that
 * loads the library until the process exits. Limits: n1 + n2 <= 16384 and at most 32768 work
 * units (e.g. n_out = 1024, n1 = n2 = 1024 in FP32 needs 16384); larger blocks return
 * DTB_EINVAL with a message. The first call on a device looks up the array's device address
 * (set-up, once per device, with that device current); make that first call before any
 * stream capture. Every call on a device shares the one array and it keeps the last call's
 * contents (each call clears what must start at zero), so calls that overlap on the GPU
 * (different streams, no ordering between them) race; order them on one stream. Alignment
 * rules and error reporting (dtb_gain_contract_status) are those of dtb_gain_contract. */
int32_t dtb_gain_contract_noalloc(int32_t dtype, const void* G, int64_t n_out, int64_t n1, int64_t n2,
                                  const void* f1, const void* f2, double* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DTB_H */
