/*
 * spgpu.h — C ABI of the B200 (sm_100a) ePlace global-placement engine.
 *
 * Plain C: POD structs, raw pointers and sizes, int status returns. No CUDA, torch or
 * C++ types cross this boundary. Every entry point returns SPG_OK (0) on success or a
 * negative SPG_E_* code; spg_last_error() gives the message of the calling thread's last
 * failure.
 *
 * Threading: one host thread per context / Poisson handle (the reference's contract,
 * src/numeric/poisson_backend.h:20-46 and src/gp/eplace.h:56-77). Independent handles
 * may be used concurrently from different threads. The host passes of a stage (the grid's
 * static maps, the footprint scan, large host copies) run on a process-wide pool of worker
 * threads (one fewer than the hardware threads, at most 15), started on first use and idle
 * between calls; results do not depend on how many there are.
 *
 * Ownership: the caller owns every host array passed in; the library owns every device
 * buffer and releases it in the matching *_destroy call.
 *
 * There is no CPU fallback: when no sm_100 device is present the create calls fail with
 * SPG_E_NO_DEVICE.
 */
#ifndef SPGPU_H_
#define SPGPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPG_ABI_VERSION 3

/* ---- status codes (map onto the reference's InvariantError kinds, src/util/invariant.h:10-19) */
#define SPG_OK 0
#define SPG_E_INVALID (-1)       /* bad argument: dims, steps, sizes, null pointers      */
#define SPG_E_NO_DEVICE (-2)     /* no usable sm_100 device                              */
#define SPG_E_CUDA (-3)          /* a CUDA runtime call failed                           */
#define SPG_E_NON_FINITE (-4)    /* InvariantError kind "non_finite"                     */
#define SPG_E_OUT_OF_CORE (-5)   /* InvariantError kind "out_of_core"                    */
#define SPG_E_CONVERGENCE (-6)   /* InvariantError kind "convergence_mismatch"           */
#define SPG_E_ROLLBACK (-7)      /* InvariantError kind "rollback_mismatch"              */
#define SPG_E_STATE (-8)         /* call out of order (e.g. run before stage_begin)      */
#define SPG_E_CAPACITY (-9)      /* a size beyond a stated maximum                       */

/* ---- node flags: same bit values as sp::NodeFlag (src/db/place_db.h:17-22) */
#define SPG_F_MACRO 1u
#define SPG_F_FIXED 2u
#define SPG_F_FILLER 4u
#define SPG_F_NI 8u

/* ---- Poisson arithmetic */
#define SPG_POISSON_FP32 0   /* cosine contractions as FP32 SIMT GEMMs ("plain FP32")        */
#define SPG_POISSON_BF16X3 1 /* tcgen05 split-BF16 (hi*hi + hi*lo + lo*hi), FP32 accumulate */
#define SPG_POISSON_FP64 2   /* the same contractions in FP64 (accuracy reference, slow)      */

/* ---- GP stages (sp::GpStage, src/gp/eplace.h:24-28) */
#define SPG_STAGE_MGP 0
#define SPG_STAGE_FILLER_ONLY 1
#define SPG_STAGE_CGP 2

/*
 * Read-only view of a PlaceDB (src/db/place_db.h:24-113): node SoA in centre coordinates,
 * segments [movable | fixed | filler], pins, and the two-way CSR built by
 * PlaceDB::finalizeCSR (src/db/place_db.cpp:67-95). node2pin_start has
 * num_nodes + num_fillers + 1 entries (fillers own no pins, src/gp/filler.cpp:130).
 */
typedef struct spg_db_view {
    int32_t num_movable; /* [0, num_movable)                          */
    int32_t num_nodes;   /* [num_movable, num_nodes) fixed           */
    int32_t num_fillers; /* [num_nodes, num_nodes + num_fillers)     */
    const float* node_x;
    const float* node_y;
    const float* node_w;
    const float* node_h;
    const uint8_t* node_flags;

    int32_t num_pins;
    const float* pin_offset_x; /* relative to the node centre */
    const float* pin_offset_y;
    const int32_t* pin2node;
    const int32_t* pin2net;

    int32_t num_nets;
    const int32_t* net2pin_start;  /* num_nets + 1 */
    const int32_t* flat_net2pin;   /* num_pins     */
    const int32_t* node2pin_start; /* total + 1    */
    const int32_t* flat_node2pin;  /* num_pins     */

    int32_t num_rows; /* PlaceDB::SiteRow, src/db/place_db.h:47-55 */
    const float* row_ly;
    const float* row_height;
    const float* row_lx;
    const float* row_step;
    const int32_t* row_num_sites;

    /* PlaceDB::computeRegions() results (src/db/place_db.cpp:97-127) */
    float core_lx, core_ly, core_hx, core_hy;
    float row_height_mode;
    double total_row_area;
} spg_db_view;

/* GP configuration: the Config keys the path reads (src/util/config.h:77-116). */
typedef struct spg_params {
    float target_density;       /* 1.0  */
    float target_overflow;      /* 0.10 */
    float cgp_target_overflow;  /* 0.10 */
    int32_t gp_max_iter;        /* 2000 */
    int32_t ignore_net_degree;  /* 100  */
    int32_t gp_bin_dim;         /* 0 = auto (power of two, cap 1024) */
    int32_t filler_only_iters;  /* 20   */
    float delta_hpwl_ref;       /* 3.5e5 */
    int32_t lambda_schedule_relative; /* 0 = "fixed", 1 = "relative" */
    double delta_hpwl_relative; /* 0.01 */
    int32_t use_bb;             /* 1 */
    int32_t gp_backtrack;       /* 1 */
    int32_t max_backtrack;      /* 10 (OptConfig::max_backtrack) */
    int32_t gp_stagnation_window;  /* 200  */
    float gp_stagnation_min_gain;  /* 0.02 */
    uint64_t random_seed;          /* 1002 */
    int32_t poisson_precision;     /* SPG_POISSON_* */
    int32_t verbose;               /* log every iteration instead of every 20th */
    /* appended in ABI version 3: the diagnostic run options GpRunOptions::freezeLambda and
     * freezeGamma (src/gp/eplace.h:45-52; eplace.cpp:374-380): lambda keeps its initial
     * value (mu = 1) and gamma its value from the lambda_0 probe. Off (0) in production. */
    int32_t freeze_lambda;
    int32_t freeze_gamma;
    /* 1: the context's one-grid split-BF16 solves run as one persistent launch (G1, the split
     * of its output, G2, G3, G4 with grid barriers between them), with the same results as the
     * separate launches. Its barriers need all of its CTAs resident at once, so it is only for
     * a context that runs alone on its device. 0 (default): separate launches, which measured
     * faster at 512x512. No counterpart in the reference. */
    int32_t poisson_single_launch;
} spg_params;

/* Defaults identical to configs/default.json of the reference. */
void spg_params_default(spg_params* p);

/* sp::GpResult (src/gp/eplace.h:32-42) plus the stage-start summary keys. */
typedef struct spg_result {
    int32_t iterations;
    double hpwl;
    float overflow;
    int32_t converged;
    int32_t stagnated;
    int32_t rollback_iter;
    int64_t evaluations;
    double elapsed_ms;      /* device-timed stage duration (CUDA events) */
    double initial_hpwl;    /* <stage>_initial_hpwl    */
    float initial_overflow; /* <stage>_initial_overflow */
    float initial_lambda;   /* <stage>_initial_lambda   */
} spg_result;

/* sp::IterMetrics (src/util/metrics.h:12-28), one row per GP iteration. */
typedef struct spg_iter_metrics {
    int32_t iter;
    double hpwl;
    float overflow;
    float lambda;
    float gamma;
    float step_size;
    float grad_norm_wl;
    float grad_norm_den;
    float eval_lambda;
    float eval_gamma;
    double delta_hpwl;
    float lambda_mu;
    int64_t evaluations;
    /* appended in ABI version 2: the reference's max_displacement (its GP never sets it: 0)
     * and elapsed_ms, the device time since the stage's iteration loop began */
    float max_displacement;
    double elapsed_ms;
} spg_iter_metrics;

/* Filler plan (sp::FillerInfo, src/gp/filler.h:18-25). */
typedef struct spg_filler_info {
    int32_t count;
    float width;
    float height;
    double whitespace_area;
    double node_area_scaled;
    double total_filler_area;
} spg_filler_info;

int spg_abi_version(void);
const char* spg_last_error(void);
/* 0 when a usable sm_100 device is visible, else SPG_E_NO_DEVICE. */
int spg_device_check(void);

/* ------------------------------------------------------------------ Poisson operator
 * Replaces PoissonBackend::solve (src/numeric/poisson_backend.h:36-37) built by
 * makePoissonBackend({nx, ny, step_x, step_y, prefer_gpu}) (poisson_backend.h:48-60).
 * Arrays are row-major data[x * ny + y] (src/numeric/bin_grid_span.h:13-23).
 * Errors: SPG_E_INVALID on nx,ny < 2 or non-positive steps (cpu_poisson.cpp:78-83);
 * SPG_E_NO_DEVICE when no device (cuda_poisson.cu:328-336 returns nullptr there).
 * solve() allocates nothing (poisson_backend.h:35).
 */
typedef struct spg_poisson spg_poisson;
int spg_poisson_create(int nx, int ny, float step_x, float step_y, int precision,
                       spg_poisson** out);
/* As spg_poisson_create, with work buffers for batched solves of up to batch_cap grids. */
int spg_poisson_create_batched(int nx, int ny, float step_x, float step_y, int precision,
                               int batch_cap, spg_poisson** out);
/* Host arrays in and out; copies inside (like CudaPoissonBackend::solve). */
int spg_poisson_solve(spg_poisson* h, const float* rho, float* phi, float* field_x,
                      float* field_y);
/* Device arrays in and out, work enqueued on `stream` (a cudaStream_t, 0 = default). */
int spg_poisson_solve_device(spg_poisson* h, const float* d_rho, float* d_phi,
                             float* d_field_x, float* d_field_y, void* stream);
/* Batched device solve: `batch` grids stored back to back (each nx*ny floats). */
int spg_poisson_solve_batch_device(spg_poisson* h, int batch, const float* d_rho,
                                   float* d_phi, float* d_field_x, float* d_field_y,
                                   void* stream);
const char* spg_poisson_name(const spg_poisson* h);
/* 1: this handle's one-grid split-BF16 solves run as one persistent launch, with the same
 * results as the separate launches (off by default). Its grid barriers need all of its CTAs
 * resident at once: only for a handle whose solves do not overlap another such launch on the
 * device (the reference allows independent handles to run concurrently). No counterpart in
 * the reference. */
int spg_poisson_set_single_launch(spg_poisson* h, int on);
int spg_poisson_destroy(spg_poisson* h);

/* Poisson solve that allocates nothing. No counterpart in the reference: it exists for
 * callers that cannot call cudaMalloc (hosts that reserve all device memory up front in
 * their own pool and forbid later driver allocations), which therefore cannot create a
 * spg_poisson plan. The plain-FP32 solve of a plan, device arrays in and out, work enqueued
 * on `stream`; its basis tables are built on the device, so it agrees with a plan's solve to
 * 1e-5 of max|result| rather than bit for bit. Its bases and work buffers live in one static
 * device array of 11 MB that every GPU loading this library holds until the process exits;
 * nx and ny must be at most 512 (larger sizes return SPG_E_CAPACITY). All calls on a device
 * share that array, so calls that overlap on the GPU race: serialise them. Each call made
 * outside a stream capture looks the array's address up again (cudaGetSymbolAddress), so a
 * device reset leaves no stale address; a call on a capturing stream reuses the last one,
 * so make the first call on a device before any stream capture. */
int spg_poisson_solve_static(int nx, int ny, float step_x, float step_y, const float* d_rho,
                             float* d_phi, float* d_field_x, float* d_field_y, void* stream);

/* ------------------------------------------------------------------ fillers (host)
 * initializeFillers (src/gp/filler.cpp:47-139): size and count from the view's movable
 * nodes, rows and fixed nodes; scatterFillers (src/gp/filler.cpp:33-45): mt19937 seeded
 * uniform positions, written to x/y (count entries each).
 */
int spg_fillers_plan(const spg_db_view* db, float target_density, spg_filler_info* out);
int spg_fillers_scatter(const spg_db_view* db, int32_t count, float width, float height,
                        uint64_t seed, float* x, float* y);

/* ------------------------------------------------------------------ placement context
 * Replaces EPlace(PlaceDB&, const Config&, MetricsSink&) + EPlace::run (src/gp/eplace.h:56-77)
 * as called by GlobalPlaceStage::run (src/stages/gp_stage.cpp:99-201). The view is copied
 * to the device at create; positions stay device-resident until spg_positions_d2h.
 */
typedef struct spg_ctx spg_ctx;
int spg_ctx_create(const spg_db_view* db, const spg_params* params, spg_ctx** out);
/* Replace the context's netlist and parameters with another instance (the next request of a
 * placement server): the context keeps its streams, staging memory and device buffers where
 * their capacity suffices, so no device memory is allocated or freed for an instance of no
 * larger size. Equivalent to destroying and creating the context. No counterpart in the
 * reference, which builds one EPlace per instance. */
int spg_ctx_load(spg_ctx* ctx, const spg_db_view* db, const spg_params* params);
int spg_ctx_destroy(spg_ctx* ctx);

/* Upload new centre positions for all num_nodes + num_fillers nodes. The arrays may be reused
 * once the call returns: page-locked arrays (spg_host_alloc) are copied by DMA and waited
 * for; pageable ones are copied into the context's pinned staging memory and their device
 * copy runs on the context's stream ahead of its next work. */
int spg_positions_h2d(spg_ctx* ctx, const float* x, const float* y);
/* Download the current centre positions of all nodes (complete on return; direct DMA into
 * page-locked arrays, through the staging memory into pageable ones). */
int spg_positions_d2h(spg_ctx* ctx, float* x, float* y);
/* Page-locked host memory for the position arrays of spg_positions_h2d / _d2h, so that their
 * copies skip the host-side staging copy. No counterpart in the reference, which keeps its
 * PlaceDB in ordinary host memory. */
int spg_host_alloc(size_t bytes, void** out);
int spg_host_free(void* p);
/* Self-check of the bin-index arithmetic of the density kernels: for each a[i], q_div[i] =
 * int(a[i] / step) with the float division of BinGrid::footprintOf (src/gp/bin_grid.cpp:49-52)
 * and q_mul[i] = the same index formed as the double product a[i] * (1/step) rounded to float,
 * which the kernels use; the two must agree everywhere. */
int spg_bin_index_check(float step, const float* a, int32_t n, int32_t* q_div, int32_t* q_mul);
/* Replace node flags (e.g. macros frozen by mLG get SPG_F_FIXED, gp_stage.cpp:130-177). */
int spg_flags_h2d(spg_ctx* ctx, const uint8_t* flags);

/* BinGrid::initialize (src/gp/bin_grid.cpp:64-189): static terminal/base density and the
 * grid dimension for the current flags. bin_dim <= 0 selects the automatic dimension. */
int spg_grid_init(spg_ctx* ctx, float target_density, int bin_dim);
int spg_grid_info(const spg_ctx* ctx, int* dim, float* step_x, float* step_y,
                  float* origin_x, float* origin_y, double* overflow_denominator);
/* which: 0 node density, 1 filler density, 2 terminal, 3 base, 4 rho, 5 phi, 6 xi_x, 7 xi_y */
int spg_grid_read(const spg_ctx* ctx, int which, float* out);
/* Overwrite a device map (which: 4 rho, 5 phi, 6 xi_x, 7 xi_y) to drive an operator in
 * isolation, e.g. gather over a given field. */
int spg_grid_write(spg_ctx* ctx, int which, const float* in);
/* The bit-exact 64-bit fixed-point density maps (node, filler) and their scale 2^-shift. */
int spg_grid_read_fixed(const spg_ctx* ctx, int64_t* node_fixed, int64_t* filler_fixed,
                        int* shift);

/* Operator parity hooks (each runs on the device over the uploaded positions). */
int spg_density_accumulate(spg_ctx* ctx);                     /* BinGrid::accumulate  */
int spg_overflow(spg_ctx* ctx, float* tau);                   /* BinGrid::overflow    */
int spg_solve_field(spg_ctx* ctx);                            /* BinGrid::solveField  */
/* BinGrid::gatherForce: force (q*xi, NOT gradient) for every non-fixed node, 2*total floats. */
int spg_gather_force(spg_ctx* ctx, float* force);
/* BinGrid::totalCharge (exact sum of the fixed-point contributions). */
int spg_total_charge(spg_ctx* ctx, double* charge);
/* WaWirelength::compute (src/gp/wa_wirelength.cpp:46-180): grad = [x..., y...] over num_movable. */
int spg_wa_wirelength(spg_ctx* ctx, float gamma, int ignore_net_degree, double* wl, float* grad);
/* computeHPWL (src/db/hpwl.cpp:13-39). */
int spg_hpwl(spg_ctx* ctx, double* hpwl);

/* EPlace::run (src/gp/eplace.cpp:223-526): the device-resident Nesterov loop for one stage.
 * Rebuilds the grid with the current flags (as constructing EPlace does,
 * gp_stage.cpp:175-177), runs to convergence, stagnation or max_iter, and leaves the
 * delivered positions on the device. */
int spg_stage_run(spg_ctx* ctx, int stage, spg_result* result);
/* Per-iteration metrics of the last stage run (up to `cap` rows). */
int spg_metrics_d2h(const spg_ctx* ctx, spg_iter_metrics* rows, int cap, int* n_rows);

/* Iteration callback: EPlace::setIterCallback (src/gp/eplace.h:71-72), which the reference calls
 * after each iteration's metrics row with the PlaceDB at that iteration's evaluation point
 * (eplace.cpp:405-409); GlobalPlaceStage's frame hook samples it every frame_stride iterations
 * (gp_stage.cpp:87-93). Here fn(user, stage, iter, x, y) runs for every iteration with
 * iter % stride == 0, with x and y the positions of all num_nodes + num_fillers nodes at that
 * evaluation point (arrays owned by the context, valid during the call). Each call pauses the
 * device loop for a host round trip; the placement is the same bit for bit with and without
 * the callback. fn NULL or stride <= 0 turns it off. */
typedef void (*spg_iter_fn)(void* user, int32_t stage, int32_t iter, const float* x, const float* y);
int spg_set_iter_callback(spg_ctx* ctx, spg_iter_fn fn, void* user, int32_t stride);
/* Called once per stage (mGP, cGP), like the iteration callback, at the iteration where the
 * stagnation guard's counter of iterations without enough overflow gain first reaches half its
 * window: the reference's stagnation_mid GP diagnostic point (eplace.cpp:428-433). fn NULL: off. */
int spg_set_stagnation_callback(spg_ctx* ctx, spg_iter_fn fn, void* user);
/* After a stage run: the positions of all nodes at its last evaluation point (which = 0) or at
 * the evaluation point before it (which = 1), the inputs of the reference's last_eval GP
 * diagnostic (writeGpDiagnostic, src/gp/diagnostics.h:13-17; eplace.cpp:476-479). */
int spg_eval_positions(spg_ctx* ctx, int32_t which, float* x, float* y);

/* Number of kernels this library launched (process-wide) so far. */
int64_t spg_ctx_launch_count(const spg_ctx* ctx);
/* The cudaStream_t every call on this context enqueues on (for caller-side CUDA events). */
void* spg_ctx_stream(const spg_ctx* ctx);
/* Per-kernel device time (microseconds, CUDA events on the context's stream, averaged
 * over `reps` back-to-back launches, L2 warm as inside the loop) of the iteration's parts
 * at the current positions, after a stage run. us[] receives up to n values in this order:
 *   0 update + density scatter of the opt nodes
 *   1 WA pass 1 + HPWL, then the cells' WA pass 2
 *   2 density scatter of the other density nodes (0 when there are none)
 *   3 rho + overflow   4 Poisson solve
 *   5 assembly (gather + gradient + the step's norms and decisions)
 *   6 unused (0: the norms run inside the assembly)   7 one evaluation
 * The stage's results are left unchanged (state and delivered positions are restored). */
int spg_ctx_profile(spg_ctx* ctx, int reps, double* us, int n);
/* 1 when the last stage run executed its iteration loop as one conditional CUDA graph,
 * 0 when it ran the host-driven loop (SPG_HOST_LOOP set, or conditional nodes refused). */
int spg_ctx_graph_loop(const spg_ctx* ctx);

/* EPlace::Impl::objAndGrad (src/gp/eplace.cpp:136-203) at caller positions, through the
 * stage loop's own kernels (the loop body with no step applied): the grid and opt set are
 * rebuilt for `stage` from the context's positions and flags (as constructing EPlace does),
 * the opt nodes are placed at pos (2*nOpt floats, x then y, in buildOptSet's order:
 * movable non-fixed non-NI nodes, minus the macros in cGP, none in FILLERONLY, then the
 * fillers, eplace.cpp:82-94), and one evaluation runs with the given lambda and gamma.
 * grad gets the preconditioned gradient precond * (dWL - lambda * q xi) (2*nOpt floats);
 * out[0..4] = WA wirelength (the objective), overflow tau, HPWL, sum|dWL|, sum|q xi|;
 * *n_opt = nOpt. With pos = NULL only *n_opt is set. The opt nodes stay at pos. */
int spg_eval_grad(spg_ctx* ctx, int stage, float lambda, float gamma, const float* pos, float* grad,
                  double* out, int32_t* n_opt);

/* The stage loop's optimizer on a test objective: NesterovOptimizer::step
 * (src/numeric/cpu/nesterov.cpp:51-122) called `steps` times from pos, as the reference's
 * optimizer tests drive it (test/test_nesterov.cpp), on f(x) = 0.5 * sum c_i (x_i - t_i)^2,
 * with the device loop's step kernel, backtracking test (redoIfOvershot, :146-169), step
 * decisions (estimateStep with BB, :221-240) and, when init_step <= 0, estimateInitialStep
 * (:190-218). n must be even and >= 2 (the vectors are kept as n/2 x-y pairs). No
 * constraint. pos gets the current solution v; out[0..3] = objective at the last counted
 * evaluation, evaluations, step size, backtracking re-evaluations. */
int spg_nesterov_quadratic(int32_t n, const float* coef, const float* target, float* pos, int32_t steps,
                           int32_t use_bb, int32_t backtrack, int32_t max_backtrack, float init_step,
                           double* out);

/* ------------------------------------------------------------------ BookShelf files (host)
 * BookshelfReader::read (src/io/bookshelf_reader.cpp:404-436): the .aux and the .scl, .nodes,
 * .nets, .pl and .wts files it names, into the PlaceDB layout: nodes reordered stably to
 * [movable | fixed] (centres; movable nodes taller than 1.5 row heights marked as macros),
 * pins in file order with offsets from the node centre, both CSR directions, unit net weights
 * where the .wts gives none. The handle owns the arrays until spg_bookshelf_destroy. */
typedef struct spg_bookshelf spg_bookshelf;
int spg_bookshelf_read(const char* aux_path, spg_bookshelf** out);
/* Message of the calling thread's last failed BookShelf call. */
const char* spg_bookshelf_last_error(void);
/* counts[0..6] = num_movable, num_nodes, num_pins, num_nets, num_rows, bytes of the node names
 * and bytes of the net names (each name NUL-terminated, back to back, in index order). */
int spg_bookshelf_counts(const spg_bookshelf* b, int64_t* counts);
/* Copies into caller arrays sized by spg_bookshelf_counts; a NULL pointer skips that array.
 * orient is the BookShelf orientation code (0..7 = N, E, S, W, FN, FE, FS, FW). */
int spg_bookshelf_nodes(const spg_bookshelf* b, float* x, float* y, float* w, float* h, uint8_t* flags,
                        uint8_t* orient, char* names);
int spg_bookshelf_pins(const spg_bookshelf* b, float* pin_offset_x, float* pin_offset_y, int32_t* pin2node,
                       int32_t* pin2net, int32_t* net2pin_start, int32_t* flat_net2pin,
                       int32_t* node2pin_start, int32_t* flat_node2pin);
int spg_bookshelf_nets(const spg_bookshelf* b, float* weight, char* names);
int spg_bookshelf_rows(const spg_bookshelf* b, float* ly, float* height, float* lx, float* step,
                       int32_t* num_sites);
int spg_bookshelf_destroy(spg_bookshelf* b);
/* ---------------------------------------------------------------------------------------------
 * B2B (Kraftwerk2) quadratic initial placement: QuadraticPlacer::place
 * (src/init/quadratic_placer.cpp:153-228), IInitialPlacer "init" (src/init/initial_placer.h:24-38).
 * The system is assembled on the host; BiCGSTAB runs on the host or, with device = 1, on the
 * GPU, with the same bits either way. The fields are the Config keys the placer reads
 * (src/util/config.h:49-83).
 * ------------------------------------------------------------------------------------------- */
typedef struct spg_qp_params {
    int32_t max_iter;          /* qp_max_iter        20   outer iterations                      */
    float tol;                 /* qp_tol             1e-6 BiCGSTAB relative residual            */
    int32_t solver_max_iter;   /* qp_solver_max_iter 100  BiCGSTAB iterations per solve         */
    float outer_tol;           /* qp_outer_tol       1e-4 stop when HPWL moves less (relative)  */
    float min_distance;        /* qp_min_distance    1.0  floor of the B2B weight denominator   */
    int32_t ignore_net_degree; /* ignore_net_degree  100  nets above it are left out            */
    int32_t threads;           /* host threads; 0 = all (results do not depend on it)           */
    int32_t device;            /* 1: BiCGSTAB on the GPU (same results); 0: on the host         */
} spg_qp_params;

/* One outer iteration: the reference's IterMetrics row of the QP (iter, hpwl, grad_norm_wl =
 * max of the two solver errors, elapsed_ms), plus the solver iterations per axis. */
typedef struct spg_qp_row {
    int32_t iter;
    int32_t solver_iters_x;
    int32_t solver_iters_y;
    float err;
    double hpwl;
    double elapsed_ms;
    double assemble_ms; /* of elapsed_ms: bound pins and both systems (host)                 */
    double solve_ms;    /* of elapsed_ms: both BiCGSTAB solves, copies included              */
} spg_qp_row;

void spg_qp_default_params(spg_qp_params* p);
/* Message of the calling thread's last failed QP call. */
const char* spg_qp_last_error(void);
/* Places the movable nodes: x, y (num_nodes centres) are read for the fixed nodes and written
 * for the movable ones (they start at the core centre). net_weight may be NULL (all 1). Up to
 * cap rows go to rows; *num_rows gets their count. Uses db's CSR, pin offsets, sizes and core. */
int spg_qp_place(const spg_db_view* db, const float* net_weight, const spg_qp_params* p, float* x, float* y,
                 spg_qp_row* rows, int32_t cap, int32_t* num_rows);
/* The linear system of one axis (0 = x, 1 = y) at positions x, y, as the reference assembles it
 * (src/init/quadratic_placer.cpp:43-112): CSR over the movable nodes (row_start num_movable + 1,
 * columns ascending) and the right-hand side. *nnz gets the entry count; with cap < *nnz
 * nothing else is written. */
int spg_qp_assemble(const spg_db_view* db, const float* net_weight, const spg_qp_params* p, int32_t axis,
                    const float* x, const float* y, int32_t* row_start, int32_t* col, float* val, float* rhs,
                    int64_t cap, int64_t* nnz);
/* computeHPWL (src/db/hpwl.cpp:13-39) at positions x, y on the host. */
int spg_host_hpwl(const spg_db_view* db, const float* x, const float* y, double* out);

/* BookshelfReader::readPlacement (src/io/bookshelf_reader.cpp:367-401): applies a .pl to nodes
 * already read, in place. Names are NUL-terminated back to back (the first of equal names
 * takes the line); x, y become lower-left + half the size, orient takes the code after ':' and
 * a token containing FIXED sets SPG_F_FIXED in flags (the nodes are not reordered). */
int spg_bookshelf_apply_pl(const char* path, int32_t num_nodes, const char* names, const float* w, const float* h,
                           float* x, float* y, uint8_t* flags, uint8_t* orient);
/* BookshelfWriter::writePl (src/io/bookshelf_writer.cpp:16-37): lower-left corners of the first
 * num_nodes nodes in index order; names NUL-terminated back to back; orient may be NULL (N). */
int spg_bookshelf_write_pl(const char* path, int32_t num_nodes, const char* names, const float* x,
                           const float* y, const float* w, const float* h, const uint8_t* flags,
                           const uint8_t* orient);

#ifdef __cplusplus
}
#endif

#endif /* SPGPU_H_ */
