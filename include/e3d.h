/*
 * e3d.h -- C ABI of the B200 residual-and-update path for euler3D cases.
 *
 * Plain C types only (no CUDA, no torch, no C++ in the signatures).  Every
 * function returns an int status: 0 on success, a negative E3D_ERR_* code on
 * failure, with a message available from e3d_last_error() on the calling
 * thread.  Nothing here calls exit() or traps on the device.
 *
 * Each entry point names the reference interface it replaces (file:line in
 * guillaumetousignant/euler3D).  A "block" argument of -1 applies the call to
 * every block, which is what one outer iteration of the reference does block
 * after block (Solver/src/Solver.cpp:83-91).
 */
#ifndef E3D_H
#define E3D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define E3D_OK 0
#define E3D_ERR_ARG (-1)       /* bad argument or unsupported deck option */
#define E3D_ERR_IO (-2)        /* file cannot be opened or read */
#define E3D_ERR_FORMAT (-3)    /* deck / topology / SU2 syntax */
#define E3D_ERR_MESH (-4)      /* inconsistent mesh (open cell, face shared by 3 cells, ...) */
#define E3D_ERR_CUDA (-5)      /* CUDA runtime error */
#define E3D_ERR_NONFINITE (-6) /* a residual norm became NaN or infinite */
#define E3D_ERR_STATE (-7)     /* call not valid in this solver state / precision */
#define E3D_ERR_LIMIT (-9)     /* size above a documented maximum */

/* strategy selectors: the reference's string choices
 * (ResidualCalculator.cpp:72-95, SecondOrder.cpp:50-61) */
#define E3D_GRAD_GREEN_GAUSS 0
#define E3D_GRAD_LEAST_SQUARES 1
#define E3D_LIM_BARTH_JESPERSEN 0
#define E3D_LIM_VENKATAKRISHNAN 1
#define E3D_FLUX_ROE 0
#define E3D_FLUX_AUSM 1

#define E3D_FP64 0 /* drop-in: reference FP64 arithmetic */
#define E3D_FP32 1 /* FP32 bulk, FP64 conserved state and reductions */
#define E3D_FP64_FMA 2 /* e3d_solver_set_precision only: FP64, batch solves with fused multiply-add */
#define E3D_FP32_DELTA 3 /* e3d_solver_set_precision only: FP32 batch solves in difference form (below) */

typedef struct e3d_case e3d_case;     /* host case: deck + topology + blocks */
typedef struct e3d_solver e3d_solver; /* device-resident solver over one case */

typedef struct e3d_deck_info {
	double cfl, gamma, aoa_deg, mach, cmac, criterion, omega, k;
	int stages, max_iter, smoothing, order;
	int flux, gradient, limiter; /* E3D_FLUX_*, E3D_GRAD_*, E3D_LIM_* as the reference selects them */
} e3d_deck_info;

typedef struct e3d_block_info {
	int n_real, n_all, n_faces, n_nodes, n_markers, n_real_boundaries, n_wall_faces;
} e3d_block_info;

/* device order of each block's real cells (e3d_options.renumber; by default
 * file order with the cells that have a ghost neighbour moved to the end of
 * their block).  No counterpart in the reference, which keeps file order.  A
 * cell's slots keep its ascending face order, so FP64 results are bit for bit
 * the same in every order; state transfers (e3d_state_get/set) stay in file
 * order.  The state blob of e3d_state_export and the rows of
 * e3d_cell_features are in device order. */
#define E3D_RENUMBER_NONE 0    /* file order */
#define E3D_RENUMBER_RCM 1     /* reverse Cuthill-McKee on the cell adjacency graph */
#define E3D_RENUMBER_MORTON 2  /* Z-order curve of the cell centres */
#define E3D_RENUMBER_SHUFFLE 3 /* seeded random order (worst case, for tests and measurement) */
/* added to any of the above: the cells with a ghost neighbour (boundary and
 * connexion faces) move to the end of their block, each group in the base
 * order, so that the stage passes' extra work for them runs in their warps only */
#define E3D_RENUMBER_BOUNDARY_LAST 16

typedef struct e3d_options {
	int precision;    /* E3D_FP64 or E3D_FP32 */
	int carry_w0;     /* -1 default (FP32: on), 0 recompute W0 from primitives, 1 carry FP64 W */
	int use_graph;    /* 1: one CUDA graph per outer iteration */
	int device;       /* -1: current device */
	void* stream;     /* cudaStream_t or NULL (solver creates its own) */
	int hist_capacity;/* iterations of history buffered on the device (0: 4096) */
	int renumber;     /* E3D_RENUMBER_* (default E3D_RENUMBER_NONE | E3D_RENUMBER_BOUNDARY_LAST) */
} e3d_options;

/* One outer iteration's post-processing (PostProcessing::process,
 * PostProcessing/src/PostProcessing.cpp:220-308). */
typedef struct e3d_iter_record {
	int iter;
	double rms[5];  /* rho, u, v, w, p residual norms summed over blocks */
	double conv[5]; /* log10(rms) - log10(rms at iteration 0) */
	double cl, cd, cmx, cmy, cmz;
} e3d_iter_record;

/* ---- errors ---------------------------------------------------------------- */
const char* e3d_last_error(void);
const char* e3d_version(void);
void e3d_default_options(e3d_options* opt);

/* ---- host case ----------------------------------------------------------------
 * e3d_case_load replaces main.cpp:61-82: Interface::readInputFile
 * (Solver/src/Interface.cpp:14-237), Interface::readNBlocks (:239-266) and
 * CompleteMesh::InitializeMyBlocks (DataStructure/src/CompleteMesh.cpp:79-293),
 * i.e. ConcreteBlockBuilder::preReadMyBlock/readMyBlock/createMyFaces
 * (BlockBuilder/src/ConcreteBlockBuilder.cpp:22-742), BlockBuilder::setConnectivity
 * (BlockBuilder/src/BlockBuilder.cpp:147-458) and MetricsInitializer::doInit
 * (Metrics/src/MetricsInitializer.cpp:27-54).  Relative paths in the deck and
 * topology are resolved against `workdir` (NULL: the current directory), as
 * the reference resolves them against its working directory. */
int e3d_case_load(const char* deck_path, const char* workdir, e3d_case** out);
int e3d_case_free(e3d_case* c);
int e3d_case_deck(const e3d_case* c, e3d_deck_info* out);
int e3d_case_n_blocks(const e3d_case* c, int* n);
int e3d_case_block_info(const e3d_case* c, int block, e3d_block_info* out);
/* Copies one per-block array (the reference Block/Cell/Face members) into dst.
 * count must equal the array length (query with dst == NULL: *count is set).
 * Float arrays: face_normal, face_area, face_center, r_left, r_right,
 * cell_volume, cell_center, ls_weights.  Int arrays: face_cells, cell_face_ptr,
 * cell_faces, cell_cells, wall_faces, marker_kind, marker_size, marker_cells. */
int e3d_case_get_f64(const e3d_case* c, int block, const char* name, double* dst, int64_t* count);
int e3d_case_get_i32(const e3d_case* c, int block, const char* name, int32_t* dst, int64_t* count);
/* The device order a solver created with e3d_options.renumber = mode gives the
 * real cells of one block: order[i] = block-local (file) index of the cell
 * placed i-th (n_real entries).  Host only.  No counterpart in the reference. */
int e3d_case_cell_order(const e3d_case* c, int block, int mode, int32_t* order, int64_t n_real);

/* ---- solver ------------------------------------------------------------------
 * e3d_solver_create replaces Initializer::initializeSolver
 * (DataStructure/src/Initializer.cpp:25-50) and the per-block
 * calculateFreeVariables/initializeFlowField (PrimitiveVariables.cpp:41-69):
 * uploads the case and sets every cell to freestream.  opt may be NULL. */
int e3d_solver_create(const e3d_case* c, const e3d_options* opt, e3d_solver** out);
int e3d_solver_free(e3d_solver* s);
int e3d_solver_sync(e3d_solver* s);
int e3d_solver_device_bytes(const e3d_solver* s, int64_t* bytes);

/* Strategy-level calls (FP64 solver only), one per reference method. */
int e3d_save_w0(e3d_solver* s, int block);           /* Solver::saveW0, Solver/src/Solver.cpp:161-210 */
int e3d_spectral_radius(e3d_solver* s, int block);   /* Timestep::computeSpectralRadius, Solver/src/Timestep.cpp:26-121 */
int e3d_timestep(e3d_solver* s, int block);          /* Timestep::computeTimestep, Timestep.cpp:123-148 */
int e3d_gradients(e3d_solver* s, int block, int kind);/* Gradient::computeGradients: GreenGauss.cpp:12-234, LeastSquares.cpp:12-186 */
int e3d_limiters(e3d_solver* s, int block, int kind, double omega, double k); /* Limiter::computeLimiters: BarthJespersen.cpp:14-333, Venkatakrishnan.cpp:12-326 */
int e3d_flux_conv(e3d_solver* s, int block, int scheme);             /* FluxScheme::computeFluxConv, FluxScheme.cpp:16-211; AusmScheme.cpp:647-871 */
int e3d_flux_diss(e3d_solver* s, int block, int scheme, double beta);/* FluxScheme::computeFluxDiss, RoeScheme.cpp:12-311; AusmScheme.cpp:12-243 */
int e3d_update_internal(e3d_solver* s, int block, double alpha);    /* Updater::updateInternalBlock, Updater.cpp:12-78 */
int e3d_update_boundary(e3d_solver* s, int block);                   /* Updater::updateBoundary, Updater.cpp:80-88 */
/* CentralIrsSmoother::smoothResidual, CentralIrsSmoother.cpp:12-166: one Jacobi
 * step of central implicit residual smoothing (eps 0.8) of the convective and
 * dissipative residuals of the real cells; the reference's dissipative v and w
 * momentum start values (its lines 90-91 copy w into v and leave w unset)
 * follow the formula of the other eight arrays here.  A deck with
 * smoothing = 1 runs it in every stage of e3d_iterate / e3d_solve (FP64). */
int e3d_smooth_residual(e3d_solver* s, int block);
int e3d_halo(e3d_solver* s);                                         /* BlockCommunicator::updateBoundaries, MPI/src/BlockCommunicator.cpp:66-270 */
/* PostProcessing::computeFlowData (PostProcessing.cpp:198-217) for every block:
 * out[b*10 + 0..4] = sum over real cells of (Rc-Rd)^2 per equation,
 * out[b*10 + 5..9] = wall sums fy, fx, cmx, cmy, cmz
 * (Convergence.cpp:27-48, AerodynamicParameters.cpp:163-239). */
int e3d_flow_data(e3d_solver* s, double* out, int64_t count);

/* Whole outer iterations with fused kernels (Solver::solve body,
 * Solver/src/Solver.cpp:76-97); records are appended to the history. */
int e3d_iterate(e3d_solver* s, int n_iter);
/* Runs until the reference stop test (PostProcessing::checkStopSolver,
 * PostProcessing.cpp:59-83: iter+1 == max_iter or conv[0] <= criterion),
 * checking every `check_every` iterations; *iters_done = iterations run. */
int e3d_solve(e3d_solver* s, int max_iter, double criterion, int check_every, int* iters_done);
/* e3d_iterate with CUDA events around the launches on the solver stream:
 * *device_ms = device time of the n iterations. */
int e3d_iterate_timed(e3d_solver* s, int n_iter, double* device_ms);
int e3d_history_length(const e3d_solver* s, int* n);
int e3d_history(const e3d_solver* s, int first, int count, e3d_iter_record* out);

/* State transfer in block-local reference order (FP64 on the host side):
 * prim/limiter [5][n_all], grad [5][n_all][3], conv_res/diss_res/w0 [5][n_real],
 * dt/spectral_radius [n_real]. */
int e3d_state_get(e3d_solver* s, int block, const char* name, double* dst, int64_t count);
int e3d_state_set(e3d_solver* s, int block, const char* name, const double* src, int64_t count);

/* ---- batches of cases (Mach / alpha sweeps on meshes of uneven size) ----------
 * No counterpart in the reference (one case per run).  e3d_batch_create puts
 * every block of every case in one device arena; the cases must share gamma,
 * CFL, RK stages and the strategy choices and may differ in mesh, Mach, alpha
 * and chord.  e3d_batch_solve (all-tetrahedron meshes; FP32 or FP64) advances
 * the cases together over a work list of tiles, `iters_per_launch` outer
 * iterations per graph launch; a case leaves the work list once its density
 * drop reaches `criterion`, it has run max_iter iterations in all, or
 * (stall_window > 0) its last stall_window iterations brought no new minimum
 * 0.05 decades below the earlier ones.  The first call autotunes the form and
 * the tile size: the persistent cooperative kernel with a tuned grid, or the
 * same phases as per-pass launches over the tiles captured in one graph
 * (cached per problem-size bucket, and in $E3D_AUTOTUNE_CACHE if set;
 * E3D_BATCH_FORM=persistent|per-pass forces a form; e3d_batch_tuning reports
 * *grid = 0 for the per-pass form).  The tuning runs on a saved copy of the
 * state, which is restored: it never changes the solution.
 * A case whose residual turns non-finite leaves the batch (iters_done[c] =
 * -1, and later e3d_batch_solve calls skip it); the others go on, and the
 * call fails with E3D_ERR_NONFINITE only when no case is left.
 * iters_done[c] = iterations case c needed (n_cases entries);
 * *device_ms = device time of the whole solve.  e3d_iterate also works on a
 * batch (every case advances; no per-case stop), so after a case has left the
 * batch it fails with E3D_ERR_NONFINITE: that case's state stays non-finite. */
int e3d_batch_create(const e3d_case* const* cases, int n_cases, const e3d_options* opt, e3d_solver** out);
int e3d_batch_solve(e3d_solver* s, int max_iter, double criterion, int iters_per_launch, int stall_window,
                    int* iters_done, double* device_ms);
int e3d_case_count(const e3d_solver* s, int* n);
int e3d_case_history_length(const e3d_solver* s, int case_index, int* n);
int e3d_case_history(const e3d_solver* s, int case_index, int first, int count, e3d_iter_record* out);
int e3d_batch_tuning(const e3d_solver* s, int* tile_cells, int* grid, double* ms_per_iter, int* from_cache);

/* ---- block sharding: one case over several processes, one GPU each ------------
 * Replaces the reference's MPI distribution and transport
 * (BlockCommunicator::BlockCommunicator, MPI/src/BlockCommunicator.cpp:29-38;
 * updateBoundaries, :66-211; getMyBlocks, :284-294).  Rank r of n_ranks holds
 * the case blocks [first_block[r], first_block[r+1]) (first_block has
 * n_ranks + 1 entries, starts at 0, ends at the block count and rises
 * strictly).  e3d_shard_first_blocks fills it the reference's way: n_blocks /
 * n_ranks blocks per rank, one more for the first n_blocks % n_ranks ranks.
 *
 * Connexions inside a rank's range stay device copies.  The others are halo
 * entries of 5 primitives (rho u v w p) that cross ranks, ordered by peer
 * rank, then by connexion in topology order, then by cell pair: a rank's send
 * entries for peer r are exactly r's receive entries from it, the layout of
 * an all-to-all with per-peer counts.  e3d_case_shard_plan lists them on the
 * host (no GPU): per-peer entry counts, and when cells are non-null the
 * (block, block-local cell) pair of each entry, [2 * total] int32 each
 * (origins for send, destination ghosts for recv).
 *
 * A shard solver (e3d_shard_create) is an e3d_solver over its blocks; its
 * block indices are local (block b is case block first_block[rank] + b).  It
 * advances one iteration per e3d_iterate / e3d_iterate_timed call, and only
 * after its halo has crossed: before the first iteration and after each one,
 * e3d_shard_pack gathers the entries the peers need into a device buffer
 * (sum of send counts x 5 values in the solver's precision: double for
 * E3D_FP64, float for E3D_FP32), the caller moves the buffers (an all-to-all;
 * NCCL over NVLink, or host-staged), and e3d_shard_unpack writes the received
 * entries (device buffer, sum of recv counts x 5) into the ghost cells.  Both
 * queue work on the solver stream and return without waiting.  Iterating
 * earlier fails with E3D_ERR_STATE; more than one iteration per call with
 * E3D_ERR_ARG.
 *
 * Norms and forces: e3d_shard_flow_data hands out the raw per-block sums of
 * the iterations run since its last call ([n][local blocks][10]: five squared
 * residual sums, then the wall force terms, as e3d_flow_data; *n_iters = n;
 * `capacity` doubles room, else E3D_ERR_ARG and nothing is taken; out = NULL
 * only sets *n_iters), and fails with E3D_ERR_NONFINITE when one of them is
 * not finite.  The caller gathers every rank's, in block order
 * ([n][all blocks][10]), and hands them to e3d_shard_push_flow_data, which
 * appends whole-case records to the shard's history, summed in block order
 * as a single GPU sums them (the reference's MPI build sums per-rank partials
 * with MPI_Allreduce instead, BlockCommunicator.cpp:299-339).  e3d_solve and
 * e3d_batch_solve fail on a shard: its stop test needs every rank's norms. */
int e3d_shard_first_blocks(int n_blocks, int n_ranks, int32_t* first_block);
int e3d_case_shard_plan(const e3d_case* c, const int32_t* first_block, int n_ranks, int rank, int64_t* send_counts,
                        int64_t* recv_counts, int32_t* send_cells, int32_t* recv_cells);
int e3d_shard_create(const e3d_case* c, const int32_t* first_block, int n_ranks, int rank, const e3d_options* opt,
                     e3d_solver** out);
int e3d_shard_halo_counts(const e3d_solver* s, int64_t* send_counts, int64_t* recv_counts);
int e3d_shard_pack(e3d_solver* s, void* send);
int e3d_shard_unpack(e3d_solver* s, const void* recv);
int e3d_shard_flow_data(e3d_solver* s, double* out, int64_t capacity, int* n_iters);
int e3d_shard_push_flow_data(e3d_solver* s, const double* all_blocks, int n_iters);

/* ---- precision switch, warm start and the learned surrogate -------------------
 * No counterpart in the reference.
 * e3d_solver_set_precision: an FP32 solver becomes an FP64 solver in place
 * (E3D_FP64 or E3D_FP64_FMA); real cells take the carried FP64 conservative
 * state, histories and the iteration-0 reference norms carry on.  With
 * E3D_FP64_FMA, e3d_batch_solve runs FP64 kernels built with fused
 * multiply-add: the same discrete equations and converged solution, not
 * bit-identical to the reference (E3D_FP64 switches an FP64 solver back).  The FP32 path's
 * residual stops dropping near 5 orders (FP32 rounding of the fluxes); a run
 * to a deeper drop continues in FP64 from there, or with E3D_FP32_DELTA in
 * FP32 difference form: the state becomes an FP64 base plus FP32 differences,
 * the base and its residual (FP64) are renewed before every batch launch of
 * e3d_batch_solve, and the per-stage residual is the FP64 base residual plus
 * the change of the fluxes since the base, evaluated in FP32 in a form whose
 * rounding scales with that change.  The residual then keeps falling below the
 * FP32 floor at FP32 cost, to the FP64 path's converged state (not bit for bit).
 * First-order AUSM on all-tetrahedron meshes; E3D_ERR_ARG otherwise.  In this
 * form only e3d_batch_solve, e3d_history / e3d_batch_case_history, reading
 * "prim" and "w0" (the full state), and a further switch to E3D_FP64 or
 * E3D_FP64_FMA are available; other calls return E3D_ERR_STATE (E3D_FP32
 * leaves the solver in difference form).  Memory: 5 floats per cell and 5
 * doubles per cell of base state, 10 floats per real cell of differences and
 * base residual.
 * e3d_cell_features: surrogate inputs of every real cell of every case, in
 * device cell order (blocks in order, real cells in the order that
 * e3d_options.renumber chose; file order by default), 8 floats per
 * cell: centroid x y z, distance to the nearest wall-face centre of the
 * cell's case, Mach, alpha (deg), 0, 0.
 * The surrogate is a 4-layer MLP 6 -> 128 -> 128 -> 128 -> 5 with exact-erf
 * GELU, BF16 weights and FP32 accumulation on the tensor cores, trained by its
 * own forward/backward kernels and Adam on FP32 master weights (deterministic:
 * no floating-point atomics).  Samples: features (6 per row, as above) and the
 * converged conservative state (rho, rho u, rho v, rho w, rho E; 5 per row).
 * e3d_warm_start writes the predicted state into every real cell of every case
 * of a solver; cells whose prediction is not physical keep the freestream
 * start (*n_fallback counts them).  Call it after one iteration from the
 * freestream start so the residual drop is measured from the same reference
 * norm as a plain start's. */
int e3d_solver_set_precision(e3d_solver* s, int precision);
int e3d_cell_features(e3d_solver* s, float* out, int64_t n_floats);

typedef struct e3d_surrogate e3d_surrogate;
#define E3D_SURROGATE_PARAMS 36232 /* flat FP32 parameter count (padded layers) */
#define E3D_SURROGATE_NORM 24      /* feature mean[8], feature std[8], target scale[8] */
int e3d_surrogate_create(int device, uint64_t seed, double gamma, e3d_surrogate** out);
int e3d_surrogate_free(e3d_surrogate* m);
int e3d_surrogate_add_solution(e3d_surrogate* m, e3d_solver* s);
int e3d_surrogate_add_samples(e3d_surrogate* m, const float* features6, const float* states5, int64_t n);
int e3d_surrogate_sample_count(const e3d_surrogate* m, int64_t* n);
int e3d_surrogate_clear(e3d_surrogate* m);
int e3d_surrogate_train(e3d_surrogate* m, int steps, int batch, double lr, float* loss_per_step, double* final_loss);
int e3d_surrogate_gradient(e3d_surrogate* m, const float* features6, const float* states5, int n, float* grad,
                           double* loss);
int e3d_surrogate_predict(e3d_surrogate* m, const float* features6, int64_t n, float* states5);
int e3d_surrogate_get_params(const e3d_surrogate* m, float* params, float* norm);
int e3d_surrogate_set_params(e3d_surrogate* m, const float* params, const float* norm);
int e3d_warm_start(e3d_solver* s, e3d_surrogate* m, int* n_fallback);

/* Checkpoint / restart of the whole solver state (the reference's restart
 * writer is an empty stub, PostProcessing/src/OutputTecplot.cpp:475-494):
 * current primitives of every cell in the solver precision, the FP64
 * conservative state W0, the iteration count and the iteration-0 norms.
 * Query the size with e3d_state_bytes; export copies device -> host buffer
 * (pinned memory makes the copy faster), import the reverse. */
int e3d_state_bytes(const e3d_solver* s, int64_t* bytes);
int e3d_state_export(e3d_solver* s, void* host, int64_t bytes);
int e3d_state_import(e3d_solver* s, const void* host, int64_t bytes);

/* ---- residual norms without device allocation ---------------------------------
 * No counterpart in the reference (its norms are host loops).  For callers that
 * cannot allocate device memory where they need the norms: a host application
 * that owns all device memory through its own pool and forbids cudaMalloc in
 * plugins, or a time-stepping loop that must not allocate.  Computes, like
 * e3d_flow_data's out[b*10 + 0..4], the per-block sums of (rc - rd)^2 per
 * equation, with its scratch in a static device array of
 * E3D_NOALLOC_MAX_PARTIALS x 5 doubles (320 KiB, held by every GPU that loads
 * the library until exit) instead of cudaMalloc.
 *   rc, rd         device [5][n_cells] FP64 residuals, equation-major
 *   block_offsets  device [n_blocks+1]: block b owns cells [off[b], off[b+1])
 *   max_block_cells  largest block size; n_blocks * ceil(max_block_cells/4096)
 *                  must not exceed E3D_NOALLOC_MAX_PARTIALS (else E3D_ERR_LIMIT)
 *   out            device [n_blocks*5]
 *   stream         cudaStream_t or NULL
 * The host cannot read the device offsets, so it trusts max_block_cells: a
 * block with more cells than ceil(max_block_cells/4096)*4096 gets NaN in all
 * five of its outputs (found on the device; the call still returns E3D_OK),
 * never a silently truncated sum.
 * Queued on `stream`, nothing is allocated or freed.  The first call on a
 * device looks up the scratch address (cudaGetSymbolAddress): make it before
 * any stream capture.  Calls share the scratch, so calls that overlap on the
 * GPU race; order them on one stream. */
#define E3D_NOALLOC_MAX_PARTIALS 8192
int e3d_residual_norms_noalloc(const double* rc, const double* rd, int64_t n_cells, int n_blocks,
                               const int32_t* block_offsets, int max_block_cells, double* out, void* stream);

/* Measurement: per-kernel CUDA-event times of n eager iterations on the solver
 * stream.  names: comma-separated kernel names; launches/total_ms/bytes per row. */
int e3d_time_kernels(e3d_solver* s, int n_iter, char* names, int names_len, int* launches, double* total_ms,
                     double* bytes_per_launch, int max_rows, int* rows);
int e3d_launches_per_iteration(const e3d_solver* s, int* n);

#ifdef __cplusplus
}
#endif
#endif /* E3D_H */
