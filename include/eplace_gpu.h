/* eplace_gpu.h -- C-ABI of the B200-native ePlace global-placement engine.
 *
 * Drop-in boundary for the Xinyu-lumos/ePlace global-placement inner loop.
 * Each entry point names the reference interface it replaces.  The engine
 * owns all device memory; inputs and outputs at this boundary are plain host
 * arrays (positions and gradients are centres, interleaved x,y, float32).
 * Every call returns an ep_status; the engine never calls exit() and never
 * traps the GPU.  One host thread per engine handle; all work is ordered on
 * the engine's CUDA stream (ep_set_stream).
 *
 * Object order follows the reference (EPlace/eplace.cpp:190-203): the
 * movable nodes of the netlist (dbNodes order), then the fillers the engine
 * creates.  Stage views (ep_stage) pick subsets of that order exactly as
 * EPlacer_2D::getPosition / getGradient do (EPlace/eplace.cpp:742-773).
 */
#ifndef EPLACE_GPU_H
#define EPLACE_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EP_ABI_VERSION 3

typedef enum ep_status {
    EP_OK = 0,
    EP_ERR_ARG = 1,     /* bad argument or netlist */
    EP_ERR_CUDA = 2,    /* a CUDA call failed (see ep_last_error) */
    EP_ERR_NAN = 3,     /* a non-finite value appeared in a reduction */
    EP_ERR_TIMEOUT = 4, /* a bounded device wait gave up */
    EP_ERR_STATE = 5,   /* call out of order (e.g. step before initialize) */
    EP_ERR_NOMEM = 6,   /* device allocation failed */
    EP_ERR_UNSUPPORTED = 7
} ep_status;

/* PLACEMENT_STAGE, EPlace/eplace.h:21-27. */
typedef enum ep_stage { EP_STAGE_MGP = 0, EP_STAGE_FILLERONLY = 1, EP_STAGE_CGP = 2 } ep_stage;

/* Wirelength model: WA (default) or LSE (gArg "LSE", EPlace/eplace.cpp:512-549). */
typedef enum ep_wl_model { EP_WL_WA = 0, EP_WL_LSE = 1 } ep_wl_model;

/* Exponential used by the wirelength model: the reference's fastExp
 * (1+a/1024)^1024 (PlaceCommon/global.h:457-471) or the exact exp. */
typedef enum ep_exp_mode { EP_EXP_FAST = 0, EP_EXP_EXACT = 1 } ep_exp_mode;

/* Step rule of EplaceNesterovOpt::opt_step (Optimization/nesterov.hpp:151-168):
 * 1/L (default), Barzilai-Borwein (gArg "bb"), backtracking (gArg "bktrk"). */
typedef enum ep_step_rule { EP_STEP_LIPSCHITZ = 0, EP_STEP_BB = 1, EP_STEP_BKTRK = 2 } ep_step_rule;

/* Arithmetic of the DCT/IDCT Poisson solve (replaces FFT_2D::doFFT,
 * FFT/fft.cpp:191-284): dense GEMMs in FP32 on the CUDA cores, on the
 * tcgen05 tensor cores with 3xBF16 split products (FP32 accumulate; bin
 * counts must be multiples of 128), or FP32 fast transforms (length-n FFTs
 * in shared memory; bin counts powers of two in [8, 2048]).  EP_DCT_AUTO
 * (the default) takes the fast transforms when the bin grid allows, else
 * the tensor cores when it allows, else the FP32 GEMMs; ep_info.dct_mode
 * tells which. */
typedef enum ep_dct_mode {
    EP_DCT_FP32 = 0,
    EP_DCT_BF16X3 = 1,
    EP_DCT_AUTO = 2,
    EP_DCT_FFT = 3
} ep_dct_mode;

/* Working precision of the global-placement loop.  EP_PREC_MIXED (the
 * default): positions, the optimizer's vectors, the Poisson solve, the field
 * gather and the wirelength terms in FP32 (as the reference computes them,
 * EPlace/eplace.cpp, PlaceCommon/objects.cpp), the overflow / HPWL /
 * Lipschitz / lambda reductions in FP64.  EP_PREC_FP64: the same kernels with
 * every vector, map and wirelength term in FP64 (the plain FP64 form; the
 * Poisson solve by fast transforms only, so bin counts must be powers of two
 * in [8, 2048]).  The density maps are int64 fixed point in both. */
typedef enum ep_precision { EP_PREC_MIXED = 0, EP_PREC_FP64 = 1 } ep_precision;

/* Netlist in plain arrays (what Parser/parser.cpp:44-97 builds into PlaceDB).
 * Nodes are movable; a node is a macro iff its height exceeds
 * common_row_height (PlaceDB/placedb.cpp:96-114).  Terminals are fixed.
 * Pins are listed net by net (net_start, CSR); pin_owner < num_nodes names a
 * node, otherwise terminal (pin_owner - num_nodes); pin offsets are from the
 * owner's centre (PlaceCommon/objects.cpp:454-459).  Rows are the site rows
 * of the .scl file (start.x, bottom, end.x, height). */
typedef struct ep_netlist {
    int32_t num_nodes;
    int32_t num_terminals;
    int32_t num_nets;
    int32_t num_rows;
    const float *node_w, *node_h;     /* [num_nodes] */
    const float *node_cx, *node_cy;   /* [num_nodes] initial centres */
    const float *term_llx, *term_lly; /* [num_terminals] lower-left corners */
    const float *term_w, *term_h;     /* [num_terminals] */
    const uint8_t *term_is_ni;        /* [num_terminals] "terminal_NI", may be NULL */
    const int32_t *net_start;         /* [num_nets + 1] */
    const int32_t *pin_owner;         /* [net_start[num_nets]] */
    const float *pin_dx, *pin_dy;     /* [net_start[num_nets]] */
    const float *row_llx, *row_lly, *row_urx, *row_h; /* [num_rows] */
    float common_row_height;          /* 0 = height of the last row (parser.cpp:271) */
} ep_netlist;

typedef struct ep_params {
    float target_density;   /* EPlacer_2D::setTargetDensity (EPlace/eplace.cpp:27-31) */
    float target_overflow;  /* mGP stop, gArg "targetOverflow", default 0.10 (nesterov.hpp:89-97) */
    int32_t bins_x, bins_y; /* 0 = the reference's rule (EPlace/eplace.cpp:237-261) */
    int32_t max_iterations; /* MAX_ITERATION, default 1000 (nesterov.hpp:36) */
    int32_t wl_model;       /* ep_wl_model */
    int32_t exp_mode;       /* ep_exp_mode */
    int32_t step_rule;      /* ep_step_rule */
    int32_t dct_mode;       /* ep_dct_mode */
    uint64_t filler_seed;   /* seed of the engine's own filler placement */
    int32_t device;         /* CUDA device ordinal */
    int32_t keep_maps;      /* 1 = keep per-evaluation bin maps queryable (tests) */
    int32_t precision;      /* ep_precision */
} ep_params;

/* Scalars of EPlacer_2D (EPlace/eplace.h:108-136) and the optimizer. */
typedef struct ep_scalars {
    double overflow;       /* globalDensityOverflow (tau) of the last evaluation */
    double lambda;         /* penalty factor */
    double hpwl;           /* HPWL of the last evaluation (bound-pin HPWL) */
    double last_hpwl;      /* lastHPWL of updatePenaltyFactor */
    double inv_gamma_x, inv_gamma_y;
    double wirelength;     /* smooth (WA/LSE) wirelength of the last evaluation;
                              summed only when ep_params.keep_maps is set, else 0 */
    double step;           /* last step size */
    double ns_param;       /* Nesterov a_k */
    int32_t iteration;     /* iter_count of the current stage */
    int32_t stage;         /* placementStage */
    int32_t mgp_iterations; /* mGPIterationCount */
    int32_t done;          /* stop condition reached */
} ep_scalars;

typedef struct ep_info {
    int32_t num_nodes, num_fillers, num_objects, num_terminals, num_nets, num_pins;
    int32_t num_macros, num_cells_and_fillers;
    int32_t bins_x, bins_y;
    float bin_step_x, bin_step_y;
    float core_llx, core_lly, core_urx, core_ury;
    float filler_w, filler_h;
    double std_area, macro_area;  /* ePlaceStdCellArea / ePlaceMacroArea */
    double total_row_area;
    double density_scale;         /* fixed-point units per unit area of the bin maps */
    int32_t dct_mode;             /* ep_dct_mode in use (never EP_DCT_AUTO) */
    int32_t precision;            /* ep_precision in use */
    /* wall seconds of ep_create: [0] checks, CUDA device, streams and
     * events, core region; [1] node classes, fillers, terminal and base
     * density maps; [2] the netlist's device layout (pin order, per-net
     * tasks, object -> pin maps); [3] device allocation and upload;
     * [4] transform plan and the final synchronisation */
    double create_seconds[5];
} ep_info;

typedef struct ep_run_stats {
    int32_t iterations;   /* steps taken in this run */
    double overflow;      /* tau at the stop */
    double hpwl;          /* exact HPWL of the final (main-solution) positions */
    double lambda;
    double seconds;       /* device time of the run, CUDA events */
    int64_t kernel_launches; /* engine kernels launched by this run */
} ep_run_stats;

/* Result of ep_quadratic_placement. */
typedef struct ep_qp_stats {
    int32_t rounds;            /* outer rounds (matrix rebuilds) */
    int32_t solver_iterations; /* BiCGSTAB iterations over all rounds */
    double hpwl;               /* HPWL after the last round (calcNetBoundPins) */
    double error_x, error_y;   /* |r| / |b| of the last solves (solver.error()) */
    double seconds;            /* device time, CUDA events */
    int64_t kernel_launches;   /* engine kernels this call launched */
} ep_qp_stats;

/* Per-kernel device times of one evaluation + step (ep_time_kernels). */
#define EP_MAX_TIMED_KERNELS 12
typedef struct ep_kernel_times {
    int32_t count;
    char names[EP_MAX_TIMED_KERNELS][24];
    double ms[EP_MAX_TIMED_KERNELS];     /* average device time per launch group */
    double bytes[EP_MAX_TIMED_KERNELS];  /* algorithmic bytes per launch group */
    double flops[EP_MAX_TIMED_KERNELS];  /* algorithmic flops per launch group */
    int32_t launches[EP_MAX_TIMED_KERNELS]; /* kernels in the group */
} ep_kernel_times;

typedef struct ep_engine ep_engine;

/* Limits of the engine's bounded device waits and retries; no counterpart in
 * the reference, which waits and retries without limit.  A tensor-core
 * pipeline wait gives up after wait_polls polls (default 2^22, about a
 * second), and the call that launched it ends with EP_ERR_TIMEOUT, the
 * engine still usable; a backtracking step (EP_STEP_BKTRK) gives up after
 * bktrk_trials rejected trials (default 64) with EP_ERR_TIMEOUT; a trial is
 * accepted when its 1/L is at least bktrk_accept times the step tried
 * (default 0.95, BKTRK_EPS of Optimization/nesterov.hpp:37).  Lowering them
 * exercises the give-up paths. */
typedef struct ep_limits {
    uint32_t wait_polls;
    int32_t bktrk_trials;
    double bktrk_accept;
} ep_limits;

/* ep_params with the reference defaults (rho_t 1.0, overflow 0.10, 1000 iterations). */
void ep_default_params(ep_params *p);
int32_t ep_abi_version(void);

/* PlaceDB + EPlacer_2D construction: copies the netlist to the device, sizes
 * the fillers (fillerInitialization, EPlace/eplace.cpp:61-208), builds the
 * bin grid and its static terminal / base density (binInitialization,
 * EPlace/eplace.cpp:221-412). */
ep_status ep_create(const ep_netlist *netlist, const ep_params *params, ep_engine **out);
void ep_destroy(ep_engine *e);
const char *ep_last_error(const ep_engine *e);
ep_status ep_get_info(const ep_engine *e, ep_info *info);
ep_status ep_get_limits(const ep_engine *e, ep_limits *limits);
ep_status ep_set_limits(ep_engine *e, const ep_limits *limits);
/* Use this CUDA stream (cudaStream_t) for all later work; NULL = engine's own. */
ep_status ep_set_stream(ep_engine *e, void *stream);
ep_status ep_synchronize(ep_engine *e);

/* EPlacer_2D::getPosition / setPosition (EPlace/eplace.cpp:759-804) for a
 * stage view; setPosition clamps into the core (PlaceDB::setModuleCenter_2D,
 * PlaceDB/placedb.cpp:253-288).  xy has 2*count floats. */
ep_status ep_get_positions(ep_engine *e, int32_t view, float *xy, int32_t count);
ep_status ep_set_positions(ep_engine *e, int32_t view, const float *xy, int32_t count);
/* ep_get_positions in double (an FP64 engine's centres without rounding). */
ep_status ep_get_positions_f64(ep_engine *e, int32_t view, double *xy, int32_t count);
/* PlaceDB::saveNodesLocation / loadNodesLocation (PlaceDB/placedb.cpp:1441-1465)
 * for every object, kept in device memory (no host copy). */
ep_status ep_save_positions(ep_engine *e);
ep_status ep_load_positions(ep_engine *e);

/* Optimizer state, for checkpoint and resume: everything a run in progress
 * carries between ep_nesterov_step calls -- every object's centre (y_k), the
 * main sequence x_k, the gradient, the previous step's point and gradient,
 * every scalar of EplaceNesterovOpt and the penalty (a_k, lambda, 1/gamma,
 * the last HPWL, overflow, step length, iteration count, stop flag) and the
 * stage -- as ep_state_size bytes in host memory.  ep_load_state, on an
 * engine created from the same netlist and parameters and initialized
 * (ep_initialize), in the saved stage, restores it: the ep_nesterov_step
 * calls that follow take the saved run's next steps bit for bit.  The
 * reference keeps positions only (PlaceDB::saveNodesLocation,
 * PlaceDB/placedb.cpp:1441-1465).  EP_ERR_ARG for a blob of another size,
 * design, grid or precision; EP_ERR_STATE before ep_initialize or in
 * another stage. */
uint64_t ep_state_size(const ep_engine *e);
ep_status ep_save_state(ep_engine *e, void *buf, uint64_t bytes);
ep_status ep_load_state(ep_engine *e, const void *buf, uint64_t bytes);

/* EPlacer_2D::initialization tail (EPlace/eplace.cpp:47-49): first
 * totalGradientUpdate with lambda 0, then penaltyFactorInitilization. */
ep_status ep_initialize(ep_engine *e);
/* EPlacer_2D::totalGradientUpdate (EPlace/eplace.cpp:687-738). */
ep_status ep_eval_gradient(ep_engine *e);
/* EPlacer_2D::getGradient (EPlace/eplace.cpp:742-756): the preconditioned
 * descent direction of the last evaluation for a stage view. */
ep_status ep_get_gradient(ep_engine *e, int32_t view, float *xy, int32_t count);
/* densityGradient / wirelengthGradient of the last evaluation, all objects
 * (keep_maps must be set). */
ep_status ep_get_component_gradients(ep_engine *e, float *density_xy, float *wirelength_xy);
/* The same in double: an FP64 engine's own values, an FP32 engine's widened.
 * No counterpart in the reference (whose vectors are float). */
ep_status ep_get_component_gradients_f64(ep_engine *e, double *density_xy, double *wirelength_xy);
/* Bin maps of the last evaluation, x-major [bins_x][bins_y] (keep_maps must
 * be set for node/filler/field): nodeDensity, fillerDensity,
 * terminalDensity, baseDensity (areas), E.x, E.y, phi.  Any may be NULL. */
ep_status ep_get_bin_maps(ep_engine *e, float *node, float *filler, float *terminal, float *base,
                          float *ex, float *ey, float *phi);
/* E.x, E.y and phi of the last evaluation in double (keep_maps must be set);
 * any may be NULL.  No counterpart in the reference. */
ep_status ep_get_field_f64(ep_engine *e, double *ex, double *ey, double *phi);
/* Raw fixed-point node / filler maps (int64, units of 1/density_scale). */
ep_status ep_get_density_fixed(ep_engine *e, int64_t *node, int64_t *filler);

ep_status ep_query(ep_engine *e, ep_scalars *s);
ep_status ep_set_lambda(ep_engine *e, double lambda);
/* penaltyFactorInitilization / updatePenaltyFactor (EPlace/eplace.cpp:812-883). */
ep_status ep_penalty_init(ep_engine *e);
ep_status ep_penalty_update(ep_engine *e);
/* PlaceDB::calcHPWL (PlaceDB/placedb.cpp:424-432) at the current positions. */
ep_status ep_hpwl(ep_engine *e, double *hpwl);

/* switch2FillerOnly / switch2cGP (EPlace/eplace.cpp:887-904).  For
 * EP_STAGE_FILLERONLY, filler_xy (2*num_fillers floats, lower-left corners as
 * setModuleLocation_2D_random writes them) may be NULL: the engine then draws
 * its own seeded positions. */
ep_status ep_switch_stage(ep_engine *e, int32_t stage, const float *filler_xy);

/* QPPlacer::quadraticPlacement (QPlace/qplace.cpp:20-106), the initial
 * placement of the reference's flow, on the device: the movable nodes start
 * at the core centre; each round builds the bound-pin quadratic model of
 * QPPlacer::createSparseMatrix (qplace.cpp:125-272, weights
 * 1/((p-1) max(d, 25)), the reference's Y pair test included) at the current
 * centres and solves X and Y with BiCGSTAB (identity preconditioner, at most
 * 100 iterations, warm start), then moves the nodes to the solution clamped
 * into the core.  Rounds stop when both solver errors are below 1e-6 after
 * the fifth, or after max_iterations + 1 rounds (0 = the reference's 20).
 * Fillers are not moved.  ep_initialize must run again afterwards. */
ep_status ep_quadratic_placement(ep_engine *e, int32_t max_iterations, ep_qp_stats *stats);
/* `rounds` rounds of the same quadratic model starting from the current
 * centres instead of the core centre (no convergence test), each with at
 * most solver_iterations BiCGSTAB iterations (0 = the reference's 100): a
 * short refinement of a start from elsewhere, e.g. ep_gnn_propose.
 * preconditioner 0: none (QPPlacer's IdentityPreconditioner); 1: Jacobi
 * (the systems' diagonals, as Eigen's DiagonalPreconditioner).  No
 * counterpart in the reference. */
ep_status ep_quadratic_refine(ep_engine *e, int32_t rounds, int32_t solver_iterations, int32_t preconditioner,
                              ep_qp_stats *stats);

/* FirstOrderOptimizer::opt (Optimization/opt.hpp:30-36) with
 * EplaceNesterovOpt (Optimization/nesterov.hpp:86-415) for the current stage:
 * init, steps until the stage's stop condition (or max_steps > 0 steps),
 * wrap_up.  The loop runs on the device (captured CUDA graphs, step size,
 * lambda and the stop test decided on the GPU).  With EP_STEP_BKTRK
 * (opt_step_bktrk, nesterov.hpp:310-369) each step is driven from the host,
 * since the number of trial evaluations is data-dependent; a step that finds
 * no acceptable trial within 64 tries ends the run with EP_ERR_TIMEOUT (the
 * reference retries without limit). */
ep_status ep_nesterov_run(ep_engine *e, int32_t max_steps, ep_run_stats *stats);
/* Binary netlist file, no counterpart in the reference (whose Bookshelf
 * parser, Parser/parser.cpp:44-819, is its slow I/O step): the arrays of
 * ep_netlist as they lie in memory (layout in eplace_b200/csrc/netbin.cu).
 * ep_netbin_write stores a netlist; ep_netbin_open maps a file and points
 * *nl at its arrays without copying (valid until ep_netbin_close(handle));
 * target_density and bins (may be NULL) receive the stored values. */
ep_status ep_netbin_write(const char *path, const ep_netlist *nl, float target_density, int32_t bins);
ep_status ep_netbin_open(const char *path, ep_netlist *nl, float *target_density, int32_t *bins,
                         void **handle);
void ep_netbin_close(void *handle);
/* Native Bookshelf reader, replacing Parser/parser.cpp:44-819 for what the
 * placer takes from a design (.aux naming .nodes/.nets/.pl/.scl; .wts is not
 * read): movable nodes first in file order, then terminals (terminal and
 * terminal_NI, the latter flagged) in file order; centres = .pl lower-left +
 * size/2 in float; pin offsets from the owner's centre; rows from the .scl
 * CoreRow blocks; common_row_height 0 (the last row's height).  *nl points
 * into arrays owned by *handle, valid until ep_bookshelf_close(handle).  On
 * failure *handle is NULL, the status EP_ERR_ARG (unreadable file, malformed
 * line, pin of an unknown node) or EP_ERR_NOMEM, and errbuf (may be NULL)
 * receives a message of at most errlen - 1 characters. */
ep_status ep_bookshelf_read(const char *aux_path, ep_netlist *nl, void **handle, char *errbuf, int32_t errlen);
/* .pl file of a design read by ep_bookshelf_read, its movable nodes at the
 * given centres (lower-left = centre - size/2 in float) and its terminals
 * where they were read (/FIXED, /FIXED_NI), under the design's own names.
 * Coordinates print with 9 significant digits, so a float read back is the
 * float written; PlaceDB::outputPL (PlaceDB/placedb.cpp:1159-1214, called
 * by outputBookShelf) prints them with %.0f. */
ep_status ep_bookshelf_write_pl(const void *handle, const char *path, const float *node_cx, const float *node_cy);
/* All files of a Bookshelf design (<dir>/<name>.aux, .nodes, .nets, .wts,
 * .pl at nl's centres, .scl) with sizes, offsets and coordinates printed
 * with 9 significant digits; PlaceDB::outputBookShelf
 * (PlaceDB/placedb.cpp:1022-1046) prints them with %.0f (offsets %.2f).
 * Node names and row site widths come from `design` (a handle of
 * ep_bookshelf_read whose node and terminal counts match nl) or, when it is
 * NULL, are o<i> / t<i> and 1; nets are named n<i>. */
ep_status ep_bookshelf_write(const char *dir, const char *name, const ep_netlist *nl, const void *design);
/* Site width of each row of a design read by ep_bookshelf_read (not part of
 * ep_netlist): count must equal its num_rows. */
ep_status ep_bookshelf_row_site_widths(const void *handle, float *out, int32_t count);
void ep_bookshelf_close(void *handle);

/* ep_nesterov_run for several independent engines (designs) at once, no
 * counterpart in the reference (which places one design per process): each
 * engine's loop runs on its own stream and the host interleaves their graph
 * replays, so small designs fill the GPU together.  Each engine ends as
 * ep_nesterov_run would leave it; stats (may be NULL) gets one entry per
 * engine.  Returns the first error met (the others still finish). */
ep_status ep_run_batch(ep_engine **engines, int32_t count, int32_t max_steps, ep_run_stats *stats);

/* The same loop one call at a time: begin = init(), step = "if
 * (!stop_condition()) opt_step(); updatePenaltyFactor()", end = wrap_up().
 * *stopped is set when the stop condition held and no step was taken. */
ep_status ep_nesterov_begin(ep_engine *e);
ep_status ep_nesterov_step(ep_engine *e, int32_t *stopped);
ep_status ep_nesterov_end(ep_engine *e);

/* Measurement hook with no reference counterpart: launches each kernel group
 * of one evaluation + step separately, reps times back to back between two
 * CUDA events on the engine's stream (less the time of any per-repetition
 * setup, such as clearing the density maps before a scatter), and reports the
 * average device time per launch with the group's algorithmic bytes / flops.
 * Positions, optimizer vectors and scalars are restored afterwards. */
ep_status ep_time_kernels(ep_engine *e, int32_t reps, ep_kernel_times *out);

/* Bin grid of ep_density_scatter_noalloc. */
typedef struct ep_scatter_grid {
    int32_t bins_x, bins_y;
    float core_llx, core_lly;     /* lower-left corner of the core region */
    float bin_step_x, bin_step_y;
    float target_density;         /* macro contributions are scaled by it */
} ep_scatter_grid;

/* Density scatter that allocates nothing.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: a host tool whose allocator has
 * reserved the device memory up front and forbids plugins from allocating, or
 * a caller that must not bring the device-wide synchronisation of a
 * cudaMalloc / cudaFree pair into its stream work.  All pointers are DEVICE
 * memory owned by the caller: object centres cx, cy, sizes w, h and flags
 * (bit 0 macro, bit 1 filler; NULL = all cells) for num_objects objects;
 * outputs node_out and filler_out (NULL allowed) are [bins_x][bins_y] float
 * maps of overlap areas, as EPlacer_2D::binNodeDensityUpdate accumulates them
 * (EPlace/eplace.cpp:1029-1133) and ep_get_bin_maps reports them.
 *
 * The int64 fixed-point scratch is a fixed file-scope device array of
 * 2 x 512 x 512 entries (4 MiB), held by every GPU that loads this library
 * until the process exits.  Grids beyond 512 x 512 bins are rejected with
 * EP_ERR_ARG and a message in err (err_len bytes, may be NULL).  The map
 * values are sums of contributions rounded to 2^-k area units, with
 * k = min(40, floor(62 - log2(1.05 * num_objects * bin_step_x * bin_step_y + 1)))
 * so that no bin sum can pass the int64 range (a contribution is at most a
 * bin's area); calls that would need k < 8 are rejected with EP_ERR_ARG.
 * target_density must be in (0, 1].  The first call in each CUDA context of
 * a device, made with that device current, looks up the scratch array's
 * device address (again after a cudaDeviceReset); make that first call before
 * any stream capture.  Every call zeroes and reuses the same scratch, so calls
 * that overlap on the GPU (on different streams, or from several threads)
 * race and must be serialised by the caller.  Work is
 * enqueued on `stream` (cudaStream_t, NULL = default stream). */
ep_status ep_density_scatter_noalloc(const ep_scatter_grid *grid, int32_t num_objects,
                                     const float *cx, const float *cy, const float *w,
                                     const float *h, const uint8_t *flags, float *node_out,
                                     float *filler_out, void *stream, char *err, int32_t err_len);

/* ---- learned warm start -----------------------------------------------------
 * No counterpart in the reference: a small message-passing network that
 * proposes the initial placement in place of QPPlacer::quadraticPlacement
 * (QPlace/qplace.cpp:20-103), which stays the fallback and the judge (a
 * caller keeps a proposal when its mGP run reaches the same overflow at an
 * HPWL within its tolerance of the QP-started run).
 *
 * Graph: an engine's movable nodes and terminals joined by its nets (read
 * from the engine's device arrays); mean aggregations node -> net -> node.
 * Input features per node: log(1 + area)/4, log(1 + pins)/3, terminal flag,
 * and its core-normalised coordinates after 8, 32 and 128 steps of
 * pad-anchored diffusion (movable nodes start at the core centre, terminals
 * stay at their centres, a step is node <- mean of its nets <- mean of their
 * pins).  Network: h0 = relu(W0 x + b0); three layers h = relu(W [h ; mean
 * of the nets' mean of h] + b), hidden 64; two heads q, f = d + 0.25
 * tanh(W4 h + b4), d the 128-step coordinates: q predicts the engine's
 * quadratic placement of the design, f its final mGP placement.  Weights
 * are FP32 masters with BF16 copies used by the forward pass (FP32
 * accumulate); training minimises the mean squared error of both heads
 * (normalised to the core) with Adam.  All work runs on the engine's
 * stream, in a workspace the network keeps (grown to the largest netlist;
 * the features of the last engine used are kept until ep_gnn_release). */
typedef struct ep_gnn ep_gnn;
int32_t ep_gnn_num_weights(void);
ep_status ep_gnn_create(int32_t device, uint64_t seed, ep_gnn **out);
void ep_gnn_destroy(ep_gnn *g);
const char *ep_gnn_last_error(const ep_gnn *g);
/* FP32 master weights (ep_gnn_num_weights floats); setting them resets Adam. */
ep_status ep_gnn_get_weights(ep_gnn *g, float *w);
ep_status ep_gnn_set_weights(ep_gnn *g, const float *w);
ep_status ep_gnn_release(ep_gnn *g, ep_engine *e);
/* Input features, [num_nodes + num_terminals][9] floats. */
ep_status ep_gnn_features(ep_gnn *g, ep_engine *e, float *x);
/* Predictions for the movable nodes (core coordinates), [num_nodes][4]:
 * q.x, q.y, f.x, f.y. */
ep_status ep_gnn_forward(ep_gnn *g, ep_engine *e, float *xy4);
/* Loss against targets [num_nodes][4] (core coordinates: the quadratic
 * placement's centre, then the final centre, of each movable node), the sum
 * of both heads' squared errors over 2 num_nodes, and its gradient with
 * respect to every weight (may be NULL). */
ep_status ep_gnn_loss_grad(ep_gnn *g, ep_engine *e, const float *target4, double *loss, float *grad);
/* One Adam step (learning rate lr) on that loss; *loss (may be NULL) is the
 * loss before the step. */
ep_status ep_gnn_train_step(ep_gnn *g, ep_engine *e, const float *target4, float lr, double *loss);
/* Move the engine's movable nodes to q + alpha (f - q), alpha in [0, 1],
 * clamped into the core; fillers stay.  Enqueued on the engine's stream;
 * ep_initialize must run again afterwards. */
ep_status ep_gnn_propose(ep_gnn *g, ep_engine *e, float alpha);
/* Polls of the tensor-core dense layers' mbarrier wait before it gives up
 * (polls < 0: the default, 2^22).  A wait that gives up leaves that forward
 * pass's outputs undefined and raises EP_ERR_TIMEOUT in the engine's status
 * word and in the network's own flag, which the network's next call reports
 * (the synchronous calls report their own pass's give-up before they
 * return).  No counterpart in the reference. */
ep_status ep_gnn_set_wait_limit(ep_gnn *g, int32_t polls);

#ifdef __cplusplus
}
#endif
#endif
