// engine.h -- internal declarations shared by the engine's translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "eplace_gpu.h"
#include "common.cuh"

namespace ep {

// Launch with programmatic stream serialization (the kernel's pdl_begin()
// orders it after the previous grid); captured into graphs as programmatic
// edges.
template <typename... KArgs, typename... Args>
inline void launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                     Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Stream priorities of the loop's two branches: the Poisson GEMMs (critical
// path) launch at the device's highest priority, the per-net pass that runs
// beside them at the lowest, so blocks of the GEMM chain are placed first
// whenever SM resources free up.
int launch_priority(bool high);

// launch_k with a scheduling priority attribute as well.
template <typename... KArgs, typename... Args>
inline void launch_kp(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                      int priority, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    attr[1].id = cudaLaunchAttributePriority;
    attr[1].val.priority = priority;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Per-net pass: one warp per task.  Nets of up to kWarpPins pins share a warp
// (floor(kWarpPins / degree) nets of one degree, a pin per lane); larger nets
// take a warp each, their first kStagedPins pins staged in shared memory.
constexpr int kWarpPins = 32;
constexpr int kStagedPins = 128;
constexpr int kNetWarps = 8;  // warps per block of the per-net pass
// Objects whose bin footprint may exceed this many bins take the
// block-per-object scatter / gather path.
constexpr int kSmallObjectBins = 16;

// ---- DCT / Poisson plan (dct.cu, dct_tc.cu) ---------------------------------
struct DctPlan {
    int nx = 0, ny = 0;
    int mode = 0;  // ep_dct_mode
    int fp64 = 0;  // maps in double (fast transforms only)
    // polls of a tensor-core pipeline wait before it gives up (ep_set_limits)
    unsigned wait_limit = 1u << 22;
    // FP32 operand tables (see dct.cu for their definitions)
    float *Cy = nullptr, *Cx = nullptr, *K = nullptr, *B3 = nullptr, *A4 = nullptr;
    // intermediates
    float *Tt = nullptr, *P = nullptr, *T3 = nullptr;
    // tensor-core path (bf16 hi/lo planes + TMA descriptors), dct_tc.cu
    void *tc = nullptr;
    // fast-transform path (twiddle tables, intermediates), dct_fft.cu
    void *fft = nullptr;
};

// fp64: the plan works on double maps (fast transforms only).
int dct_plan_init(DctPlan &p, int nx, int ny, float step_x, float step_y, int mode, int fp64,
                  std::string &err);
void dct_plan_free(DctPlan &p);
// rho (R [nx][ny]) -> field (vec2<R> [nx][ny]) and, when phi != nullptr, phi
// (R [nx][ny]); R = double when the plan was made with fp64, else float.
int dct_run(DctPlan &p, const void *rho, void *field, void *phi, const DevScalars *S, cudaStream_t st);
// Kernel launches of one dct_run.
inline int dct_launches(const DctPlan &p) { return p.mode == EP_DCT_FFT ? 3 : 4; }
// The tensor-core path reads rho as bf16 hi/lo planes written by the prep kernel.
void *dct_tc_rho_planes(DctPlan &p);

// ---- kernels (kernels.cu) ---------------------------------------------------
struct DeviceNetlist {
    int n_obj, n_nodes, n_terms;
    int n_nets, n_pins;
    const void *pos;         // [n_obj + n_terms] centres (vec2<R>); terminals after objects
    const float2 *size;      // [n_obj] (w, h)
    const uint8_t *flags;    // [n_obj]
    const float *npins;      // [n_obj] pin count (float, as the preconditioner reads it)
    const float *area;       // [n_obj] Module::area
    const float *sxy;        // [n_obj] local-smoothing scale sx*sy (EPlace/eplace.cpp:1061-1072)
    // pins in DEVICE order: nets grouped by degree (see the per-net pass in
    // kernels.cu); obj_pin_dev maps each object's pins to their positions
    const int32_t *pin_owner;
    const float2 *pin_off;
    const int32_t *obj_pin_start;  // [n_obj + 1] object -> its pins (reference pin order)
    const int32_t *obj_pin_dev;    // device position of each of those pins
    const int32_t *pin_obj_slot;   // [n_pins] device pin -> its slot in that object-major
                                   // order (-1 for terminal pins): where the per-net pass
                                   // writes the pin's gradient, so each object's pin
                                   // gradients lie contiguous for the combine
    const int4 *net_tasks;         // per warp of the per-net pass: degree, first pin, nets,
                                   // ceil(2^16 / degree) (0 for nets above kWarpPins pins)
    int n_net_tasks;
    const int32_t *big_objs;  // indices of kBig objects
    const int32_t *big_slot;  // object -> index in big_objs (or -1)
    int n_big_objs;
};

struct KernelCtx {
    Grid grid;
    double qscale, inv_qscale;
    double bin_area, inv_bin_area;
    double area_norm;  // stdArea + macroArea * td (overflow denominator)
    int exact_exp, lse;
    int fp64;           // working precision of the loop: 0 = FP32 (mixed), 1 = FP64
    int want_wl_value;  // also sum the smooth wirelength value (off in the hot loop)
    // per-block partials of the deterministic grid reductions
    double *part_prep, *part_wl, *part_comb, *part_hp;
};
int prep_blocks(const Grid &g);
// The L1/shared split of the loop's kernels (kernels.cu): every kernel asks
// for kLoopSmemBytes of shared memory, kernels that need more for the
// smallest split that holds them.
constexpr size_t kLoopSmemBytes = 64 * 1024;
int carveout_percent(size_t smem_bytes);
void set_loop_carveout();
void set_sgemm_carveout(int carveout);
// grid sizes of the reductions: 0 = per-net passes (both kernels), 1 = combine
int reduction_blocks(const DeviceNetlist &d, int which);

// Vectors typed void * hold vec2<R> (float2 / double2, KernelCtx::fp64) and
// rho holds R.
void launch_scatter(const KernelCtx &c, const DeviceNetlist &d, unsigned long long *node_q,
                    unsigned long long *filler_q, const DevScalars *S, cudaStream_t st);
void launch_prep(const KernelCtx &c, unsigned long long *node_q, unsigned long long *filler_q,
                 const float2 *static_map, void *rho, void *rho_bf16, float *node_f,
                 float *filler_f, int zero_maps, DevScalars *S, cudaStream_t st);
void launch_wirelength(const KernelCtx &c, const DeviceNetlist &d, void *pin_grad, DevScalars *S,
                       cudaStream_t st);
void launch_gather_big(const KernelCtx &c, const DeviceNetlist &d, const void *field, void *gd_big,
                       const DevScalars *S, cudaStream_t st);
void launch_combine(const KernelCtx &c, const DeviceNetlist &d, const void *field, const void *gd_big,
                    const void *pin_grad, void *g, const void *g_prev, const void *y_prev, void *dump_gd,
                    void *dump_gwl, int stepping, DevScalars *S, cudaStream_t st);
void launch_update(const KernelCtx &c, const DeviceNetlist &d, void *pos, void *x, const void *g, void *y_prev,
                   void *g_prev, DevScalars *S, cudaStream_t st);
// The update of the captured loop: also scatters the new positions into the
// (clear) density maps for the next evaluation, unless the step ends the stage.
void launch_update_scatter(const KernelCtx &c, const DeviceNetlist &d, void *pos, void *x, const void *g,
                           void *y_prev, void *g_prev, unsigned long long *node_q, unsigned long long *filler_q,
                           DevScalars *S, cudaStream_t st);
// Backtracking step rule: one trial move from y_k (ysave) along g_k, and the
// scalar commit of an accepted trial (combine in stepping mode 2 decides).
void launch_bktrk_move(const KernelCtx &c, const DeviceNetlist &d, const void *ysave, const void *g, const void *x,
                       void *pos, void *xtrial, const DevScalars *S, cudaStream_t st);
void launch_bktrk_commit(DevScalars *S, cudaStream_t st);
void launch_stage_begin(const KernelCtx &c, const DeviceNetlist &d, const void *pos, void *x, DevScalars *S,
                        cudaStream_t st);
void launch_wrap_up(const KernelCtx &c, const DeviceNetlist &d, void *pos, const void *x, cudaStream_t st);
// HPWL at the current positions; mode 0 stores it, mode 1 also applies the
// updatePenaltyFactor rule, mode 2 applies it only if a lambda update is pending.
void launch_hpwl(const KernelCtx &c, const DeviceNetlist &d, int mode, DevScalars *S, cudaStream_t st);

// ---- an engine's netlist for the learned warm start (gnn.cu) ------------------
// Host arrays owned by the engine; valid while it lives.
struct EngineGraph {
    uint64_t uid;                        // distinct per engine in this process
    int nn, n_obj, nt, nnet, np;         // movable nodes, objects, terminals, nets, pins
    const int32_t *pin_owner;            // [np] device pin order: object index, or n_obj + terminal
    const int32_t *net_first, *net_deg;  // [nnet] first device pin and pin count of each net
    const int32_t *pin_net;              // [np] net of each device pin
    const float *node_area, *node_pins;  // [nn]
    const float2 *term_centre;           // [nt]
    // the same netlist on the device
    const int32_t *d_pin_owner, *d_net_first, *d_net_deg, *d_pin_net;
    const int32_t *d_net_dev_order;  // [nnet] nets in device pin order (grouped by degree)
    int n_big_nets;                  // nets above kWarpPins pins: the first n_big_nets of that order
    const int32_t *d_obj_pin_start, *d_obj_pin_dev;  // object -> its device pins
    const float *d_area, *d_npins;                   // [n_obj]
    const void *d_pos;                               // [n_obj + nt] centres, vec2<R>
    int fp64;
    Grid grid;
    cudaStream_t st;
    int device;
    int *d_status;                   // the engine's device status word (EP_ERR_* bits)
};
int engine_graph(ep_engine *e, EngineGraph *g);
// Movable-node centres from a device float2 array (clamped into the core).
int engine_set_node_centres(ep_engine *e, const float2 *xy);
void engine_set_error(ep_engine *e, const char *msg);

// ---- quadratic placement (qp.cu) ---------------------------------------------
// Scalars of the device BiCGSTAB (per axis: X, Y), see qp.cu.
struct QpSolve {
    double rho[2], rho_old[2], alpha[2], w[2], r0sq[2], rr[2], bb[2], tol2[2], r0r[2];
    int it[2], restarts[2], active[2];
    int restart_mask, zero_mask, iters, max_it;
    int overflow;  // the last matrix build needed more entries than allocated
};
// Device view of one engine's quadratic placement: the netlist in device pin
// order (nets contiguous) plus the per-round systems and BiCGSTAB vectors,
// both axes side by side in float2 (x for the X system, y for the Y system).
struct QpDev {
    int nn, nnet;
    const int32_t *obj_pin_start, *obj_pin_dev;  // movable node -> its pins (modulePins order)
    const int32_t *pin_net;                      // device pin -> net
    const int32_t *net_first, *net_deg;          // net -> first device pin, pins
    const int32_t *net_order;                    // nets in device pin order
    int n_big;                                   // nets above kWarpPins pins (the head of net_order)
    const int32_t *owner;
    const float2 *off;
    int4 *bound;                                 // per net: x-min, x-max, y-min, y-max pin (in net)
    float2 *abspin;                              // [np] pin positions (device order) at the last bounds pass
    int32_t *count;                              // [2 nn] entries per row (X then Y)
    int32_t *row_x, *row_y;                      // [nn + 1] CSR offsets
    int32_t *col_x, *col_y;
    float *val_x, *val_y;
    float2 *diag, *rhs;
    float2 *x, *r, *r0, *p, *v, *s, *t;
    float2 *y, *z, *dinv;  // Jacobi-preconditioned solves: M^-1 p, M^-1 s, 1 / diagonal
    double *partials;
    unsigned *cnt;
    double *out;      // [4] sums of the last reduction (bounds: HPWL)
    QpSolve *solve;   // device BiCGSTAB state
    int32_t *scan;    // [qp_scan_blocks + 2] chunk totals of the row counts, then the two totals
    int cap_x, cap_y; // entries allocated per system
};
void qp_bounds(const QpDev &q, const float2 *pos, double *hpwl, cudaStream_t st);
// the rows read the pin positions the last qp_bounds stored
void qp_rows(const QpDev &q, int fill, cudaStream_t st);
// CSR row offsets of both systems from the counts, on the device
void qp_offsets(const QpDev &q, cudaStream_t st);
int qp_scan_blocks(int nn);
// r = b - A x and the solver's initial state (zero right-hand sides give x = 0)
void qp_init(const QpDev &q, int max_it, cudaStream_t st);
// enqueue `count` BiCGSTAB iterations (no-ops once both axes have stopped)
void qp_iterations(const QpDev &q, int count, bool jacobi, cudaStream_t st);
// 1 / diagonal of both systems (the Jacobi preconditioner), after a build
void qp_dinv(const QpDev &q, cudaStream_t st);
void qp_to_x(const QpDev &q, const float2 *pos, cudaStream_t st);
void qp_from_x(const QpDev &q, const Grid &g, const float2 *size, float2 *pos, cudaStream_t st);
void qp_center(const QpDev &q, const Grid &g, const float2 *size, float2 *pos, cudaStream_t st);
int qp_partial_blocks(int nn, int nnet);

}  // namespace ep
