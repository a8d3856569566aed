// engine.cu -- host side of the engine and the C-ABI of include/eplace_gpu.h.
//
// Construction mirrors what the reference does before the hot loop:
//   PlaceDB::setCoreRegion            PlaceDB/placedb.cpp:52-77
//   PlaceDB::addNode (macro test)     PlaceDB/placedb.cpp:96-114
//   EPlacer_2D::fillerInitialization  EPlace/eplace.cpp:61-208
//   EPlacer_2D::binInitialization     EPlace/eplace.cpp:221-412
// with the same float arithmetic, so filler counts, bin geometry and the
// static terminal / base density maps equal the reference's.  The netlist is
// then laid out on the device as SoA arrays plus two CSRs (net -> pins,
// object -> pins) and the loop of kernels.cu / dct.cu runs there.
#include <algorithm>
#include <future>
#include <thread>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <chrono>
#include <cstring>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "engine.h"

using namespace ep;

struct ep_engine {
    // the error text keeps room for the out-of-memory message, so reporting
    // that one never allocates
    ep_engine() { err.reserve(256); }
    ep_params prm{};
    std::string err;
    int device = 0;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    // the per-net pass runs on its own stream, forked after prep and joined
    // before the gather / combine, beside the Poisson GEMMs
    cudaStream_t st_wl = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;

    int n_nodes = 0, n_fillers = 0, n_obj = 0, n_terms = 0, n_nets = 0, n_pins = 0;
    int n_macros = 0, n_cgp = 0;
    Grid grid{};
    KernelCtx kc{};
    float filler_w = 0, filler_h = 0;
    double std_area = 0, macro_area = 0, total_row_area = 0;

    std::vector<uint8_t> h_flags;  // kMacro / kFiller / kBig (no view bit)
    std::vector<float2> h_size;
    std::vector<int32_t> h_view[3];

    // working precision of the loop (ep_params.precision): vectors of the
    // optimizer, pin gradients and the field hold vec2<R> (v2 bytes each),
    // rho and phi hold R (r bytes each); R = double when fp64, else float
    int fp64 = 0;
    size_t v2 = sizeof(float2), r = sizeof(float);
    // device buffers
    void *pos = nullptr, *x = nullptr, *g = nullptr, *y_prev = nullptr, *g_prev = nullptr;
    void *pin_grad = nullptr, *gd_big = nullptr, *field = nullptr;
    float2 *size = nullptr, *pin_off = nullptr;
    void *dump_gd = nullptr, *dump_gwl = nullptr;  // component gradients (vec2<R>), keep_maps only
    float2 *static_map = nullptr;
    double2 *staging64 = nullptr;  // FP64 read-back of a view (made on first use)
    float2 *staging = nullptr;  // host-facing float2 positions / gradients of a view
    float2 *qp_pos = nullptr;   // FP32 centres the quadratic placement works on (FP64 engines)
    void *bk_ysave = nullptr, *bk_gtrial = nullptr, *bk_xtrial = nullptr;  // backtracking trials
    uint8_t *flags = nullptr;
    float *npins = nullptr, *area = nullptr, *node_f = nullptr, *filler_f = nullptr;
    void *rho = nullptr, *phi = nullptr;
    float *sxy = nullptr;
    int32_t *pin_owner = nullptr, *obj_pin_start = nullptr, *obj_pin_dev = nullptr, *pin_obj_slot = nullptr;
    int32_t *big_objs = nullptr, *big_slot = nullptr;
    int4 *net_tasks = nullptr;
    int32_t *view_idx[3] = {nullptr, nullptr, nullptr};
    unsigned long long *node_q = nullptr, *filler_q = nullptr;
    DevScalars *S = nullptr;
    DevScalars *hS = nullptr;  // pinned mirror
    // device memory: buffers are carved from a few large chunks (one
    // cudaMalloc per chunk, chunks doubling from 4 MiB), freed together
    std::vector<void *> allocs;
    unsigned char *arena_cur = nullptr;
    size_t arena_left = 0, arena_next = 4u << 20;

    DeviceNetlist dn{};
    DctPlan dct;

    int stage = EP_STAGE_MGP;
    bool initialized = false;
    bool in_run = false;

    cudaGraphExec_t graph = nullptr;
    int graph_iters = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ev_poll = nullptr;  // the run's read-back of `done` has landed
    std::mt19937_64 rng;
    void *snap = nullptr;     // ep_save_positions
    bool has_snap = false;
    // quadratic placement (qp.cu): net -> first device pin / pins, pin -> net
    std::vector<int32_t> h_net_first, h_net_deg, h_pin_net;
    // owner of each pin in device order (object index, terminals n_obj + t) and
    // the movable nodes' areas and pin counts, for the learned warm start
    std::vector<int32_t> h_pin_owner;
    std::vector<float> h_node_area, h_node_pins;
    std::vector<float2> h_term_centre;
    // device copies of the net -> device pins and pin -> net maps (made at
    // creation; the quadratic placement and the learned warm start read them)
    int32_t *net_first = nullptr, *net_deg = nullptr, *pin_net = nullptr;
    int32_t *net_dev_order = nullptr;  // nets in device pin order (grouped by degree)
    int n_big_nets = 0;                // nets above kWarpPins pins (the head of that order)
    double create_s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // ep_create phases (ep_info.create_seconds)
    int64_t qp_launches = 0;                         // kernels of the current quadratic placement call
    uint64_t uid = 0;  // distinct per engine created in this process
    QpDev qp{};
    bool qp_ready = false;
    size_t qp_cap_x = 0, qp_cap_y = 0;
    double *qp_out_h = nullptr;  // pinned mirror of qp.out
    QpSolve *qp_state_h = nullptr;  // pinned mirror of the device solver state
    int bk_trials = 64;       // backtracking trials per step before EP_ERR_TIMEOUT (ep_limits)
    int64_t launches = 0;     // engine kernels launched so far
    int64_t graph_kernels = 0;  // kernels in one replay of the step graph
};

namespace {

constexpr double kHostEps = 1.0e-15;

// A host allocation failed inside an entry point: the message fits the
// capacity reserved at construction, so this assignment does not allocate.
ep_status host_oom(ep_engine *e) {
    if (e) e->err.assign("out of host memory");
    return EP_ERR_NOMEM;
}

bool f_less_h(float a, float b) { return (double)(a - b) < -1.0 * kHostEps; }
bool f_greater_h(float a, float b) { return (double)(a - b) > 1.0 * kHostEps; }
bool f_equal_h(float a, float b) { return std::fabs((double)(a - b)) < kHostEps; }

double overlap_len_h(double a0, double a1, double b0, double b1) {
    double s = std::max(a0, b0), e = std::min(a1, b1);
    return s >= e ? 0.0 : (s - e);
}

double overlap_area_h(double l1, double b1, double r1, double t1, double l2, double b2, double r2,
                      double t2) {
    double h = overlap_len_h(l1, r1, l2, r2);
    if (h == 0) return 0;
    double v = overlap_len_h(b1, t1, b2, t2);
    if (v == 0) return 0;
    return h * v;
}

// PlaceDB::setModuleCenter_2D clamp (PlaceDB/placedb.cpp:257-281).
void clamp_center_h(const Grid &g, float &x, float &y, float w, float h) {
    if (x - 0.5 * w < g.llx) x = (float)(g.llx + 0.5 * w + kHostEps);
    if (x + 0.5 * w > g.urx) x = (float)(g.urx - 0.5 * w - kHostEps);
    if (y - 0.5 * h < g.lly) y = (float)(g.lly + 0.5 * h + kHostEps);
    if (y + 0.5 * h > g.ury) y = (float)(g.ury - 0.5 * h - kHostEps);
}

// PlaceDB::setModuleLocation_2D clamp of the lower-left corner
// (PlaceDB/placedb.cpp:207-228), then Module::setLocation_2D's centre.
void location_to_center_h(const Grid &g, float llx, float lly, float w, float h, float &cx, float &cy) {
    float x = llx, y = lly;
    if (x < g.llx) x = g.llx;
    if (x + w > g.urx) x = (float)(g.urx - w - kHostEps);
    if (y < g.lly) y = g.lly;
    if (y + h > g.ury) y = (float)(g.ury - h - kHostEps);
    cx = x + (float)0.5 * w;
    cy = y + (float)0.5 * h;
}

#define CK(call)                                                                   \
    do {                                                                           \
        cudaError_t _e = (call);                                                   \
        if (_e != cudaSuccess) {                                                   \
            e->err = std::string(#call) + ": " + cudaGetErrorString(_e);           \
            return EP_ERR_CUDA;                                                    \
        }                                                                          \
    } while (0)

template <typename T>
ep_status dalloc(ep_engine *e, T *&p, size_t n) {
    if (n == 0) n = 1;
    const size_t bytes = (n * sizeof(T) + 255) & ~(size_t)255;  // 256-byte aligned buffers
    if (bytes > e->arena_left) {
        const size_t chunk = std::max(bytes, e->arena_next);
        void *q = nullptr;
        cudaError_t rc = cudaMalloc(&q, chunk);
        if (rc != cudaSuccess) {
            e->err = std::string("cudaMalloc: ") + cudaGetErrorString(rc);
            p = nullptr;
            return EP_ERR_NOMEM;
        }
        e->allocs.push_back(q);
        e->arena_cur = static_cast<unsigned char *>(q);
        e->arena_left = chunk;
        e->arena_next = std::min<size_t>(2 * e->arena_next, (size_t)1 << 30);
    }
    p = reinterpret_cast<T *>(e->arena_cur);
    e->arena_cur += bytes;
    e->arena_left -= bytes;
    return EP_OK;
}

// n bytes of device memory for a buffer whose element type is the working
// precision's (vec2<R> or R).
ep_status dalloc_bytes(ep_engine *e, void *&p, size_t n) {
    unsigned char *q = nullptr;
    ep_status s = dalloc(e, q, n);
    p = q;
    return s;
}

template <typename T>
ep_status dupload(ep_engine *e, T *&p, const std::vector<T> &v) {
    ep_status s = dalloc(e, p, v.size());
    if (s) return s;
    if (!v.empty()) CK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return EP_OK;
}

// Reference bin-count rule, EPlace/eplace.cpp:230-261.
int bin_dimension(float std_area, float macro_area, int num_nodes, float core_w, float core_h,
                  float td) {
    float node_area = std_area + macro_area;
    float core_area = core_w * core_h;
    float avg = (float)(1.0 * node_area / num_nodes);
    float ideal = avg / td;
    int ideal_count = (int)(1.0 * (core_area / ideal) + 0.5f);
    for (int i = 1; i < 10; i++) {
        long a = (long)(2 << i) * (2 << i), b = (long)(2 << (i + 1)) * (2 << (i + 1));
        if (a <= ideal_count && b > ideal_count) return 2 << i;
    }
    return 1024;
}

ep_status check_netlist(ep_engine *e, const ep_netlist *nl) {
    if (!nl || nl->num_nodes <= 0 || nl->num_terminals < 0 || nl->num_nets < 0 || nl->num_rows <= 0) {
        e->err = "netlist: counts must be positive (nodes, rows) / non-negative";
        return EP_ERR_ARG;
    }
    if (!nl->node_w || !nl->node_h || !nl->node_cx || !nl->node_cy || !nl->row_llx ||
        !nl->row_lly || !nl->row_urx || !nl->row_h) {
        e->err = "netlist: missing node or row arrays";
        return EP_ERR_ARG;
    }
    if (nl->num_terminals > 0 && (!nl->term_llx || !nl->term_lly || !nl->term_w || !nl->term_h)) {
        e->err = "netlist: missing terminal arrays";
        return EP_ERR_ARG;
    }
    if (nl->num_nets > 0 && (!nl->net_start || !nl->pin_owner || !nl->pin_dx || !nl->pin_dy)) {
        e->err = "netlist: missing net / pin arrays";
        return EP_ERR_ARG;
    }
    if (nl->num_nets > 0) {
        if (nl->net_start[0] != 0) {
            e->err = "netlist: net_start[0] must be 0";
            return EP_ERR_ARG;
        }
        for (int n = 0; n < nl->num_nets; n++)
            if (nl->net_start[n + 1] < nl->net_start[n]) {
                e->err = "netlist: net_start must be non-decreasing";
                return EP_ERR_ARG;
            }
        int np = nl->net_start[nl->num_nets];
        for (int p = 0; p < np; p++)
            if (nl->pin_owner[p] < 0 || nl->pin_owner[p] >= nl->num_nodes + nl->num_terminals) {
                e->err = "netlist: pin_owner out of range";
                return EP_ERR_ARG;
            }
    }
    for (int i = 0; i < nl->num_nodes; i++)
        if (!(nl->node_w[i] > 0) || !(nl->node_h[i] > 0) || !std::isfinite(nl->node_cx[i]) ||
            !std::isfinite(nl->node_cy[i])) {
            e->err = "netlist: node sizes must be positive and centres finite";
            return EP_ERR_ARG;
        }
    for (int n = 0; n < nl->num_nets; n++)
        if (nl->net_start[n + 1] == nl->net_start[n]) {
            e->err = "netlist: empty net (the reference asserts bound pins exist)";
            return EP_ERR_ARG;
        }
    return EP_OK;
}

void set_view_flags(ep_engine *e, int stage, std::vector<uint8_t> &fl) {
    fl = e->h_flags;
    for (int o : e->h_view[stage]) fl[o] |= kInView;
}

ep_status upload_view(ep_engine *e, int stage) {
    std::vector<uint8_t> fl;
    set_view_flags(e, stage, fl);
    CK(cudaMemcpyAsync(e->flags, fl.data(), fl.size(), cudaMemcpyHostToDevice, e->st));
    CK(cudaStreamSynchronize(e->st));
    return EP_OK;
}

ep_status fetch_scalars(ep_engine *e) {
    CK(cudaMemcpyAsync(e->hS, e->S, sizeof(DevScalars), cudaMemcpyDeviceToHost, e->st));
    CK(cudaStreamSynchronize(e->st));
    return EP_OK;
}

template <typename F>
ep_status update_scalars(ep_engine *e, F f) {
    ep_status s = fetch_scalars(e);
    if (s) return s;
    f(*e->hS);
    CK(cudaMemcpyAsync(e->S, e->hS, sizeof(DevScalars), cudaMemcpyHostToDevice, e->st));
    CK(cudaStreamSynchronize(e->st));
    return EP_OK;
}

ep_status device_status(ep_engine *e) {
    int st = e->hS->status;
    if (st & (1 << EP_ERR_NAN)) {
        e->err = "non-finite value in a device reduction (overflow, HPWL, lambda or step)";
        return EP_ERR_NAN;
    }
    if (st & (1 << EP_ERR_TIMEOUT)) {
        e->err = "a bounded device wait gave up";
        return EP_ERR_TIMEOUT;
    }
    return EP_OK;
}

// Kernels one enqueue_eval launches (the DCT is four GEMMs).
int kernels_per_eval(const ep_engine *e) {
    const DeviceNetlist &d = e->dn;
    return 1 + 1 + dct_launches(e->dct) + (d.n_net_tasks > 0) + (d.n_big_objs > 0) + 1;
}

int kernels_per_hpwl(const ep_engine *e) { return e->dn.n_net_tasks > 0; }

// totalGradientUpdate: enqueue one gradient evaluation at the current
// positions.  The direction goes to gout; the Lipschitz sums compare with
// (g_ref, y_ref).
void enqueue_eval_to(ep_engine *e, int stepping, void *gout, const void *g_ref, const void *y_ref,
                     bool scatter = true) {
    e->launches += kernels_per_eval(e) - (scatter ? 0 : 1);
    cudaStream_t st = e->st;
    bool keep = e->prm.keep_maps != 0;
    if (keep) {
        cudaMemsetAsync(e->node_q, 0, sizeof(unsigned long long) * e->grid.nx * e->grid.ny, st);
        cudaMemsetAsync(e->filler_q, 0, sizeof(unsigned long long) * e->grid.nx * e->grid.ny, st);
    }
    if (scatter) launch_scatter(e->kc, e->dn, e->node_q, e->filler_q, e->S, st);
    void *bf = e->dct.mode == EP_DCT_BF16X3 ? dct_tc_rho_planes(e->dct) : nullptr;
    launch_prep(e->kc, e->node_q, e->filler_q, e->static_map, bf ? nullptr : e->rho, bf,
                keep ? e->node_f : nullptr, keep ? e->filler_f : nullptr, keep ? 0 : 1, e->S, st);
    // fork: the per-net pass needs the positions and 1/gamma (from prep), not
    // the field, so it runs beside the Poisson solve
    cudaEventRecord(e->ev_fork, st);
    cudaStreamWaitEvent(e->st_wl, e->ev_fork, 0);
    launch_wirelength(e->kc, e->dn, e->pin_grad, e->S, e->st_wl);
    cudaEventRecord(e->ev_join, e->st_wl);
    dct_run(e->dct, e->rho, e->field, keep ? e->phi : nullptr, e->S, st);
    cudaStreamWaitEvent(st, e->ev_join, 0);
    launch_gather_big(e->kc, e->dn, e->field, e->gd_big, e->S, st);
    launch_combine(e->kc, e->dn, e->field, e->gd_big, e->pin_grad, gout, g_ref, y_ref,
                   keep ? e->dump_gd : nullptr, keep ? e->dump_gwl : nullptr, stepping, e->S, st);
}

void enqueue_eval(ep_engine *e, int stepping) { enqueue_eval_to(e, stepping, e->g, e->g_prev, e->y_prev); }

// A step of the captured loop when the maps are not kept: the evaluation
// finds the maps already filled by the previous step's update (or by the
// scatter the run issues first), and the update fills them for the next one.
bool fused_loop(const ep_engine *e) { return e->prm.keep_maps == 0; }

void enqueue_step(ep_engine *e);

void enqueue_loop_step(ep_engine *e) {
    if (!fused_loop(e)) {
        enqueue_step(e);
        return;
    }
    enqueue_eval_to(e, 1, e->g, e->g_prev, e->y_prev, false);
    launch_update_scatter(e->kc, e->dn, e->pos, e->x, e->g, e->y_prev, e->g_prev, e->node_q, e->filler_q,
                          e->S, e->st);
    e->launches += 1;
}

void enqueue_step(ep_engine *e) {
    enqueue_eval(e, 1);
    launch_update(e->kc, e->dn, e->pos, e->x, e->g, e->y_prev, e->g_prev, e->S, e->st);
    e->launches += 1;
}

void enqueue_hpwl(ep_engine *e, int mode) {
    launch_hpwl(e->kc, e->dn, mode, e->S, e->st);
    e->launches += kernels_per_hpwl(e);
}

// One step of EplaceNesterovOpt::opt_step_bktrk (Optimization/nesterov.hpp:
// 310-369) plus updatePenaltyFactor: evaluate at y_k (1/L step, a_{k+1}),
// then move from y_k along g_k and re-evaluate at the trial point until the
// new 1/L is at least 0.95 of the step tried (combine, stepping mode 2),
// then make the trial the new iterate.  Returns with the step committed.
// The reference retries forever when no trial is accepted; the engine stops
// after e->bk_trials trials of one step and reports EP_ERR_TIMEOUT.
ep_status bktrk_step(ep_engine *e) {
    const size_t bytes = e->v2 * e->n_obj;
    cudaStream_t st = e->st;
    enqueue_eval(e, 1);
    CK(cudaMemcpyAsync(e->bk_ysave, e->pos, bytes, cudaMemcpyDeviceToDevice, st));
    for (int t = 0;; t++) {
        launch_bktrk_move(e->kc, e->dn, e->bk_ysave, e->g, e->x, e->pos, e->bk_xtrial, e->S, st);
        enqueue_eval_to(e, 2, e->bk_gtrial, e->g, e->bk_ysave);
        e->launches += 1;
        CK(cudaGetLastError());
        ep_status s = fetch_scalars(e);
        if (s) return s;
        if (e->hS->bk_accept || e->hS->status) break;
        if (t + 1 >= e->bk_trials) {
            s = update_scalars(e, [](DevScalars &h) {
                h.status |= 1 << EP_ERR_TIMEOUT;
                h.stop_pending = 1;
            });
            if (s) return s;
            break;
        }
    }
    // last_iter = cur_iter; cur_iter = new_iter (nesterov.hpp:365-367)
    CK(cudaMemcpyAsync(e->y_prev, e->bk_ysave, bytes, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(e->g_prev, e->g, bytes, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(e->g, e->bk_gtrial, bytes, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(e->x, e->bk_xtrial, bytes, cudaMemcpyDeviceToDevice, st));
    launch_bktrk_commit(e->S, st);
    e->launches += 1;
    enqueue_hpwl(e, 2);  // updatePenaltyFactor at the new positions
    CK(cudaGetLastError());
    return fetch_scalars(e);
}

ep_status build_graph(ep_engine *e, int iters) {
    if (e->graph) {
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    int64_t before = e->launches;
    CK(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < iters; i++) enqueue_loop_step(e);
    CK(cudaStreamEndCapture(e->st, &g));
    e->graph_kernels = e->launches - before;  // counted per replay, not at capture
    e->launches = before;
    cudaError_t rc = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    if (rc != cudaSuccess) {
        e->err = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(rc);
        e->graph = nullptr;
        return EP_ERR_CUDA;
    }
    e->graph_iters = iters;
    return EP_OK;
}

// A stage view of a working-precision vector, as float2 (the boundary's type).
template <typename R>
__global__ void k_gather_view(const int32_t *__restrict__ idx, int n, const vec2<R> *__restrict__ src,
                              float2 *__restrict__ dst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const vec2<R> v = src[idx[i]];
        dst[i] = make_float2((float)v.x, (float)v.y);
    }
}

// setPosition of a stage view: float2 centres clamped into the core
// (PlaceDB::setModuleCenter_2D) and stored in the working precision.
template <typename R>
__global__ void k_scatter_view(Grid g, const int32_t *__restrict__ idx, int n, const float2 *__restrict__ src,
                               const float2 *__restrict__ size, vec2<R> *__restrict__ pos) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int o = idx[i];
    float2 c = src[i];
    pos[o] = clamp_center<R>(g, mk2<R>((R)c.x, (R)c.y), size[o]);
}

// Precision conversion of n vec2 entries.
template <typename A, typename B>
__global__ void k_convert2(const vec2<A> *__restrict__ src, vec2<B> *__restrict__ dst, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = mk2<B>((B)src[i].x, (B)src[i].y);
}

template <typename R>
__global__ void k_gather_view64(const int32_t *__restrict__ idx, int n, const vec2<R> *__restrict__ src,
                                double2 *__restrict__ dst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const vec2<R> v = src[idx[i]];
        dst[i] = make_double2(v.x, v.y);
    }
}

void gather_view(ep_engine *e, int view, const void *src, int count) {
    const int32_t *idx = e->view_idx[view];
    if (e->fp64)
        k_gather_view<double><<<(count + 255) / 256, 256, 0, e->st>>>(idx, count, (const double2 *)src, e->staging);
    else
        k_gather_view<float><<<(count + 255) / 256, 256, 0, e->st>>>(idx, count, (const float2 *)src, e->staging);
}

ep_status check_view(ep_engine *e, int view, int count) {
    if (view < 0 || view > 2) {
        e->err = "view must be an ep_stage";
        return EP_ERR_ARG;
    }
    if (count != (int)e->h_view[view].size()) {
        e->err = "count does not match the size of the stage view";
        return EP_ERR_ARG;
    }
    return EP_OK;
}

}  // namespace

extern "C" {

int32_t ep_abi_version(void) { return EP_ABI_VERSION; }

void ep_default_params(ep_params *p) {
    std::memset(p, 0, sizeof(*p));
    p->target_density = 1.0f;
    p->target_overflow = 0.10f;
    p->max_iterations = 1000;
    p->wl_model = EP_WL_WA;
    p->exp_mode = EP_EXP_FAST;
    p->step_rule = EP_STEP_LIPSCHITZ;
    p->dct_mode = EP_DCT_AUTO;
    p->filler_seed = 1;
}

const char *ep_last_error(const ep_engine *e) { return e ? e->err.c_str() : "null engine"; }

// ep_create's body; the host arrays it builds may throw std::bad_alloc,
// which ep_create turns into EP_ERR_NOMEM.
extern "C++" {
// Host threads for a loop over n items (pins or nets): one per 100k items,
// at most 8 and at most the hardware's.
static int host_threads(long long n) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    return (int)std::max<long long>(1, std::min<long long>({8LL, (long long)hw, n / 100000 + 1}));
}

// fn(thread, begin, end) over `nth` contiguous ranges of [0, n), the first
// on the calling thread.
template <typename F>
static void parallel_ranges(int n, int nth, F &&fn) {
    if (nth <= 1 || n < 2) {
        fn(0, 0, n);
        return;
    }
    std::vector<std::future<void>> jobs;
    for (int t = 1; t < nth; t++)
        jobs.push_back(std::async(std::launch::async, [&fn, t, n, nth] {
            fn(t, (int)((long long)n * t / nth), (int)((long long)n * (t + 1) / nth));
        }));
    fn(0, 0, (int)((long long)n / nth));
    for (auto &j : jobs) j.get();
}
}  // extern "C++"

// Ascending sort of non-negative floats (the node areas) by their bit
// patterns, which order like the values: three 11-bit LSD radix passes.
// Anything else (a negative or NaN area) goes through std::sort.
static void sort_areas(std::vector<float> &a) {
    for (float v : a)
        if (!(v >= 0.0f)) {
            std::sort(a.begin(), a.end());
            return;
        }
    const size_t n = a.size();
    std::vector<uint32_t> k(n), tmp(n);
    for (size_t i = 0; i < n; i++) std::memcpy(&k[i], &a[i], 4);
    for (int shift = 0; shift < 33; shift += 11) {
        size_t cnt[2049] = {0};
        for (size_t i = 0; i < n; i++) cnt[((k[i] >> shift) & 2047) + 1]++;
        for (int d = 0; d < 2048; d++) cnt[d + 1] += cnt[d];
        for (size_t i = 0; i < n; i++) tmp[cnt[(k[i] >> shift) & 2047]++] = k[i];
        k.swap(tmp);
    }
    for (size_t i = 0; i < n; i++) std::memcpy(&a[i], &k[i], 4);
}

static ep_status create_engine(ep_engine *e, const ep_netlist *nl, const ep_params *params) {
    const auto t_start = std::chrono::steady_clock::now();
    auto lap = [&e, &t_start](int k) {
        const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
        double before = 0.0;
        for (int j = 0; j < k; j++) before += e->create_s[j];
        e->create_s[k] = t - before;
    };
    e->prm = *params;
    const ep_params &P = e->prm;
    ep_status s = check_netlist(e, nl);
    if (s) return s;
    if (!(P.target_density > 0) || P.target_density > 1.0f + 1e-6f) {
        e->err = "target_density must be in (0, 1]";
        return EP_ERR_ARG;
    }
    if (P.dct_mode != EP_DCT_FP32 && P.dct_mode != EP_DCT_BF16X3 && P.dct_mode != EP_DCT_AUTO &&
        P.dct_mode != EP_DCT_FFT) {
        e->err = "unknown dct_mode";
        return EP_ERR_ARG;
    }
    if (P.precision != EP_PREC_MIXED && P.precision != EP_PREC_FP64) {
        e->err = "unknown precision";
        return EP_ERR_ARG;
    }
    e->fp64 = P.precision == EP_PREC_FP64;
    e->v2 = e->fp64 ? sizeof(double2) : sizeof(float2);
    e->r = e->fp64 ? sizeof(double) : sizeof(float);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        e->err = "no CUDA device: the engine has no CPU fallback";
        return EP_ERR_CUDA;
    }
    e->device = P.device;
    CK(cudaSetDevice(P.device));
    CK(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
    e->own_stream = true;
    CK(cudaEventCreate(&e->ev0));
    CK(cudaEventCreate(&e->ev1));
    {
        int lo = 0, hi = 0;
        CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        CK(cudaStreamCreateWithPriority(&e->st_wl, cudaStreamNonBlocking, lo));
        CK(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&e->ev_poll, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming));
    }
    e->rng.seed(P.filler_seed);

    const int nn = nl->num_nodes, nt = nl->num_terminals, nnet = nl->num_nets, nr = nl->num_rows;
    const int np = nnet > 0 ? nl->net_start[nnet] : 0;
    e->n_nodes = nn;
    e->n_terms = nt;
    e->n_nets = nnet;
    e->n_pins = np;

    // ---- core region and row area (PlaceDB::setCoreRegion) ----
    float bottom = nl->row_lly[0];
    float top = (float)((double)nl->row_lly[nr - 1] + (double)nl->row_h[nr - 1]);
    float left = nl->row_llx[0], right = nl->row_urx[0];
    float total_row_area = 0;
    for (int r = 0; r < nr; r++) {
        left = std::min(left, nl->row_llx[r]);
        right = std::max(right, nl->row_urx[r]);
        float cur = (float)((double)(nl->row_urx[r] - nl->row_llx[r]) * (double)nl->row_h[r]);
        total_row_area += cur;
    }
    if (!(right > left) || !(top > bottom)) {
        e->err = "rows give an empty core region";
        return EP_ERR_ARG;
    }
    e->total_row_area = total_row_area;
    float row_h = nl->common_row_height > 0 ? nl->common_row_height : nl->row_h[nr - 1];
    Grid &g = e->grid;
    g.llx = left;
    g.lly = bottom;
    g.urx = right;
    g.ury = top;
    g.td = P.target_density;

    lap(0);
    // ---- node classes (PlaceDB::addNode) ----
    std::vector<uint8_t> is_macro(nn, 0);
    for (int i = 0; i < nn; i++) {
        if (f_greater_h(nl->node_h[i], row_h)) {
            is_macro[i] = 1;
            e->n_macros++;
        } else if (f_greater_h(row_h, nl->node_h[i])) {
            e->err = "a node is lower than the row height (PlaceDB::addNode rejects it)";
            return EP_ERR_ARG;
        }
    }

    // ---- fillers (fillerInitialization) ----
    // Terminal area on the rows, summed over terminals then rows in order.  A
    // row outside a terminal's y-range adds an exact zero, so only the rows
    // whose bottom lies below the terminal's top and above its bottom minus
    // the tallest row are visited (found by bisection), still in row order.
    float overlap = 0;
    {
        std::vector<int> by_y(nr);
        for (int r = 0; r < nr; r++) by_y[r] = r;
        std::stable_sort(by_y.begin(), by_y.end(), [&](int a, int b) { return nl->row_lly[a] < nl->row_lly[b]; });
        std::vector<float> ys(nr);
        float max_h = 0.0f;
        for (int k = 0; k < nr; k++) {
            ys[k] = nl->row_lly[by_y[k]];
            max_h = std::max(max_h, nl->row_h[by_y[k]]);
        }
        std::vector<int> cand;
        for (int t = 0; t < nt; t++) {
            if (nl->term_is_ni && nl->term_is_ni[t]) continue;
            const float tb = nl->term_lly[t], tt = nl->term_lly[t] + nl->term_h[t];
            const size_t k0 = std::lower_bound(ys.begin(), ys.end(), (float)((double)tb - max_h) - 1.0f) - ys.begin();
            const size_t k1 = std::upper_bound(ys.begin(), ys.end(), tt) - ys.begin();
            cand.assign(by_y.begin() + k0, by_y.begin() + k1);
            std::sort(cand.begin(), cand.end());
            for (int r : cand)
                overlap += (float)overlap_area_h(nl->term_llx[t], nl->term_lly[t],
                                                 nl->term_llx[t] + nl->term_w[t],
                                                 nl->term_lly[t] + nl->term_h[t], nl->row_llx[r],
                                                 nl->row_lly[r], nl->row_urx[r],
                                                 (float)((double)nl->row_lly[r] + nl->row_h[r]));
        }
    }
    float whitespace = total_row_area - overlap;
    float sa = 0, ma = 0;
    std::vector<float> areas(nn);
    for (int i = 0; i < nn; i++) {
        float a = nl->node_w[i] * nl->node_h[i];
        areas[i] = a;
        if (is_macro[i])
            ma += a;
        else
            sa += a;
    }
    e->std_area = sa;
    e->macro_area = ma;
    float node_scaled = sa + ma * P.target_density;
    float total_filler = whitespace * P.target_density - node_scaled;
    sort_areas(areas);
    int lo = (int)(0.05 * (float)nn), hi = (int)(0.95 * (float)nn);
    float acc = 0;
    for (int i = lo; i < hi; i++) acc += areas[i];
    float filler_area = hi > lo ? acc / ((float)(hi - lo)) : (nn > 0 ? areas[nn / 2] : 1.0f);
    e->filler_h = row_h;
    e->filler_w = filler_area / row_h;
    int nf = (int)(total_filler / filler_area + 0.5);
    if (nf < 0) nf = 0;
    e->n_fillers = nf;
    const int no = nn + nf;
    e->n_obj = no;

    // ---- bin grid (binInitialization) ----
    int nbx = P.bins_x, nby = P.bins_y;
    if (nbx <= 0 || nby <= 0) {
        nbx = nby = bin_dimension(sa, ma, nn, right - left, top - bottom, P.target_density);
    }
    if (nbx < 2 || nby < 2 || nbx > 4096 || nby > 4096) {
        e->err = "bins must be in [2, 4096]";
        return EP_ERR_ARG;
    }
    g.nx = nbx;
    g.ny = nby;
    g.sx = (right - left) / (float)nbx;
    g.sy = (top - bottom) / (float)nby;
    g.isx = 1.0f / g.sx;
    g.isy = 1.0f / g.sy;
    const int nb = nbx * nby;
    const float bin_area_f = g.sx * g.sy;

    // terminal density (EPlace/eplace.cpp:327-374) and base density
    // (:385-409): read-only inputs, computed on a second host thread while
    // this one lays out the objects and pins
    std::future<std::vector<float2>> stat_job = std::async(std::launch::async, [&, nbx, nby, nb]() {
        std::vector<float> term_d(nb, 0.0f), base_d(nb, 0.0f);
        auto bin_box = [&](int i, int j, float &l, float &b, float &r, float &t) {
            l = (float)i * g.sx + g.llx;
            b = (float)j * g.sy + g.lly;
            r = l + g.sx;
            t = b + g.sy;
        };
        for (int t = 0; t < nt; t++) {
            float llx = nl->term_llx[t], lly = nl->term_lly[t];
            float urx = llx + nl->term_w[t], ury = lly + nl->term_h[t];
            if (llx < g.llx || llx + nl->term_w[t] > g.urx) continue;
            if (lly < g.lly || lly + nl->term_h[t] > g.ury) continue;
            int i0 = (int)((llx - g.llx) / g.sx), i1 = (int)((urx - g.llx) / g.sx);
            int j0 = (int)((lly - g.lly) / g.sy), j1 = (int)((ury - g.lly) / g.sy);
            i1 = std::min(i1, nbx - 1);
            j1 = std::min(j1, nby - 1);
            for (int i = std::max(i0, 0); i <= i1; i++)
                for (int j = std::max(j0, 0); j <= j1; j++) {
                    float l, b, r, tt;
                    bin_box(i, j, l, b, r, tt);
                    term_d[(size_t)i * nby + j] +=
                        (float)(P.target_density * overlap_area_h(l, b, r, tt, llx, lly, urx, ury));
                }
        }
        {
            // only rows meeting a bin's y-range contribute non-zero terms; they
            // are summed in row order, as the reference's full loop would
            std::vector<std::vector<int>> rows_of(nby);
            for (int j = 0; j < nby; j++) {
                float l, b, r, t;
                bin_box(0, j, l, b, r, t);
                for (int rr = 0; rr < nr; rr++) {
                    double rb = nl->row_lly[rr], rt = (float)((double)nl->row_lly[rr] + nl->row_h[rr]);
                    if (overlap_len_h(b, t, rb, rt) != 0) rows_of[j].push_back(rr);
                }
            }
            for (int i = 0; i < nbx; i++)
                for (int j = 0; j < nby; j++) {
                    float l, b, r, t;
                    bin_box(i, j, l, b, r, t);
                    float avail = 0;
                    for (int rr : rows_of[j])
                        avail += (float)overlap_area_h(l, b, r, t, nl->row_llx[rr], nl->row_lly[rr],
                                                       nl->row_urx[rr],
                                                       (float)((double)nl->row_lly[rr] + nl->row_h[rr]));
                    base_d[(size_t)i * nby + j] =
                        f_equal_h(bin_area_f, avail) ? 0.0f : P.target_density * (bin_area_f - avail);
                }
        }
        std::vector<float2> st(nb);
        for (int k = 0; k < nb; k++) st[k] = make_float2(term_d[k], base_d[k]);
        return st;
    });

    // ---- objects ----
    e->h_size.resize(no);
    e->h_flags.assign(no, 0);
    std::vector<float2> pos(no + nt);
    std::vector<float> h_area(no), h_npins(no, 0.0f);
    for (int i = 0; i < nn; i++) {
        e->h_size[i] = make_float2(nl->node_w[i], nl->node_h[i]);
        h_area[i] = nl->node_w[i] * nl->node_h[i];
        if (is_macro[i]) e->h_flags[i] |= kMacro;
        float cx = nl->node_cx[i], cy = nl->node_cy[i];
        clamp_center_h(g, cx, cy, nl->node_w[i], nl->node_h[i]);
        pos[i] = make_float2(cx, cy);
    }
    // fillers at seeded random spots, drawn like setModuleLocation_2D_random
    // (PlaceDB/placedb.cpp:353-379): lower-left = u * (core size - filler size)
    for (int f = 0; f < nf; f++) {
        int o = nn + f;
        e->h_size[o] = make_float2(e->filler_w, e->filler_h);
        h_area[o] = e->filler_w * e->filler_h;
        e->h_flags[o] |= kFiller;
        float ux = (float)((e->rng() >> 40) * (1.0 / 16777216.0));
        float uy = (float)((e->rng() >> 40) * (1.0 / 16777216.0));
        float llx = ux * ((g.urx - g.llx) - e->filler_w);
        float lly = uy * ((g.ury - g.lly) - e->filler_h);
        float cx, cy;
        location_to_center_h(g, llx, lly, e->filler_w, e->filler_h, cx, cy);
        pos[o] = make_float2(cx, cy);
    }
    for (int t = 0; t < nt; t++)
        pos[no + t] = make_float2(nl->term_llx[t] + (float)0.5 * nl->term_w[t],
                                  nl->term_lly[t] + (float)0.5 * nl->term_h[t]);
    // big objects: may cover more bins than the thread-per-object path loops over.
    // Local smoothing depends on the size only, so its flags and sx*sy scale
    // are fixed here (EPlace/eplace.cpp:1061-1072, float division and product).
    std::vector<int32_t> big, big_slot(no, -1);
    std::vector<float> h_sxy(no);
    for (int o = 0; o < no; o++) {
        float w = e->h_size[o].x, h = e->h_size[o].y;
        float fsx = 1.0f, fsy = 1.0f;
        if (f_less_h(w, g.sx)) {
            e->h_flags[o] |= kSmoothX;
            fsx = w / g.sx;
        }
        if (f_less_h(h, g.sy)) {
            e->h_flags[o] |= kSmoothY;
            fsy = h / g.sy;
        }
        h_sxy[o] = fsx * fsy;
        long sx = f_less_h(w, g.sx) ? 2 : (long)(w / g.sx) + 2;
        long sy = f_less_h(h, g.sy) ? 2 : (long)(h / g.sy) + 2;
        if (sx * sy > kSmallObjectBins) {
            e->h_flags[o] |= kBig;
            big_slot[o] = (int32_t)big.size();
            big.push_back(o);
        }
    }

    // ---- pins: net CSR and the object -> pin CSR (pins in id order) ----
    lap(1);
    // ---- pins: net CSR and the object -> pin CSR (pins in id order) ----
    // Host loops over pins and nets run on `nth` threads in contiguous
    // ranges; every result is what the sequential loops give.
    const int nth = host_threads(np);
    std::vector<int32_t> owner(np), net_start(nnet + 1, 0);
    std::vector<float2> off(np);
    for (int n = 0; n <= nnet; n++) net_start[n] = nnet > 0 ? nl->net_start[n] : 0;
    parallel_ranges(np, nth, [&](int, int p0, int p1) {
        for (int p = p0; p < p1; p++) {
            const int ow = nl->pin_owner[p];
            owner[p] = ow < nn ? ow : no + (ow - nn);  // terminals follow all objects
            off[p] = make_float2(nl->pin_dx[p], nl->pin_dy[p]);
        }
    });
    // each object's pins in the reference's pin order (pin_slot: place of a
    // pin in that list), so the gradient sum runs in the reference's order:
    // a counting sort, each thread's range of pins starting where the
    // previous ranges' pins of the same object end
    std::vector<int32_t> ops(no + 1, 0), pin_slot(np, -1);
    {
        std::vector<std::vector<int32_t>> cnt(nth, std::vector<int32_t>(no, 0));
        parallel_ranges(np, nth, [&](int t, int p0, int p1) {
            for (int p = p0; p < p1; p++)
                if (owner[p] < no) cnt[t][owner[p]]++;
        });
        for (int o = 0; o < no; o++) {
            int32_t at = 0;
            for (int t = 0; t < nth; t++) {
                const int32_t c = cnt[t][o];
                cnt[t][o] = at;  // this thread's first slot, relative to the object's start
                at += c;
            }
            ops[o + 1] = ops[o] + at;
            if (o < nn) h_npins[o] = (float)at;
        }
        parallel_ranges(np, nth, [&](int t, int p0, int p1) {
            for (int p = p0; p < p1; p++)
                if (owner[p] < no) pin_slot[p] = ops[owner[p]] + cnt[t][owner[p]]++;
        });
    }
    // Device pin order for the per-net pass (kernels.cu): nets above
    // kWarpPins pins first, largest first (a warp each), then degree
    // kWarpPins down to 1, floor(kWarpPins / degree) nets per warp; original
    // order inside a degree.  Nets without pins take no task.
    std::vector<int4> net_tasks;
    std::vector<int32_t> dev_owner(np), dev_of_pin(np);
    std::vector<float2> dev_off(np);
    {
        std::vector<std::vector<int>> by_deg(kWarpPins + 1);
        std::vector<int> big_list;
        for (int n = 0; n < nnet; n++) {
            int deg = net_start[n + 1] - net_start[n];
            (deg > kWarpPins ? big_list : by_deg[deg]).push_back(n);
        }
        std::stable_sort(big_list.begin(), big_list.end(), [&](int a, int b) {
            return net_start[a + 1] - net_start[a] > net_start[b + 1] - net_start[b];
        });
        // nets in device order with their first device pin, then the copy
        std::vector<int> order;
        std::vector<int32_t> first;
        order.reserve(nnet);
        first.reserve(nnet);
        int q = 0;
        auto put_net = [&](int n) {
            order.push_back(n);
            first.push_back(q);
            const int at = q;
            q += net_start[n + 1] - net_start[n];
            return at;
        };
        e->n_big_nets = (int)big_list.size();
        for (int n : big_list) {
            int at = put_net(n);
            net_tasks.push_back(make_int4(net_start[n + 1] - net_start[n], at, 1, 0));
        }
        for (int d = kWarpPins; d >= 1; d--) {
            const size_t per = kWarpPins / d;
            for (size_t i = 0; i < by_deg[d].size(); i += per) {
                int at = q, count = (int)std::min(per, by_deg[d].size() - i);
                for (int j = 0; j < count; j++) put_net(by_deg[d][i + j]);
                net_tasks.push_back(make_int4(d, at, count, (65536 + d - 1) / d));
            }
        }
        parallel_ranges((int)order.size(), nth, [&](int, int i0, int i1) {
            for (int i = i0; i < i1; i++) {
                const int n = order[i], a = net_start[n], deg = net_start[n + 1] - a, at = first[i];
                for (int k = 0; k < deg; k++) {
                    dev_owner[at + k] = owner[a + k];
                    dev_off[at + k] = off[a + k];
                    dev_of_pin[a + k] = at + k;
                }
            }
        });
    }
    // quadratic placement: nets in device order
    e->h_pin_owner = dev_owner;
    e->h_term_centre.assign(pos.begin() + no, pos.end());
    e->h_node_area.assign(h_area.begin(), h_area.begin() + nn);
    e->h_node_pins.assign(h_npins.begin(), h_npins.begin() + nn);
    e->h_net_first.assign(nnet, 0);
    e->h_net_deg.assign(nnet, 0);
    e->h_pin_net.assign(np, 0);
    parallel_ranges(nnet, nth, [&](int, int n0, int n1) {
        for (int n = n0; n < n1; n++) {
            const int a = net_start[n], d = net_start[n + 1] - a;
            e->h_net_deg[n] = d;
            if (d > 0) e->h_net_first[n] = dev_of_pin[a];
            for (int k = 0; k < d; k++) e->h_pin_net[dev_of_pin[a + k]] = n;
        }
    });
    // each object's pins (reference order) -> their device positions, and back
    std::vector<int32_t> obj_pin_dev(std::max(ops[no], 1), 0), pin_obj_slot(std::max(np, 1), -1);
    parallel_ranges(np, nth, [&](int, int p0, int p1) {
        for (int p = p0; p < p1; p++)
            if (pin_slot[p] >= 0) {
                obj_pin_dev[pin_slot[p]] = dev_of_pin[p];
                pin_obj_slot[dev_of_pin[p]] = pin_slot[p];
            }
    });

    // stage views (EPlace/eplace.cpp:190-203)
    for (int v = 0; v < 3; v++) e->h_view[v].reserve(no);
    for (int o = 0; o < no; o++) {
        e->h_view[EP_STAGE_MGP].push_back(o);
        if (o >= nn) e->h_view[EP_STAGE_FILLERONLY].push_back(o);
        if (o >= nn || !is_macro[o]) e->h_view[EP_STAGE_CGP].push_back(o);
    }
    e->n_cgp = (int)e->h_view[EP_STAGE_CGP].size();

    // ---- fixed-point scale: every partial sum stays below 2^62 ----
    double total_area = 0;
    for (int o = 0; o < no; o++) total_area += (double)h_area[o];
    int qbits = (int)std::floor(62.0 - std::log2(total_area * 1.05 + 1.0));
    qbits = std::max(8, std::min(40, qbits));
    KernelCtx &kc = e->kc;
    kc.grid = g;
    kc.qscale = std::ldexp(1.0, qbits);
    kc.inv_qscale = std::ldexp(1.0, -qbits);
    kc.bin_area = (double)bin_area_f;
    kc.inv_bin_area = (double)(float)(1.0 / (double)bin_area_f);
    kc.area_norm = (double)(sa + ma * P.target_density);
    kc.exact_exp = P.exp_mode == EP_EXP_EXACT;
    kc.lse = P.wl_model == EP_WL_LSE;
    kc.want_wl_value = P.keep_maps ? 1 : 0;
    kc.fp64 = e->fp64;

    const std::vector<float2> stat = stat_job.get();
    lap(2);
    // ---- device ----
    const size_t v2 = e->v2;
    if ((s = dalloc_bytes(e, e->pos, v2 * (no + nt))) || (s = dalloc_bytes(e, e->x, v2 * no)) ||
        (s = dalloc_bytes(e, e->g, v2 * no)) || (s = dalloc_bytes(e, e->y_prev, v2 * no)) ||
        (s = dalloc_bytes(e, e->g_prev, v2 * no)) || (s = dupload(e, e->size, e->h_size)) ||
        (s = dupload(e, e->pin_off, dev_off)) || (s = dalloc_bytes(e, e->pin_grad, v2 * std::max(np, 1))) ||
        (s = dalloc_bytes(e, e->gd_big, v2 * std::max<size_t>(big.size(), 1))) ||
        (s = dalloc_bytes(e, e->field, v2 * nb)) || (s = dupload(e, e->static_map, stat)) ||
        (s = dalloc(e, e->staging, no + nt)) || (s = dalloc(e, e->flags, no)) ||
        (s = dupload(e, e->npins, h_npins)) || (s = dupload(e, e->area, h_area)) ||
        (s = dalloc_bytes(e, e->rho, e->r * nb)) || (s = dupload(e, e->sxy, h_sxy)) ||
        (s = dupload(e, e->pin_owner, dev_owner)) || (s = dupload(e, e->obj_pin_start, ops)) ||
        (s = dupload(e, e->obj_pin_dev, obj_pin_dev)) || (s = dupload(e, e->net_tasks, net_tasks)) ||
        (s = dupload(e, e->pin_obj_slot, pin_obj_slot)) ||
        (s = dupload(e, e->big_objs, big)) ||
        (s = dupload(e, e->big_slot, big_slot)) || (s = dalloc(e, e->node_q, nb)) ||
        (s = dalloc(e, e->filler_q, nb)) || (s = dalloc(e, e->S, 1)))
        return s;
    // centres: through the float2 staging buffer into the working precision
    // (exact for FP64)
    CK(cudaMemcpy(e->staging, pos.data(), sizeof(float2) * (no + nt), cudaMemcpyHostToDevice));
    if (e->fp64)
        k_convert2<float, double><<<(no + nt + 255) / 256, 256>>>(e->staging, (double2 *)e->pos, no + nt);
    else
        CK(cudaMemcpy(e->pos, e->staging, sizeof(float2) * (no + nt), cudaMemcpyDeviceToDevice));
    CK(cudaGetLastError());
    for (int v = 0; v < 3; v++)
        if ((s = dupload(e, e->view_idx[v], e->h_view[v]))) return s;
    {
        std::vector<int32_t> order;
        order.reserve(nnet);
        for (int p = 0; p < np; p++)
            if (p == 0 || e->h_pin_net[p] != e->h_pin_net[p - 1]) order.push_back(e->h_pin_net[p]);
        for (int n = 0; n < nnet; n++)  // nets without pins last, so the order holds every net
            if (e->h_net_deg[n] == 0) order.push_back(n);
        if ((s = dupload(e, e->net_first, e->h_net_first)) || (s = dupload(e, e->net_deg, e->h_net_deg)) ||
            (s = dupload(e, e->pin_net, e->h_pin_net)) || (s = dupload(e, e->net_dev_order, order)))
            return s;
    }
    if (P.step_rule == EP_STEP_BKTRK &&
        ((s = dalloc_bytes(e, e->bk_ysave, v2 * no)) || (s = dalloc_bytes(e, e->bk_gtrial, v2 * no)) ||
         (s = dalloc_bytes(e, e->bk_xtrial, v2 * no))))
        return s;
    if (P.keep_maps) {
        if ((s = dalloc(e, e->node_f, nb)) || (s = dalloc(e, e->filler_f, nb)) ||
            (s = dalloc_bytes(e, e->phi, e->r * nb)) || (s = dalloc_bytes(e, e->dump_gd, v2 * no)) ||
            (s = dalloc_bytes(e, e->dump_gwl, v2 * no)))
            return s;
    }
    CK(cudaMemset(e->node_q, 0, sizeof(unsigned long long) * nb));
    CK(cudaMemset(e->filler_q, 0, sizeof(unsigned long long) * nb));
    CK(cudaMemset(e->g, 0, v2 * no));
    CK(cudaMemset(e->g_prev, 0, v2 * no));
    CK(cudaMemset(e->y_prev, 0, v2 * no));
    CK(cudaMemset(e->x, 0, v2 * no));
    CK(cudaMemset(e->pin_grad, 0, v2 * std::max(np, 1)));
    CK(cudaMallocHost((void **)&e->hS, sizeof(DevScalars)));
    std::memset(e->hS, 0, sizeof(DevScalars));
    e->hS->a = 1.0;
    e->hS->stage = EP_STAGE_MGP;
    e->hS->max_iter = P.max_iterations > 0 ? P.max_iterations : 1000;
    e->hS->target_overflow = P.target_overflow > 0 ? P.target_overflow : 0.10f;
    e->hS->step_rule = P.step_rule;
    e->hS->bk_ratio = 0.95;
    CK(cudaMemcpy(e->S, e->hS, sizeof(DevScalars), cudaMemcpyHostToDevice));

    DeviceNetlist &d = e->dn;
    d.n_obj = no;
    d.n_nodes = nn;
    d.n_terms = nt;
    d.n_nets = nnet;
    d.n_pins = np;
    d.pos = e->pos;
    d.size = e->size;
    d.flags = e->flags;
    d.npins = e->npins;
    d.area = e->area;
    d.sxy = e->sxy;
    d.pin_owner = e->pin_owner;
    d.pin_off = e->pin_off;
    d.obj_pin_start = e->obj_pin_start;
    d.obj_pin_dev = e->obj_pin_dev;
    d.pin_obj_slot = e->pin_obj_slot;
    d.net_tasks = e->net_tasks;
    d.n_net_tasks = (int)net_tasks.size();
    d.big_objs = e->big_objs;
    d.big_slot = e->big_slot;
    d.n_big_objs = (int)big.size();
    if ((s = dalloc(e, kc.part_prep, (size_t)prep_blocks(g))) ||
        (s = dalloc(e, kc.part_wl, (size_t)2 * std::max(1, reduction_blocks(d, 0)))) ||
        (s = dalloc(e, kc.part_comb, (size_t)5 * std::max(1, reduction_blocks(d, 1)))) ||
        (s = dalloc(e, kc.part_hp, (size_t)2 * std::max(1, reduction_blocks(d, 0)))))
        return s;

    lap(3);
    int rc = EP_ERR_UNSUPPORTED;
    if (P.dct_mode == EP_DCT_AUTO && e->fp64) {
        // the FP64 form has the fast transforms only
        rc = dct_plan_init(e->dct, nbx, nby, g.sx, g.sy, EP_DCT_FFT, 1, e->err);
    } else if (P.dct_mode == EP_DCT_AUTO) {
        // fast transforms where the grid allows (fastest and most accurate),
        // else the tensor-core GEMMs, else the FP32 GEMMs (any grid)
        for (int mode : {EP_DCT_FFT, EP_DCT_BF16X3, EP_DCT_FP32}) {
            rc = dct_plan_init(e->dct, nbx, nby, g.sx, g.sy, mode, 0, e->err);
            if (rc != EP_ERR_UNSUPPORTED) break;
            dct_plan_free(e->dct);
            e->err.clear();
        }
    } else {
        rc = dct_plan_init(e->dct, nbx, nby, g.sx, g.sy, P.dct_mode, e->fp64, e->err);
    }
    if (rc) return (ep_status)rc;
    set_loop_carveout();
    e->stage = EP_STAGE_MGP;
    s = upload_view(e, EP_STAGE_MGP);
    if (s) return s;
    CK(cudaDeviceSynchronize());
    lap(4);
    return EP_OK;
}

ep_status ep_create(const ep_netlist *nl, const ep_params *params, ep_engine **out) {
    if (!out || !params) return EP_ERR_ARG;
    *out = nullptr;
    ep_engine *e = nullptr;
    try {
        e = new ep_engine();
    } catch (const std::bad_alloc &) {
        return EP_ERR_NOMEM;
    }
    *out = e;
    static std::atomic<uint64_t> next_uid{1};
    e->uid = next_uid++;
    try {
        return create_engine(e, nl, params);
    } catch (const std::bad_alloc &) {
        return host_oom(e);
    }
}

void ep_destroy(ep_engine *e) {
    if (!e) return;
    if (e->graph) cudaGraphExecDestroy(e->graph);
    dct_plan_free(e->dct);
    for (void *p : e->allocs) cudaFree(p);
    if (e->hS) cudaFreeHost(e->hS);
    if (e->qp_out_h) cudaFreeHost(e->qp_out_h);
    if (e->qp_state_h) cudaFreeHost(e->qp_state_h);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    if (e->ev_fork) cudaEventDestroy(e->ev_fork);
    if (e->ev_poll) cudaEventDestroy(e->ev_poll);
    if (e->ev_join) cudaEventDestroy(e->ev_join);
    if (e->st_wl) cudaStreamDestroy(e->st_wl);
    if (e->own_stream && e->st) cudaStreamDestroy(e->st);
    delete e;
}

ep_status ep_get_info(const ep_engine *e, ep_info *info) {
    if (!e || !info) return EP_ERR_ARG;
    info->num_nodes = e->n_nodes;
    info->num_fillers = e->n_fillers;
    info->num_objects = e->n_obj;
    info->num_terminals = e->n_terms;
    info->num_nets = e->n_nets;
    info->num_pins = e->n_pins;
    info->num_macros = e->n_macros;
    info->num_cells_and_fillers = e->n_cgp;
    info->bins_x = e->grid.nx;
    info->bins_y = e->grid.ny;
    info->bin_step_x = e->grid.sx;
    info->bin_step_y = e->grid.sy;
    info->core_llx = e->grid.llx;
    info->core_lly = e->grid.lly;
    info->core_urx = e->grid.urx;
    info->core_ury = e->grid.ury;
    info->filler_w = e->filler_w;
    info->filler_h = e->filler_h;
    info->std_area = e->std_area;
    info->macro_area = e->macro_area;
    info->total_row_area = e->total_row_area;
    info->density_scale = e->kc.qscale;
    info->dct_mode = e->dct.mode;
    info->precision = e->fp64 ? EP_PREC_FP64 : EP_PREC_MIXED;
    for (int k = 0; k < 5; k++) info->create_seconds[k] = e->create_s[k];
    return EP_OK;
}

ep_status ep_get_limits(const ep_engine *e, ep_limits *l) {
    if (!e || !l) return EP_ERR_ARG;
    l->wait_polls = e->dct.wait_limit;
    l->bktrk_trials = e->bk_trials;
    l->bktrk_accept = e->hS->bk_ratio;
    return EP_OK;
}

ep_status ep_set_limits(ep_engine *e, const ep_limits *l) {
    if (!e || !l) return EP_ERR_ARG;
    if (l->bktrk_trials < 1 || !(l->bktrk_accept > 0)) {
        e->err = "ep_limits: bktrk_trials must be >= 1 and bktrk_accept > 0";
        return EP_ERR_ARG;
    }
    e->dct.wait_limit = l->wait_polls;
    e->bk_trials = l->bktrk_trials;
    if (e->graph) {  // its launches hold the old poll limit
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
    }
    const double ratio = l->bktrk_accept;
    return update_scalars(e, [ratio](DevScalars &h) { h.bk_ratio = ratio; });
}

ep_status ep_set_stream(ep_engine *e, void *stream) {
    if (!e) return EP_ERR_ARG;
    if (e->graph) {
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
    }
    if (stream) {
        if (e->own_stream && e->st) cudaStreamDestroy(e->st);
        e->st = (cudaStream_t)stream;
        e->own_stream = false;
    } else if (!e->own_stream) {
        CK(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
        e->own_stream = true;
    }
    return EP_OK;
}

ep_status ep_synchronize(ep_engine *e) {
    if (!e) return EP_ERR_ARG;
    CK(cudaStreamSynchronize(e->st));
    return EP_OK;
}

ep_status ep_get_positions(ep_engine *e, int32_t view, float *xy, int32_t count) {
    if (!e || !xy) return EP_ERR_ARG;
    ep_status s = check_view(e, view, count);
    if (s) return s;
    if (count == 0) return EP_OK;
    gather_view(e, view, e->pos, count);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(xy, e->staging, sizeof(float2) * count, cudaMemcpyDeviceToHost, e->st));
    CK(cudaStreamSynchronize(e->st));
    return EP_OK;
}

ep_status ep_set_positions(ep_engine *e, int32_t view, const float *xy, int32_t count) try {
    if (!e || !xy) return EP_ERR_ARG;
    ep_status s = check_view(e, view, count);
    if (s) return s;
    if (count == 0) return EP_OK;
    CK(cudaMemcpyAsync(e->staging, xy, sizeof(float2) * count, cudaMemcpyHostToDevice, e->st));
    if (e->fp64)
        k_scatter_view<double><<<(count + 255) / 256, 256, 0, e->st>>>(e->grid, e->view_idx[view], count,
                                                                       e->staging, e->size, (double2 *)e->pos);
    else
        k_scatter_view<float><<<(count + 255) / 256, 256, 0, e->st>>>(e->grid, e->view_idx[view], count,
                                                                      e->staging, e->size, (float2 *)e->pos);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(e->st));
    return EP_OK;
} catch (const std::bad_alloc &) {
    return host_oom(e);
}

ep_status ep_eval_gradient(ep_engine *e) {
    if (!e) return EP_ERR_ARG;
    enqueue_eval(e, 0);
    CK(cudaGetLastError());
    ep_status s = fetch_scalars(e);
    if (s) return s;
    return device_status(e);
}

ep_status ep_initialize(ep_engine *e) try {
    if (!e) return EP_ERR_ARG;
    ep_status s = update_scalars(e, [](DevScalars &h) {
        h.lambda0_mode = 1;
        h.lambda = 0.0;
        h.status = 0;
        h.done = 0;
    });
    if (s) return s;
    enqueue_eval(e, 0);
    CK(cudaGetLastError());
    s = fetch_scalars(e);
    if (s) return s;
    e->initialized = true;
    return device_status(e);
} catch (const std::bad_alloc &) {
    return host_oom(e);
}

ep_status ep_get_gradient(ep_engine *e, int32_t view, float *xy, int32_t count) {
    if (!e || !xy) return EP_ERR_ARG;
    ep_status s = check_view(e, view, count);
    if (s) return s;
    if (count == 0) return EP_OK;
    gather_view(e, view, e->g, count);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(xy, e->staging, sizeof(float2) * count, cudaMemcpyDeviceToHost, e->st));
    CK(cudaStreamSynchronize(e->st));
    return EP_OK;
}

ep_status ep_get_component_gradients(ep_engine *e, float *density_xy, float *wirelength_xy) try {
    if (!e) return EP_ERR_ARG;
    if (!e->prm.keep_maps) {
        e->err = "component gradients need keep_maps";
        return EP_ERR_STATE;
    }
    const void *src[2] = {e->dump_gd, e->dump_gwl};
    float *dst[2] = {density_xy, wirelength_xy};
    std::vector<double2> tmp;
    for (int k = 0; k < 2; k++) {
        if (!dst[k]) continue;
        if (e->fp64) {
            tmp.resize(e->n_obj);
            CK(cudaMemcpyAsync(tmp.data(), src[k], sizeof(double2) * e->n_obj, cudaMemcpyDeviceToHost, e->st));
            CK(cudaStreamSynchronize(e->st));
            for (int o = 0; o < e->n_obj; o++) {
                dst[k][2 * o] = (float)tmp[o].x;
                dst[k][2 * o + 1] = (float)tmp[o].y;
            }
        } else {
            CK(cudaMemcpyAsync(dst[k], src[k], sizeof(float2) * e->n_obj, cudaMemcpyDeviceToHost, e->st));
        }
    }
    CK(cudaStreamSynchronize(e->st));
    return EP_OK;
} catch (const std::bad_alloc &) {
    return host_oom(e);
}

ep_status ep_get_component_gradients_f64(ep_engine *e, double *density_xy, double *wirelength_xy) try {
    if (!e) return EP_ERR_ARG;
    if (!e->prm.keep_maps) {
        e->err = "component gradients need keep_maps";
        return EP_ERR_STATE;
    }
    const void *src[2] = {e->dump_gd, e->dump_gwl};
    double *dst[2] = {density_xy, wirelength_xy};
    std::vector<float2> tmp;
    for (int k = 0; k < 2; k++) {
        if (!dst[k]) continue;
        if (e->fp64) {
            CK(cudaMemcpyAsync(dst[k], src[k], sizeof(double2) * e->n_obj, cudaMemcpyDeviceToHost, e->st));
        } else {
            tmp.resize(e->n_obj);
            CK(cudaMemcpyAsync(tmp.data(), src[k], sizeof(float2) * e->n_obj, cudaMemcpyDeviceToHost, e->st));
            CK(cudaStreamSynchronize(e->st));
            for (int o = 0; o < e->n_obj; o++) {
                dst[k][2 * o] = tmp[o].x;
                dst[k][2 * o + 1] = tmp[o].y;
            }
        }
    }
    CK(cudaStreamSynchronize(e->st));
    return EP_OK;
} catch (const std::bad_alloc &) {
    return host_oom(e);
}

ep_status ep_get_positions_f64(ep_engine *e, int32_t view, double *xy, int32_t count) {
    if (!e || !xy) return EP_ERR_ARG;
    ep_status s = check_view(e, view, count);
    if (s) return s;
    if (count == 0) return EP_OK;
    if (!e->staging64 && (s = dalloc(e, e->staging64, e->n_obj))) return s;
    const int32_t *idx = e->view_idx[view];
    if (e->fp64)
        k_gather_view64<double><<<(count + 255) / 256, 256, 0, e->st>>>(idx, count, (const double2 *)e->pos,
                                                                        e->staging64);
    else
        k_gather_view64<float><<<(count + 255) / 256, 256, 0, e->st>>>(idx, count, (const float2 *)e->pos,
                                                                       e->staging64);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(xy, e->staging64, sizeof(double2) * count, cudaMemcpyDeviceToHost, e->st));
    CK(cudaStreamSynchronize(e->st));
    return EP_OK;
}

ep_status ep_get_field_f64(ep_engine *e, double *ex, double *ey, double *phi) try {
    if (!e) return EP_ERR_ARG;
    if (!e->prm.keep_maps) {
        e->err = "field maps need keep_maps";
        return EP_ERR_STATE;
    }
    const int nb = e->grid.nx * e->grid.ny;
    std::vector<double2> f64(nb);
    std::vector<double> p64(phi ? nb : 0);
    if (e->fp64) {
        CK(cudaMemcpyAsync(f64.data(), e->field, sizeof(double2) * nb, cudaMemcpyDeviceToHost, e->st));
        if (phi) CK(cudaMemcpyAsync(p64.data(), e->phi, sizeof(double) * nb, cudaMemcpyDeviceToHost, e->st));
        CK(cudaStreamSynchronize(e->st));
    } else {
        std::vector<float2> f32(nb);
        std::vector<float> p32(phi ? nb : 0);
        CK(cudaMemcpyAsync(f32.data(), e->field, sizeof(float2) * nb, cudaMemcpyDeviceToHost, e->st));
        if (phi) CK(cudaMemcpyAsync(p32.data(), e->phi, sizeof(float) * nb, cudaMemcpyDeviceToHost, e->st));
        CK(cudaStreamSynchronize(e->st));
        for (int k = 0; k < nb; k++) f64[k] = make_double2(f32[k].x, f32[k].y);
        for (size_t k = 0; k < p32.size(); k++) p64[k] = p32[k];
    }
    for (int k = 0; k < nb; k++) {
        if (ex) ex[k] = f64[k].x;
        if (ey) ey[k] = f64[k].y;
        if (phi) phi[k] = p64[k];
    }
    return EP_OK;
} catch (const std::bad_alloc &) {
    return host_oom(e);
}

ep_status ep_get_bin_maps(ep_engine *e, float *node, float *filler, float *terminal, float *base,
                          float *ex, float *ey, float *phi) try {
    if (!e) return EP_ERR_ARG;
    const int nb = e->grid.nx * e->grid.ny;
    if ((node || filler || ex || ey || phi) && !e->prm.keep_maps) {
        e->err = "node/filler/field maps need keep_maps";
        return EP_ERR_STATE;
    }
    if (node) CK(cudaMemcpyAsync(node, e->node_f, sizeof(float) * nb, cudaMemcpyDeviceToHost, e->st));
    if (filler) CK(cudaMemcpyAsync(filler, e->filler_f, sizeof(float) * nb, cudaMemcpyDeviceToHost, e->st));
    std::vector<double> phi64;
    if (phi && e->fp64) {
        phi64.resize(nb);
        CK(cudaMemcpyAsync(phi64.data(), e->phi, sizeof(double) * nb, cudaMemcpyDeviceToHost, e->st));
    } else if (phi) {
        CK(cudaMemcpyAsync(phi, e->phi, sizeof(float) * nb, cudaMemcpyDeviceToHost, e->st));
    }
    std::vector<float2> tmp;
    if (terminal || base || ex || ey) tmp.resize(nb);
    if (terminal || base) {
        CK(cudaMemcpyAsync(tmp.data(), e->static_map, sizeof(float2) * nb, cudaMemcpyDeviceToHost, e->st));
        CK(cudaStreamSynchronize(e->st));
        for (int k = 0; k < nb; k++) {
            if (terminal) terminal[k] = tmp[k].x;
            if (base) base[k] = tmp[k].y;
        }
    }
    if ((ex || ey) && e->fp64) {
        std::vector<double2> f64(nb);
        CK(cudaMemcpyAsync(f64.data(), e->field, sizeof(double2) * nb, cudaMemcpyDeviceToHost, e->st));
        CK(cudaStreamSynchronize(e->st));
        for (int k = 0; k < nb; k++) {
            if (ex) ex[k] = (float)f64[k].x;
            if (ey) ey[k] = (float)f64[k].y;
        }
    } else if (ex || ey) {
        CK(cudaMemcpyAsync(tmp.data(), e->field, sizeof(float2) * nb, cudaMemcpyDeviceToHost, e->st));
        CK(cudaStreamSynchronize(e->st));
        for (int k = 0; k < nb; k++) {
            if (ex) ex[k] = tmp[k].x;
            if (ey) ey[k] = tmp[k].y;
        }
    }
    CK(cudaStreamSynchronize(e->st));
    for (size_t k = 0; k < phi64.size(); k++) phi[k] = (float)phi64[k];
    return EP_OK;
} catch (const std::bad_alloc &) {
    return host_oom(e);
}

ep_status ep_get_density_fixed(ep_engine *e, int64_t *node, int64_t *filler) {
    if (!e) return EP_ERR_ARG;
    if (!e->prm.keep_maps) {
        e->err = "fixed-point maps need keep_maps";
        return EP_ERR_STATE;
    }
    const int nb = e->grid.nx * e->grid.ny;
    if (node) CK(cudaMemcpyAsync(node, e->node_q, sizeof(int64_t) * nb, cudaMemcpyDeviceToHost, e->st));
    if (filler) CK(cudaMemcpyAsync(filler, e->filler_q, sizeof(int64_t) * nb, cudaMemcpyDeviceToHost, e->st));
    CK(cudaStreamSynchronize(e->st));
    return EP_OK;
}

ep_status ep_query(ep_engine *e, ep_scalars *out) {
    if (!e || !out) return EP_ERR_ARG;
    ep_status s = fetch_scalars(e);
    if (s) return s;
    const DevScalars &h = *e->hS;
    out->overflow = h.tau;
    out->lambda = h.lambda;
    out->hpwl = h.hpwl;
    out->last_hpwl = h.last_hpwl;
    out->inv_gamma_x = h.inv_gamma_x;
    out->inv_gamma_y = h.inv_gamma_y;
    out->wirelength = h.wirelength;
    out->step = h.step;
    out->ns_param = h.a;
    out->iteration = h.iter;
    out->stage = h.stage;
    out->mgp_iterations = h.mgp_iterations;
    out->done = h.done;
    return device_status(e);
}

ep_status ep_set_lambda(ep_engine *e, double lambda) {
    if (!e) return EP_ERR_ARG;
    return update_scalars(e, [lambda](DevScalars &h) { h.lambda = lambda; });
}

ep_status ep_penalty_init(ep_engine *e) {
    // lambda_0 from the component gradients of the last evaluation needs them
    // resident; the engine computes it inside ep_initialize's evaluation.
    if (!e) return EP_ERR_ARG;
    ep_status s = update_scalars(e, [](DevScalars &h) { h.lambda0_mode = 1; });
    if (s) return s;
    enqueue_eval(e, 0);
    CK(cudaGetLastError());
    s = fetch_scalars(e);
    if (s) return s;
    return device_status(e);
}

ep_status ep_penalty_update(ep_engine *e) {
    if (!e) return EP_ERR_ARG;
    enqueue_hpwl(e, 1);
    CK(cudaGetLastError());
    ep_status s = fetch_scalars(e);
    if (s) return s;
    return device_status(e);
}

ep_status ep_hpwl(ep_engine *e, double *hpwl) {
    if (!e || !hpwl) return EP_ERR_ARG;
    enqueue_hpwl(e, 0);
    CK(cudaGetLastError());
    ep_status s = fetch_scalars(e);
    if (s) return s;
    *hpwl = e->hS->hpwl_query;
    return EP_OK;
}

ep_status ep_switch_stage(ep_engine *e, int32_t stage, const float *filler_xy) try {
    if (!e) return EP_ERR_ARG;
    if (stage < 0 || stage > 2) {
        e->err = "unknown stage";
        return EP_ERR_ARG;
    }
    ep_status s;
    if (stage == EP_STAGE_FILLERONLY && e->n_fillers > 0) {
        // switch2FillerOnly: fillers re-spread at random (EPlace/eplace.cpp:887-894)
        std::vector<float2> fp(e->n_fillers);
        for (int f = 0; f < e->n_fillers; f++) {
            float llx, lly;
            if (filler_xy) {
                llx = filler_xy[2 * f];
                lly = filler_xy[2 * f + 1];
            } else {
                float ux = (float)((e->rng() >> 40) * (1.0 / 16777216.0));
                float uy = (float)((e->rng() >> 40) * (1.0 / 16777216.0));
                llx = ux * ((e->grid.urx - e->grid.llx) - e->filler_w);
                lly = uy * ((e->grid.ury - e->grid.lly) - e->filler_h);
            }
            float cx, cy;
            location_to_center_h(e->grid, llx, lly, e->filler_w, e->filler_h, cx, cy);
            fp[f] = make_float2(cx, cy);
        }
        if (e->fp64) {
            std::vector<double2> fp64(e->n_fillers);
            for (int f = 0; f < e->n_fillers; f++) fp64[f] = make_double2(fp[f].x, fp[f].y);
            CK(cudaMemcpyAsync((double2 *)e->pos + e->n_nodes, fp64.data(), sizeof(double2) * e->n_fillers,
                               cudaMemcpyHostToDevice, e->st));
            CK(cudaStreamSynchronize(e->st));  // fp64 goes out of scope
        } else {
            CK(cudaMemcpyAsync((float2 *)e->pos + e->n_nodes, fp.data(), sizeof(float2) * e->n_fillers,
                               cudaMemcpyHostToDevice, e->st));
        }
    }
    s = update_scalars(e, [stage](DevScalars &h) {
        if (stage == EP_STAGE_CGP) h.lambda = h.lambda / std::pow(1.1, h.mgp_iterations * 0.1);
        h.stage = stage;
    });
    if (s) return s;
    e->stage = stage;
    if (e->graph) {
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
    }
    return upload_view(e, stage);
} catch (const std::bad_alloc &) {
    return host_oom(e);
}

ep_status ep_nesterov_begin(ep_engine *e) {
    if (!e) return EP_ERR_ARG;
    if (!e->initialized) {
        e->err = "ep_initialize must run before the optimizer";
        return EP_ERR_STATE;
    }
    ep_status s = update_scalars(e, [](DevScalars &h) { h.step_cap = 0; });
    if (s) return s;
    launch_stage_begin(e->kc, e->dn, e->pos, e->x, e->S, e->st);
    e->launches += 1;
    CK(cudaGetLastError());
    e->in_run = true;
    return EP_OK;
}

ep_status ep_nesterov_step(ep_engine *e, int32_t *stopped) try {
    if (!e) return EP_ERR_ARG;
    if (!e->in_run) {
        e->err = "ep_nesterov_begin must run first";
        return EP_ERR_STATE;
    }
    ep_status s = fetch_scalars(e);
    if (s) return s;
    if (e->hS->done) {
        if (stopped) *stopped = 1;
        return device_status(e);
    }
    if (stopped) *stopped = 0;
    if (e->prm.step_rule == EP_STEP_BKTRK) {
        s = bktrk_step(e);
        if (s) return s;
        return device_status(e);
    }
    enqueue_step(e);
    enqueue_hpwl(e, 2);  // updatePenaltyFactor
    CK(cudaGetLastError());
    s = fetch_scalars(e);
    if (s) return s;
    return device_status(e);
} catch (const std::bad_alloc &) {
    return host_oom(e);
}

ep_status ep_nesterov_end(ep_engine *e) {
    if (!e) return EP_ERR_ARG;
    if (!e->in_run) return EP_OK;
    enqueue_hpwl(e, 2);
    launch_wrap_up(e->kc, e->dn, e->pos, e->x, e->st);
    e->launches += 1;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(e->st));
    e->in_run = false;
    return EP_OK;
}

}  // extern "C"

namespace {

// One optimizer run split into phases, so that several engines' runs can be
// interleaved (ep_run_batch): start, then launch / check until the stop,
// then finish.
struct RunState {
    int K = 8;
    bool bktrk = false;
    int64_t launches0 = 0;
    int cap = 0, launched = 0;
};

ep_status run_start(ep_engine *e, int32_t max_steps, RunState &r) {
    ep_status s = ep_nesterov_begin(e);
    if (s) return s;
    s = update_scalars(e, [max_steps](DevScalars &h) { h.step_cap = max_steps > 0 ? max_steps : 0; });
    if (s) return s;
    r.bktrk = e->prm.step_rule == EP_STEP_BKTRK;
    if (!r.bktrk && (!e->graph || e->graph_iters != r.K)) {
        s = build_graph(e, r.K);
        if (s) return s;
    }
    r.launches0 = e->launches - 1;  // include the stage-begin kernel
    CK(cudaEventRecord(e->ev0, e->st));
    r.cap = (max_steps > 0 ? max_steps : e->hS->max_iter + 1) + r.K;
    r.launched = 0;
    if (!r.bktrk && fused_loop(e)) {
        // the first step's maps (the graph's steps start at prep)
        launch_scatter(e->kc, e->dn, e->node_q, e->filler_q, e->S, e->st);
        e->launches += 1;
    }
    return EP_OK;
}

// Enqueue the next K steps (one graph replay) and the read-back of `done`;
// backtracking steps run one at a time from the host.
ep_status run_launch(ep_engine *e, RunState &r) {
    if (r.bktrk) {
        ep_status s = fetch_scalars(e);
        if (s || e->hS->done) return s;
        r.launched++;
        return bktrk_step(e);
    }
    CK(cudaGraphLaunch(e->graph, e->st));
    e->launches += e->graph_kernels;
    r.launched += r.K;
    CK(cudaMemcpyAsync(&e->hS->done, &e->S->done, sizeof(int), cudaMemcpyDeviceToHost, e->st));
    CK(cudaEventRecord(e->ev_poll, e->st));
    return EP_OK;
}

ep_status run_check(ep_engine *e, RunState &r, bool &more) {
    if (r.bktrk) {
        more = !e->hS->done && r.launched <= r.cap;
        return EP_OK;
    }
    CK(cudaEventSynchronize(e->ev_poll));
    more = !(e->hS->done || r.launched > r.cap + r.K);
    return EP_OK;
}

ep_status run_finish(ep_engine *e, RunState &r, ep_run_stats *stats) {
    if (!r.bktrk && fused_loop(e)) {
        // clear in any case: the maps must be empty when the next evaluation
        // scatters (the stopping step scatters nothing, so this is a no-op
        // unless the loop was cut off)
        const size_t nb = (size_t)e->grid.nx * e->grid.ny;
        CK(cudaMemsetAsync(e->node_q, 0, sizeof(unsigned long long) * nb, e->st));
        CK(cudaMemsetAsync(e->filler_q, 0, sizeof(unsigned long long) * nb, e->st));
    }
    enqueue_hpwl(e, 2);  // the lambda update owed by the last step
    launch_wrap_up(e->kc, e->dn, e->pos, e->x, e->st);
    e->launches += 1;
    CK(cudaEventRecord(e->ev1, e->st));
    enqueue_hpwl(e, 0);
    CK(cudaGetLastError());
    ep_status s = fetch_scalars(e);
    e->in_run = false;
    if (s) return s;
    if (stats) {
        float ms = 0;
        cudaEventElapsedTime(&ms, e->ev0, e->ev1);
        stats->iterations = e->hS->iter;
        stats->overflow = e->hS->tau;
        stats->hpwl = e->hS->hpwl_query;
        stats->lambda = e->hS->lambda;
        stats->seconds = ms * 1e-3;
        stats->kernel_launches = e->launches - r.launches0;
    }
    return device_status(e);
}

}  // namespace

extern "C" {

ep_status ep_nesterov_run(ep_engine *e, int32_t max_steps, ep_run_stats *stats) try {
    if (!e) return EP_ERR_ARG;
    RunState r;
    ep_status s = run_start(e, max_steps, r);
    if (s) return s;
    for (bool more = true; more;) {
        if ((s = run_launch(e, r)) || (s = run_check(e, r, more))) {
            e->in_run = false;
            return s;
        }
    }
    return run_finish(e, r, stats);
} catch (const std::bad_alloc &) {
    return host_oom(e);
}

ep_status ep_run_batch(ep_engine **engines, int32_t count, int32_t max_steps, ep_run_stats *stats) try {
    if (!engines || count < 0) return EP_ERR_ARG;
    for (int i = 0; i < count; i++)
        if (!engines[i]) return EP_ERR_ARG;
    std::vector<RunState> rs(count);
    std::vector<char> active(count, 0);
    ep_status first_error = EP_OK;
    auto stop_all = [&]() {
        for (int i = 0; i < count; i++) engines[i]->in_run = false;
    };
    for (int i = 0; i < count; i++) {
        ep_status s = run_start(engines[i], max_steps, rs[i]);
        if (s) {
            stop_all();
            return s;
        }
        active[i] = 1;
    }
    for (int left = count; left > 0;) {
        for (int i = 0; i < count; i++)
            if (active[i]) {
                ep_status s = run_launch(engines[i], rs[i]);
                if (s) {
                    stop_all();
                    return s;
                }
            }
        for (int i = 0; i < count; i++) {
            if (!active[i]) continue;
            bool more = true;
            ep_status s = run_check(engines[i], rs[i], more);
            if (s) {
                stop_all();
                return s;
            }
            if (!more) {
                s = run_finish(engines[i], rs[i], stats ? &stats[i] : nullptr);
                if (s && !first_error) first_error = s;
                active[i] = 0;
                left--;
            }
        }
    }
    return first_error;
} catch (const std::bad_alloc &) {
    for (int i = 0; i < count; i++) engines[i]->in_run = false;
    return EP_ERR_NOMEM;
}

ep_status ep_save_positions(ep_engine *e) {
    if (!e) return EP_ERR_ARG;
    if (!e->snap) {
        ep_status s = dalloc_bytes(e, e->snap, e->v2 * e->n_obj);
        if (s) return s;
    }
    CK(cudaMemcpyAsync(e->snap, e->pos, e->v2 * e->n_obj, cudaMemcpyDeviceToDevice, e->st));
    CK(cudaStreamSynchronize(e->st));
    e->has_snap = true;
    return EP_OK;
}

ep_status ep_load_positions(ep_engine *e) {
    if (!e) return EP_ERR_ARG;
    if (!e->has_snap) {
        e->err = "ep_save_positions must run first";
        return EP_ERR_STATE;
    }
    CK(cudaMemcpyAsync(e->pos, e->snap, e->v2 * e->n_obj, cudaMemcpyDeviceToDevice, e->st));
    return EP_OK;
}

}  // extern "C"

namespace {
// Header of an optimizer-state blob; the five vectors and the scalars follow.
struct StateHeader {
    char magic[8];
    int32_t abi, precision, n_obj, n_nodes, n_terms, n_nets, n_pins, nx, ny, stage, in_run, initialized;
    uint32_t scalar_bytes, vec_bytes;
};
constexpr char kStateMagic[8] = {'E', 'P', 'S', 'T', 'A', 'T', 'E', '1'};
constexpr int kStateVecs = 5;  // pos, x, g, y_prev, g_prev

StateHeader state_header(const ep_engine *e) {
    StateHeader h{};
    std::memcpy(h.magic, kStateMagic, sizeof(h.magic));
    h.abi = EP_ABI_VERSION;
    h.precision = e->fp64 ? EP_PREC_FP64 : EP_PREC_MIXED;
    h.n_obj = e->n_obj;
    h.n_nodes = e->n_nodes;
    h.n_terms = e->n_terms;
    h.n_nets = e->n_nets;
    h.n_pins = e->n_pins;
    h.nx = e->grid.nx;
    h.ny = e->grid.ny;
    h.stage = e->stage;
    h.in_run = e->in_run ? 1 : 0;
    h.initialized = e->initialized ? 1 : 0;
    h.scalar_bytes = (uint32_t)sizeof(DevScalars);
    h.vec_bytes = (uint32_t)(e->v2 * e->n_obj);
    return h;
}
}  // namespace

extern "C" {

uint64_t ep_state_size(const ep_engine *e) {
    if (!e) return 0;
    return sizeof(StateHeader) + sizeof(DevScalars) + (uint64_t)kStateVecs * e->v2 * e->n_obj;
}

ep_status ep_save_state(ep_engine *e, void *buf, uint64_t bytes) {
    if (!e || !buf || bytes != ep_state_size(e)) return EP_ERR_ARG;
    ep_status s = fetch_scalars(e);  // synchronises the stream
    if (s) return s;
    const StateHeader h = state_header(e);
    unsigned char *p = static_cast<unsigned char *>(buf);
    std::memcpy(p, &h, sizeof(h));
    std::memcpy(p + sizeof(h), e->hS, sizeof(DevScalars));
    unsigned char *v = p + sizeof(h) + sizeof(DevScalars);
    const void *src[kStateVecs] = {e->pos, e->x, e->g, e->y_prev, e->g_prev};
    for (int k = 0; k < kStateVecs; k++)
        CK(cudaMemcpyAsync(v + (size_t)k * h.vec_bytes, src[k], h.vec_bytes, cudaMemcpyDeviceToHost, e->st));
    CK(cudaStreamSynchronize(e->st));
    return EP_OK;
}

ep_status ep_load_state(ep_engine *e, const void *buf, uint64_t bytes) {
    if (!e || !buf) return EP_ERR_ARG;
    if (bytes != ep_state_size(e)) {
        e->err = "state blob of another size than this engine's";
        return EP_ERR_ARG;
    }
    const unsigned char *p = static_cast<const unsigned char *>(buf);
    StateHeader h;
    std::memcpy(&h, p, sizeof(h));
    StateHeader mine = state_header(e);
    if (std::memcmp(h.magic, kStateMagic, sizeof(h.magic)) || h.abi != mine.abi || h.precision != mine.precision ||
        h.n_obj != mine.n_obj || h.n_nodes != mine.n_nodes || h.n_terms != mine.n_terms ||
        h.n_nets != mine.n_nets || h.n_pins != mine.n_pins || h.nx != mine.nx || h.ny != mine.ny ||
        h.scalar_bytes != mine.scalar_bytes || h.vec_bytes != mine.vec_bytes) {
        e->err = "state blob of another design, grid, precision or library version";
        return EP_ERR_ARG;
    }
    if (!e->initialized) {
        e->err = "ep_initialize must run before ep_load_state";
        return EP_ERR_STATE;
    }
    if (h.stage != e->stage) {
        e->err = "the state was saved in another stage: switch the engine to it first";
        return EP_ERR_STATE;
    }
    std::memcpy(e->hS, p + sizeof(h), sizeof(DevScalars));
    DevScalars &S = *e->hS;
    S.cnt_prep = S.cnt_wl = S.cnt_comb = S.cnt_upd = S.cnt_hp = 0;  // no reduction in flight
    const unsigned char *v = p + sizeof(h) + sizeof(DevScalars);
    void *dst[kStateVecs] = {e->pos, e->x, e->g, e->y_prev, e->g_prev};
    for (int k = 0; k < kStateVecs; k++)
        CK(cudaMemcpyAsync(dst[k], v + (size_t)k * h.vec_bytes, h.vec_bytes, cudaMemcpyHostToDevice, e->st));
    CK(cudaMemcpyAsync(e->S, e->hS, sizeof(DevScalars), cudaMemcpyHostToDevice, e->st));
    CK(cudaStreamSynchronize(e->st));
    e->in_run = h.in_run != 0;
    return EP_OK;
}

ep_status ep_time_kernels(ep_engine *e, int32_t reps, ep_kernel_times *out) try {
    if (!e || !out || reps <= 0) return EP_ERR_ARG;
    std::memset(out, 0, sizeof(*out));
    const int no = e->n_obj, np = e->n_pins, nb = e->grid.nx * e->grid.ny;
    const DeviceNetlist &d = e->dn;
    // state the timed launches mutate, restored at the end
    std::vector<unsigned char> keep[5];
    void *bufs[5] = {e->pos, e->x, e->g, e->y_prev, e->g_prev};
    for (int k = 0; k < 5; k++) {
        keep[k].resize(e->v2 * no);
        CK(cudaMemcpyAsync(keep[k].data(), bufs[k], e->v2 * no, cudaMemcpyDeviceToHost, e->st));
    }
    ep_status s = fetch_scalars(e);
    if (s) return s;
    DevScalars saved = *e->hS;
    s = update_scalars(e, [](DevScalars &h) {
        h.done = 0;
        h.lambda0_mode = 0;
        h.step_cap = 0;
    });
    if (s) return s;
    const bool keep_maps = e->prm.keep_maps != 0;
    const bool tc = e->dct.mode == EP_DCT_BF16X3;
    void *bf = tc ? dct_tc_rho_planes(e->dct) : nullptr;
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    auto timed = [&](const char *name, int launches, double bytes, double flops, auto &&fn,
                     auto &&before) -> ep_status {
        int k = out->count++;
        std::snprintf(out->names[k], sizeof(out->names[k]), "%s", name);
        // reps back-to-back launches (as in the loop: no host gaps), minus
        // the same number of the per-repetition setup alone
        before();
        fn();
        float ms_all = 0, ms_setup = 0;
        CK(cudaEventRecord(a, e->st));
        for (int r = 0; r < reps; r++) {
            before();
            fn();
        }
        CK(cudaEventRecord(b, e->st));
        CK(cudaEventSynchronize(b));
        cudaEventElapsedTime(&ms_all, a, b);
        CK(cudaEventRecord(a, e->st));
        for (int r = 0; r < reps; r++) before();
        CK(cudaEventRecord(b, e->st));
        CK(cudaEventSynchronize(b));
        cudaEventElapsedTime(&ms_setup, a, b);
        out->ms[k] = std::max(0.0, (double)ms_all - (double)ms_setup) / reps;
        out->bytes[k] = bytes;
        out->flops[k] = flops;
        out->launches[k] = launches;
        return EP_OK;
    };
    auto nothing = [] {};
    auto zero_maps = [&] {
        cudaMemsetAsync(e->node_q, 0, sizeof(unsigned long long) * nb, e->st);
        cudaMemsetAsync(e->filler_q, 0, sizeof(unsigned long long) * nb, e->st);
    };
    const double nobj = no, npin = np, nnet = e->n_nets, nbin = nb;
    const double q = (double)e->v2 / sizeof(float2);  // 2 for the FP64 form's vectors
    const double nx = e->grid.nx, ny = e->grid.ny;
    // algorithmic bytes: compulsory reads + writes of each group, per launch
    s = timed("scatter", 1 + (d.n_big_objs > 0), (9.0 + 8.0 * q) * nobj + 16.0 * nbin, 0.0,
              [&] { launch_scatter(e->kc, d, e->node_q, e->filler_q, e->S, e->st); }, zero_maps);
    if (s) return s;
    s = timed("prep", 1, 24.0 * nbin + 4.0 * q * nbin + (keep_maps ? 0.0 : 16.0 * nbin), 0.0,
              [&] {
                  launch_prep(e->kc, e->node_q, e->filler_q, e->static_map, bf ? nullptr : e->rho, bf,
                              nullptr, nullptr, keep_maps ? 0 : 1, e->S, e->st);
              }, nothing);
    if (s) return s;
    // dense: G1 2nx*ny*ny + G2 2nx*nx*ny + G3 2nx*2ny*ny + G4 2*(2nx*ny*nx) flops;
    // fast transforms: bytes of the three passes (rho 4 -> T 4; T 4 -> X1, X2
    // 8; X1, X2 8 -> field 8)
    const bool fft = e->dct.mode == EP_DCT_FFT;
    double dct_flops = fft ? 0.0 : 2 * nx * ny * ny + 2 * nx * nx * ny + 4 * nx * ny * ny + 4 * nx * ny * nx;
    s = timed("poisson_dct", dct_launches(e->dct), (fft ? 36.0 * q : 16.0) * nbin, dct_flops,
              [&] { dct_run(e->dct, e->rho, e->field, nullptr, e->S, e->st); }, nothing);
    if (s) return s;
    s = timed("wirelength", d.n_net_tasks > 0, (16.0 + 16.0 * q) * npin + 16.0 * d.n_net_tasks, 0.0,
              [&] { launch_wirelength(e->kc, d, e->pin_grad, e->S, e->st); }, nothing);
    if (s) return s;
    if (d.n_big_objs > 0) {
        s = timed("gather_big", 1, 0.0, 0.0,
                  [&] { launch_gather_big(e->kc, d, e->field, e->gd_big, e->S, e->st); }, nothing);
        if (s) return s;
    }
    s = timed("combine", 1, (29.0 + 56.0 * q) * nobj + 8.0 * q * npin, 0.0,
              [&] {
                  launch_combine(e->kc, d, e->field, e->gd_big, e->pin_grad, e->g, e->g_prev,
                                 e->y_prev, nullptr, nullptr, 1, e->S, e->st);
              }, nothing);
    if (s) return s;
    s = timed("update", 1, (9.0 + 56.0 * q) * nobj, 0.0,
              [&] { launch_update(e->kc, d, e->pos, e->x, e->g, e->y_prev, e->g_prev, e->S, e->st); },
              [&] {
                  // a pending stop would make the following repetitions no-ops
                  cudaMemsetAsync(&e->S->stop_pending, 0, sizeof(int), e->st);
              });
    if (s) return s;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    for (int k = 0; k < 5; k++)
        CK(cudaMemcpyAsync(bufs[k], keep[k].data(), e->v2 * no, cudaMemcpyHostToDevice, e->st));
    *e->hS = saved;
    CK(cudaMemcpyAsync(e->S, e->hS, sizeof(DevScalars), cudaMemcpyHostToDevice, e->st));
    if (!keep_maps) zero_maps();
    CK(cudaStreamSynchronize(e->st));
    return EP_OK;
} catch (const std::bad_alloc &) {
    return host_oom(e);
}

}  // extern "C"

// ---- quadratic placement ---------------------------------------------------------
namespace {

ep_status qp_setup(ep_engine *e) {
    if (e->qp_ready) return EP_OK;
    QpDev &q = e->qp;
    const int nn = e->n_nodes, nnet = e->n_nets, np = e->n_pins;
    q.nn = nn;
    q.nnet = nnet;
    q.obj_pin_start = e->obj_pin_start;
    q.obj_pin_dev = e->obj_pin_dev;
    q.owner = e->pin_owner;
    q.off = e->pin_off;

    // at most 4 entries per pin and axis: every counted pair of a net involves
    // one of its two bound pins (< 2 d pairs, two entries each)
    const size_t cap = 4 * (size_t)np + 16;
    const int pb = qp_partial_blocks(nn, nnet);
    ep_status s;
    if ((s = dalloc(e, q.bound, std::max(nnet, 1))) || (s = dalloc(e, q.abspin, std::max(np, 1))) ||
        (s = dalloc(e, q.count, 2 * (size_t)nn)) || (s = dalloc(e, q.row_x, (size_t)nn + 1)) ||
        (s = dalloc(e, q.row_y, (size_t)nn + 1)) || (s = dalloc(e, q.col_x, cap)) || (s = dalloc(e, q.col_y, cap)) ||
        (s = dalloc(e, q.val_x, cap)) || (s = dalloc(e, q.val_y, cap)) || (s = dalloc(e, q.diag, nn)) ||
        (s = dalloc(e, q.rhs, nn)) || (s = dalloc(e, q.x, nn)) || (s = dalloc(e, q.r, nn)) ||
        (s = dalloc(e, q.r0, nn)) || (s = dalloc(e, q.p, nn)) || (s = dalloc(e, q.v, nn)) ||
        (s = dalloc(e, q.s, nn)) || (s = dalloc(e, q.t, nn)) || (s = dalloc(e, q.partials, 4 * (size_t)pb)) ||
        (s = dalloc(e, q.cnt, 1)) || (s = dalloc(e, q.out, 4)) || (s = dalloc(e, q.solve, 1)) ||
        (s = dalloc(e, q.scan, (size_t)qp_scan_blocks(nn) + 2)) || (s = dalloc(e, q.y, nn)) ||
        (s = dalloc(e, q.z, nn)) || (s = dalloc(e, q.dinv, nn)))
        return s;
    q.pin_net = e->pin_net;
    q.net_first = e->net_first;
    q.net_deg = e->net_deg;
    q.net_order = e->net_dev_order;
    q.n_big = e->n_big_nets;
    CK(cudaMemset(q.cnt, 0, sizeof(unsigned)));
    CK(cudaMallocHost((void **)&e->qp_out_h, 4 * sizeof(double)));
    CK(cudaMallocHost((void **)&e->qp_state_h, sizeof(QpSolve)));
    e->qp_cap_x = e->qp_cap_y = cap;
    q.cap_x = q.cap_y = (int)std::min<size_t>(cap, (size_t)INT32_MAX);
    e->qp_ready = true;
    return EP_OK;
}

ep_status qp_read(ep_engine *e, int n) {
    CK(cudaMemcpyAsync(e->qp_out_h, e->qp.out, n * sizeof(double), cudaMemcpyDeviceToHost, e->st));
    CK(cudaStreamSynchronize(e->st));
    CK(cudaGetLastError());
    return EP_OK;
}

// Build both systems at the centres of the last bounds pass (its bound pins
// and pin positions): count, prefix sum, fill.
ep_status qp_build(ep_engine *e) {
    // counts, the CSR offsets by a scan on the device, then the entries: no
    // host round trip (an allocation overflow is flagged in the solver state
    // and reported by qp_solve)
    QpDev &q = e->qp;
    qp_rows(q, 0, e->st);
    qp_offsets(q, e->st);
    qp_rows(q, 1, e->st);
    e->qp_launches += 5;
    CK(cudaGetLastError());
    return EP_OK;
}

// BiCGSTAB as Eigen implements it (van der Vorst's method with a restart
// when r0.r vanishes; identity preconditioner), both axes at once, on the
// device (qp.cu): stop when |r|^2 <= (eps |b|)^2 with eps the float epsilon,
// or after max_it iterations; the current centres are the initial guess.
// The host enqueues iterations in chunks and reads the solver state once per
// chunk.  err[c] = |r|/|b| at the end, the value QPPlacer reads as
// solver.error().
ep_status qp_solve(ep_engine *e, const float2 *qpos, int max_it, bool jacobi, double err[2], int &iters) {
    QpDev &q = e->qp;
    cudaStream_t st = e->st;
    constexpr int kChunk = 10;
    qp_to_x(q, qpos, st);
    if (jacobi) qp_dinv(q, st);
    qp_init(q, max_it, st);
    e->qp_launches += 3 + (jacobi ? 1 : 0);
    QpSolve h{};
    for (int done = 0; done < max_it;) {
        const int n = std::min(kChunk, max_it - done);
        qp_iterations(q, n, jacobi, st);
        e->qp_launches += 6LL * n;
        done += n;
        CK(cudaMemcpyAsync(e->qp_state_h, q.solve, sizeof(QpSolve), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        h = *e->qp_state_h;
        if (h.overflow) {
            e->err = "quadratic placement: more matrix entries than the bound allows";
            return EP_ERR_STATE;
        }
        if (!h.active[0] && !h.active[1]) break;
    }
    CK(cudaGetLastError());
    iters = h.iters;
    for (int c = 0; c < 2; c++) err[c] = h.bb[c] > 0.0 ? std::sqrt(h.rr[c] / h.bb[c]) : 0.0;
    return EP_OK;
}

}  // namespace

extern "C" {

// ep_quadratic_placement's body (its set-up builds host arrays).
// from_centre: the reference's flow (every node to the core centre first,
// rounds until converged or max_iterations + 1); otherwise exactly
// max_iterations rounds from the current centres.  solver_its: BiCGSTAB
// iterations per round (the reference's 100).
static ep_status quadratic_placement(ep_engine *e, int32_t max_iterations, bool from_centre, int solver_its,
                                     bool jacobi, ep_qp_stats *stats) {
    if (e->in_run) {
        e->err = "ep_quadratic_placement cannot run inside an optimizer run";
        return EP_ERR_STATE;
    }
    ep_status s = qp_setup(e);
    if (s) return s;
    QpDev &q = e->qp;
    cudaStream_t st = e->st;
    // the quadratic placement works on FP32 centres; an FP64 engine's centres
    // (terminals included) are rounded into qp_pos and the result copied back
    const int ncent = e->n_obj + e->n_terms;
    if (e->fp64 && !e->qp_pos && (s = dalloc(e, e->qp_pos, ncent))) return s;
    float2 *qpos = e->fp64 ? e->qp_pos : (float2 *)e->pos;
    if (e->fp64) k_convert2<double, float><<<(ncent + 255) / 256, 256, 0, st>>>((const double2 *)e->pos, qpos, ncent);
    const int max_outer = max_iterations > 0 ? max_iterations : 20;  // IPiteCount, default 20
    const double target_error = 0.000001;                           // qplace.cpp:47
    CK(cudaEventRecord(e->ev0, st));
    e->qp_launches = (e->fp64 ? 2 : 0) + (from_centre ? 1 : 0) + 1;
    if (from_centre) qp_center(q, e->grid, e->size, qpos, st);  // moveNodesCenterToCenter
    qp_bounds(q, qpos, q.out, st);
    if ((s = qp_read(e, 1))) return s;
    double hpwl = e->qp_out_h[0], err[2] = {0, 0};
    int outer = 0, solver_iters = 0;
    for (int i = 0;; i++) {
        if ((s = qp_build(e))) return s;
        int it = 0;
        if ((s = qp_solve(e, qpos, solver_its, jacobi, err, it))) return s;  // solver.setMaxIterations(100)
        solver_iters += it;
        qp_from_x(q, e->grid, e->size, qpos, st);  // updateModuleLocation
        qp_bounds(q, qpos, q.out, st);             // calcNetBoundPins
        e->qp_launches += 2;
        if ((s = qp_read(e, 1))) return s;
        hpwl = e->qp_out_h[0];
        outer = i + 1;
        if (!from_centre) {
            if (outer >= max_iterations) break;
            continue;
        }
        if (std::fabs(err[0]) < target_error && std::fabs(err[1]) < target_error && i > 4) break;
        if (i >= max_outer) break;
    }
    if (e->fp64) k_convert2<float, double><<<(ncent + 255) / 256, 256, 0, st>>>(qpos, (double2 *)e->pos, ncent);
    CK(cudaEventRecord(e->ev1, st));
    CK(cudaEventSynchronize(e->ev1));
    e->initialized = false;  // the gradient state belongs to the old positions
    if (stats) {
        float ms = 0;
        cudaEventElapsedTime(&ms, e->ev0, e->ev1);
        stats->rounds = outer;
        stats->solver_iterations = solver_iters;
        stats->hpwl = hpwl;
        stats->error_x = err[0];
        stats->error_y = err[1];
        stats->seconds = ms * 1e-3;
        stats->kernel_launches = e->qp_launches;
    }
    return EP_OK;
}

ep_status ep_quadratic_placement(ep_engine *e, int32_t max_iterations, ep_qp_stats *stats) {
    if (!e) return EP_ERR_ARG;
    try {
        return quadratic_placement(e, max_iterations, true, 100, false, stats);
    } catch (const std::bad_alloc &) {
        return host_oom(e);
    }
}

ep_status ep_quadratic_refine(ep_engine *e, int32_t rounds, int32_t solver_iterations, int32_t preconditioner,
                              ep_qp_stats *stats) {
    if (!e || rounds < 1 || solver_iterations < 0 || preconditioner < 0 || preconditioner > 1) return EP_ERR_ARG;
    try {
        return quadratic_placement(e, rounds, false, solver_iterations > 0 ? solver_iterations : 100,
                                   preconditioner == 1, stats);
    } catch (const std::bad_alloc &) {
        return host_oom(e);
    }
}

}  // extern "C"

// ---- views of an engine for other translation units (gnn.cu) ----------------
namespace ep {

int engine_graph(ep_engine *e, EngineGraph *g) {
    if (!e || !g) return EP_ERR_ARG;
    g->uid = e->uid;
    g->nn = e->n_nodes;
    g->n_obj = e->n_obj;
    g->nt = e->n_terms;
    g->nnet = e->n_nets;
    g->np = e->n_pins;
    g->pin_owner = e->h_pin_owner.data();
    g->net_first = e->h_net_first.data();
    g->net_deg = e->h_net_deg.data();
    g->pin_net = e->h_pin_net.data();
    g->d_pin_owner = e->pin_owner;
    g->d_net_first = e->net_first;
    g->d_net_deg = e->net_deg;
    g->d_pin_net = e->pin_net;
    g->d_net_dev_order = e->net_dev_order;
    g->n_big_nets = e->n_big_nets;
    g->d_obj_pin_start = e->obj_pin_start;
    g->d_obj_pin_dev = e->obj_pin_dev;
    g->d_area = e->area;
    g->d_npins = e->npins;
    g->d_pos = e->pos;
    g->fp64 = e->fp64;
    g->node_area = e->h_node_area.data();
    g->node_pins = e->h_node_pins.data();
    g->term_centre = e->h_term_centre.data();
    g->grid = e->grid;
    g->st = e->st;
    g->device = e->device;
    g->d_status = &e->S->status;
    return EP_OK;
}

// The movable nodes at these device-resident float2 centres (nn of them),
// clamped into the core and stored in the engine's working precision.
int engine_set_node_centres(ep_engine *e, const float2 *xy) {
    const int n = e->n_nodes;
    if (n == 0) return EP_OK;
    if (e->fp64)
        k_scatter_view<double><<<(n + 255) / 256, 256, 0, e->st>>>(e->grid, e->view_idx[EP_STAGE_MGP], n, xy, e->size,
                                                                   (double2 *)e->pos);
    else
        k_scatter_view<float><<<(n + 255) / 256, 256, 0, e->st>>>(e->grid, e->view_idx[EP_STAGE_MGP], n, xy, e->size,
                                                                  (float2 *)e->pos);
    e->initialized = false;
    return cudaGetLastError() == cudaSuccess ? EP_OK : EP_ERR_CUDA;
}

void engine_set_error(ep_engine *e, const char *msg) {
    if (e) e->err.assign(msg);
}

}  // namespace ep
