/* eplace_oracle.h -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * A plain-C restatement of the ePlace global-placement hot path of
 * Xinyu-lumos/ePlace, used by tests/ to check the CUDA engine and pinned
 * against the reference's own outputs (oracle/_ref, tests/golden/).  Every
 * function names the reference lines it follows.  Arithmetic is FP64 except
 * where a function says it reproduces the reference's float rounding (the
 * rectangle / overlap / contribution chain of the density scatter, which the
 * engine's fixed-point scatter must match bit for bit).
 *
 * Layouts: objects are nodes (movable cells and macros) followed by fillers;
 * positions are centres; bin maps are x-major (index x*ny + y); pins are CSR
 * by net; pin_owner < num_objects is an object, otherwise a fixed terminal
 * whose centre is term_cx/term_cy[pin_owner - num_objects].
 */
#ifndef EPLACE_ORACLE_H
#define EPLACE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_grid {
    int nx, ny;
    float core_llx, core_lly, core_urx, core_ury;
    float step_x, step_y;
    float target_density;
} or_grid;

/* Object flags (bit set). */
#define OR_MACRO 1u
#define OR_FILLER 2u

/* EPlacer_2D::binInitialization bin-count rule, EPlace/eplace.cpp:230-261. */
int or_bin_dimension(double std_area, double macro_area, int num_nodes,
                     float core_w, float core_h, float target_density);

/* fillerInitialization sizing, EPlace/eplace.cpp:61-167.  Returns the filler
 * count; writes filler width/height and the std/macro areas. */
int or_filler_sizing(int num_nodes, const float *node_w, const float *node_h,
                     const uint8_t *node_is_macro, int num_terms,
                     const float *term_llx, const float *term_lly, const float *term_w,
                     const float *term_h, const uint8_t *term_is_ni, int num_rows,
                     const float *row_llx, const float *row_lly, const float *row_urx,
                     const float *row_h, float total_row_area, float target_density,
                     float common_row_height, float *filler_w, float *filler_h,
                     float *std_area, float *macro_area);

/* Static maps of binInitialization, EPlace/eplace.cpp:321-409 (float
 * accumulation in the reference order). */
void or_terminal_base_density(const or_grid *g, int num_terms, const float *term_llx,
                              const float *term_lly, const float *term_w, const float *term_h,
                              int num_rows, const float *row_llx, const float *row_lly,
                              const float *row_urx, const float *row_h,
                              float *terminal, float *base);

/* Density scatter, EPlace/eplace.cpp:1029-1133.
 *  node_fp64/filler_fp64 : FP64 sums of the float contributions (may be NULL)
 *  node_q/filler_q       : int64 fixed-point sums, each contribution rounded
 *                          to nearest-even of contribution * qscale (may be NULL)
 * Contributions are formed with the reference's float arithmetic. */
void or_scatter(const or_grid *g, int n, const float *cx, const float *cy, const float *w,
                const float *h, const uint8_t *flags, double qscale,
                double *node_fp64, double *filler_fp64, int64_t *node_q, int64_t *filler_q);

/* Electrostatic Poisson solve of FFT_2D::doFFT (FFT/fft.cpp:98-148,191-284),
 * restated as the dense DCT-II / DCT-III / DST-III sums, FP64.  rho is the
 * bin density (area / bin area), x-major.  Any output may be NULL. */
void or_poisson(int nx, int ny, float step_x, float step_y, const double *rho,
                double *ex, double *ey, double *phi);

/* Field gather, EPlace/eplace.cpp:599-674, FP64: grad += sx*sy*ovl*E. */
void or_gather(const or_grid *g, int n, const float *cx, const float *cy, const float *w,
               const float *h, const double *ex, const double *ey, double *grad_xy);

/* Overflow tau, EPlace/eplace.cpp:438-453 (FP64). */
double or_overflow(const or_grid *g, const double *node, const double *terminal,
                   const double *base, double std_area, double macro_area);

/* 1/gamma schedule, EPlace/eplace.cpp:475-500. */
void or_inv_gamma(double tau, float step_x, float step_y, double *igx, double *igy);

/* Exact HPWL, PlaceDB::calcHPWL / Net::calcNetHPWL (PlaceDB/placedb.cpp:424-432,
 * PlaceCommon/objects.cpp:35-73), FP64. */
double or_hpwl(int num_nets, const int32_t *net_start, const int32_t *pin_owner,
               const float *pin_dx, const float *pin_dy, int num_objects, const float *cx,
               const float *cy, const float *term_cx, const float *term_cy);

/* Weighted-average wirelength and its gradient summed per object in pin
 * order, Net::calcBoundPin / calcWirelengthWA_2D / getWirelengthGradientWA_2D
 * (PlaceCommon/objects.cpp:75-144,248-415) and EPlace/eplace.cpp:531-549.
 * exp_mode 0 = the reference's fastExp (global.h:457-471), 1 = exact exp.
 * lse != 0 selects the LSE model (objects.cpp:161-241,423-437).
 * grad_xy has 2*num_objects entries (fillers stay 0).  Returns the smooth
 * wirelength; *hpwl receives the bound-pin HPWL. */
double or_wirelength_grad(int num_nets, const int32_t *net_start, const int32_t *pin_owner,
                          const float *pin_dx, const float *pin_dy, int num_objects,
                          const float *cx, const float *cy, const float *term_cx,
                          const float *term_cy, double igx, double igy, int exp_mode, int lse,
                          double *grad_xy, double *hpwl);

/* Preconditioned descent direction, EPlace/eplace.cpp:698-737:
 * p = 1/max(1, pins + lambda*area); cells g = p*(lambda*gD - gWL),
 * fillers g = p*lambda*gD. */
void or_combine(int n, const int32_t *pins_per_object, const float *area, const uint8_t *flags,
                double lambda, const double *grad_density, const double *grad_wl, double *g);

/* lambda_0 = sum|gWL|_1 / sum|gD|_1, EPlace/eplace.cpp:812-835. */
double or_lambda0(int num_nodes, int num_objects, const double *grad_wl, const double *grad_density);

/* updatePenaltyFactor multiplier, EPlace/eplace.cpp:846-883. */
double or_lambda_multiplier(double cur_hpwl, double last_hpwl);

/* setModuleCenter_2D clamp into the core, PlaceDB/placedb.cpp:253-288. */
void or_clamp(float *x, float *y, float w, float h, float core_llx, float core_lly,
              float core_urx, float core_ury);

/* ----- whole mGP loop (EplaceNesterovOpt with the 1/L step) ------------- */
typedef struct or_design {
    or_grid grid;
    int num_nodes, num_fillers, num_terms, num_nets;
    const float *w, *h;          /* [num_nodes + num_fillers] */
    const uint8_t *flags;        /* [num_nodes + num_fillers] */
    const int32_t *pins_per_object;
    const int32_t *net_start, *pin_owner;
    const float *pin_dx, *pin_dy;
    const float *term_cx, *term_cy;
    const float *terminal, *base; /* static maps (float, reference order) */
    double std_area, macro_area;
    float target_overflow;
    int max_iterations;
    int exp_mode;
} or_design;

typedef struct or_run_stats {
    int iterations;
    double overflow, hpwl, lambda;
} or_run_stats;

/* initialization() gradient + lambda_0, then FirstOrderOptimizer::opt for
 * the mGP view (Optimization/nesterov.hpp:86-223,375-415,
 * Optimization/optutils.hpp:20-35) with FP64 reductions.  cx/cy hold the
 * start positions of all objects and receive the final (main-solution)
 * positions. */
void or_mgp_run(const or_design *d, float *cx, float *cy, or_run_stats *stats);

#ifdef __cplusplus
}
#endif
#endif
