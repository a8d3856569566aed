/* eplace_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 * Plain-C restatement of the ePlace hot path; see eplace_oracle.h.
 * Built with -ffp-contract=off so float expressions round like the
 * reference's (x86-64 SSE, no fused multiply-add). */
#include "eplace_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_EPS 1.0e-15          /* global.h:39 */
#define OR_PI 3.14159265358979323846
#define OR_NEG_MAX_EXP (-300.0) /* global.h:46 */

/* float_less / float_greater of PlaceCommon/global.h:345-353. */
static int f_less(float a, float b) { return (double)(a - b) < -1.0 * OR_EPS; }
static int f_greater(float a, float b) { return (double)(a - b) > 1.0 * OR_EPS; }
static int f_equal(float a, float b) { return fabs((double)(a - b)) < OR_EPS; }

/* getOverlap / getOverlapArea, PlaceCommon/global.h:477-518 (FP64; the
 * reference returns the negated length and multiplies two of them). */
static double overlap_len(double a0, double a1, double b0, double b1)
{
    double s = a0 > b0 ? a0 : b0;
    double e = a1 < b1 ? a1 : b1;
    return s >= e ? 0.0 : (s - e);
}

static double overlap_area(double l1, double b1, double r1, double t1, double l2, double b2,
                           double r2, double t2)
{
    double h = overlap_len(l1, r1, l2, r2);
    if (h == 0)
        return 0;
    double v = overlap_len(b1, t1, b2, t2);
    if (v == 0)
        return 0;
    return h * v;
}

/* fastExp, PlaceCommon/global.h:457-471, evaluated in FP64. */
static double fast_exp(double a)
{
    a = 1.0 + a / 1024.0;
    for (int i = 0; i < 10; i++)
        a *= a;
    return a;
}

static double wl_exp(double a, int exp_mode) { return exp_mode ? exp(a) : fast_exp(a); }

/* Object rectangle with local smoothing (EPlace/eplace.cpp:1052-1072):
 * the lower-left corner is centre - 0.5f*w in float (Module::setCenter_2D,
 * PlaceCommon/objects.cpp:530-539); a side shorter than the bin is widened to
 * one bin around the centre (double arithmetic stored to float) and its
 * contribution scaled by side/binStep. */
static void obj_rect(const or_grid *g, float cx, float cy, float w, float h, float *llx,
                     float *lly, float *urx, float *ury, float *sx, float *sy)
{
    float cllx = cx - (float)0.5 * w;
    float clly = cy - (float)0.5 * h;
    *llx = cllx;
    *urx = cllx + w;
    *lly = clly;
    *ury = clly + h;
    *sx = 1.0f;
    *sy = 1.0f;
    if (f_less(w, g->step_x))
    {
        *sx = w / g->step_x;
        *llx = (float)((double)cx - 0.5 * (double)g->step_x);
        *urx = (float)((double)cx + 0.5 * (double)g->step_x);
    }
    if (f_less(h, g->step_y))
    {
        *sy = h / g->step_y;
        *lly = (float)((double)cy - 0.5 * (double)g->step_y);
        *ury = (float)((double)cy + 0.5 * (double)g->step_y);
    }
}

/* Bin index range (EPlace/eplace.cpp:1079-1104): INT_DOWN truncation of the
 * float quotient, end clamped to dim-1.  The start is clamped at 0 here; the
 * reference asserts it (the core clamp keeps it there). */
static void bin_range(const or_grid *g, float llx, float lly, float urx, float ury, int *i0,
                      int *i1, int *j0, int *j1)
{
    *i0 = (int)((llx - g->core_llx) / g->step_x);
    *i1 = (int)((urx - g->core_llx) / g->step_x);
    *j0 = (int)((lly - g->core_lly) / g->step_y);
    *j1 = (int)((ury - g->core_lly) / g->step_y);
    if (*i0 < 0) *i0 = 0;
    if (*j0 < 0) *j0 = 0;
    if (*i1 >= g->nx) *i1 = g->nx - 1;
    if (*j1 >= g->ny) *j1 = g->ny - 1;
}

/* Bin corners as binInitialization stores them (EPlace/eplace.cpp:292-313). */
static void bin_box(const or_grid *g, int i, int j, float *llx, float *lly, float *urx, float *ury)
{
    *llx = (float)i * g->step_x + g->core_llx;
    *lly = (float)j * g->step_y + g->core_lly;
    *urx = *llx + g->step_x;
    *ury = *lly + g->step_y;
}

int or_bin_dimension(double std_area, double macro_area, int num_nodes, float core_w,
                     float core_h, float target_density)
{
    float node_area = (float)(std_area + macro_area);
    float core_area = core_w * core_h;
    float avg = (float)(1.0 * node_area / num_nodes);
    float ideal_area = avg / target_density;
    int ideal_count = (int)(1.0 * (core_area / ideal_area) + 0.5f);
    for (int i = 1; i < 10; i++)
    {
        long a = (long)(2 << i) * (2 << i);
        long b = (long)(2 << (i + 1)) * (2 << (i + 1));
        if (a <= ideal_count && b > ideal_count)
            return 2 << i;
    }
    return 1024;
}

static int cmp_float(const void *a, const void *b)
{
    float x = *(const float *)a, y = *(const float *)b;
    return (x > y) - (x < y);
}

int or_filler_sizing(int num_nodes, const float *node_w, const float *node_h,
                     const uint8_t *node_is_macro, int num_terms, const float *term_llx,
                     const float *term_lly, const float *term_w, const float *term_h,
                     const uint8_t *term_is_ni, int num_rows, const float *row_llx,
                     const float *row_lly, const float *row_urx, const float *row_h,
                     float total_row_area, float target_density, float common_row_height,
                     float *filler_w, float *filler_h, float *std_area, float *macro_area)
{
    /* whitespace (EPlace/eplace.cpp:69-92): float accumulation, reference order */
    float overlap = 0;
    for (int t = 0; t < num_terms; t++)
    {
        if (term_is_ni && term_is_ni[t])
            continue;
        for (int r = 0; r < num_rows; r++)
            overlap += (float)overlap_area(term_llx[t], term_lly[t], term_llx[t] + term_w[t],
                                           term_lly[t] + term_h[t], row_llx[r], row_lly[r],
                                           row_urx[r], row_lly[r] + row_h[r]);
    }
    float whitespace = total_row_area - overlap;
    float sa = 0, ma = 0;
    float *areas = (float *)malloc(sizeof(float) * (num_nodes > 0 ? num_nodes : 1));
    for (int i = 0; i < num_nodes; i++)
    {
        float a = node_w[i] * node_h[i];
        areas[i] = a;
        if (node_is_macro[i])
            ma += a;
        else
            sa += a;
    }
    *std_area = sa;
    *macro_area = ma;
    float node_scaled = sa + ma * target_density;
    float total_filler = whitespace * target_density - node_scaled;
    qsort(areas, num_nodes, sizeof(float), cmp_float);
    int lo = (int)(0.05 * (float)num_nodes);
    int hi = (int)(0.95 * (float)num_nodes);
    float acc = 0;
    for (int i = lo; i < hi; i++)
        acc += areas[i];
    free(areas);
    float avg = acc / ((float)(hi - lo));
    *filler_h = common_row_height;
    *filler_w = avg / *filler_h;
    return (int)(total_filler / avg + 0.5);
}

void or_terminal_base_density(const or_grid *g, int num_terms, const float *term_llx,
                              const float *term_lly, const float *term_w, const float *term_h,
                              int num_rows, const float *row_llx, const float *row_lly,
                              const float *row_urx, const float *row_h, float *terminal,
                              float *base)
{
    int nx = g->nx, ny = g->ny;
    memset(terminal, 0, sizeof(float) * (size_t)nx * ny);
    /* terminal density, EPlace/eplace.cpp:327-374 */
    for (int t = 0; t < num_terms; t++)
    {
        float llx = term_llx[t], lly = term_lly[t];
        float urx = llx + term_w[t], ury = lly + term_h[t];
        if (llx < g->core_llx || llx + term_w[t] > g->core_urx)
            continue;
        if (lly < g->core_lly || lly + term_h[t] > g->core_ury)
            continue;
        int i0, i1, j0, j1;
        bin_range(g, llx, lly, urx, ury, &i0, &i1, &j0, &j1);
        for (int i = i0; i <= i1; i++)
            for (int j = j0; j <= j1; j++)
            {
                float bl, bb, br, bt;
                bin_box(g, i, j, &bl, &bb, &br, &bt);
                terminal[(size_t)i * ny + j] +=
                    (float)(g->target_density * overlap_area(bl, bb, br, bt, llx, lly, urx, ury));
            }
    }
    /* base density, EPlace/eplace.cpp:385-409 */
    float bin_area = g->step_x * g->step_y;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
        {
            float bl, bb, br, bt;
            bin_box(g, i, j, &bl, &bb, &br, &bt);
            float avail = 0;
            for (int r = 0; r < num_rows; r++)
                avail += (float)overlap_area(bl, bb, br, bt, row_llx[r], row_lly[r], row_urx[r],
                                             row_lly[r] + row_h[r]);
            base[(size_t)i * ny + j] =
                f_equal(bin_area, avail) ? 0.0f : g->target_density * (bin_area - avail);
        }
}

void or_scatter(const or_grid *g, int n, const float *cx, const float *cy, const float *w,
                const float *h, const uint8_t *flags, double qscale, double *node_fp64,
                double *filler_fp64, int64_t *node_q, int64_t *filler_q)
{
    size_t nb = (size_t)g->nx * g->ny;
    if (node_fp64) memset(node_fp64, 0, nb * sizeof(double));
    if (filler_fp64) memset(filler_fp64, 0, nb * sizeof(double));
    if (node_q) memset(node_q, 0, nb * sizeof(int64_t));
    if (filler_q) memset(filler_q, 0, nb * sizeof(int64_t));
    for (int o = 0; o < n; o++)
    {
        float llx, lly, urx, ury, sx, sy;
        obj_rect(g, cx[o], cy[o], w[o], h[o], &llx, &lly, &urx, &ury, &sx, &sy);
        int i0, i1, j0, j1;
        bin_range(g, llx, lly, urx, ury, &i0, &i1, &j0, &j1);
        int is_filler = (flags[o] & OR_FILLER) != 0;
        int is_macro = (flags[o] & OR_MACRO) != 0;
        for (int i = i0; i <= i1; i++)
            for (int j = j0; j <= j1; j++)
            {
                float bl, bb, br, bt;
                bin_box(g, i, j, &bl, &bb, &br, &bt);
                float ovl = (float)overlap_area(bl, bb, br, bt, llx, lly, urx, ury);
                float c = is_macro ? sx * sy * g->target_density * ovl : sx * sy * ovl;
                size_t k = (size_t)i * g->ny + j;
                if (is_filler)
                {
                    if (filler_fp64) filler_fp64[k] += c;
                    if (filler_q) filler_q[k] += llrint((double)c * qscale);
                }
                else
                {
                    if (node_fp64) node_fp64[k] += c;
                    if (node_q) node_q[k] += llrint((double)c * qscale);
                }
            }
    }
}

/* One axis of the separable transforms, in place on an n1 x n2 x-major grid.
 * axis 0 transforms along x, axis 1 along y.  kind: 0 forward DCT-II,
 * 1 inverse cosine sum, 2 inverse sine sum. */
static void transform_axis(double *a, int n1, int n2, int axis, int kind)
{
    int n = axis == 0 ? n1 : n2;
    int m = axis == 0 ? n2 : n1;
    double *tab = (double *)malloc(sizeof(double) * (size_t)n * n);
    double *in = (double *)malloc(sizeof(double) * n);
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
        {
            /* forward: out[k] = sum_j in[j] cos(pi (j+1/2) k / n)
             * inverse: out[j] = sum_k in[k] {cos,sin}(pi k (j+1/2) / n) */
            double ang = OR_PI * (j + 0.5) * k / n;
            tab[(size_t)k * n + j] = kind == 2 ? sin(ang) : cos(ang);
        }
    for (int r = 0; r < m; r++)
    {
        for (int t = 0; t < n; t++)
            in[t] = axis == 0 ? a[(size_t)t * n2 + r] : a[(size_t)r * n2 + t];
        for (int t = 0; t < n; t++)
        {
            double s = 0;
            if (kind == 0)
                for (int j = 0; j < n; j++)
                    s += in[j] * tab[(size_t)t * n + j];
            else
                for (int k = 0; k < n; k++)
                    s += in[k] * tab[(size_t)k * n + t];
            if (axis == 0)
                a[(size_t)t * n2 + r] = s;
            else
                a[(size_t)r * n2 + t] = s;
        }
    }
    free(tab);
    free(in);
}

void or_poisson(int nx, int ny, float step_x, float step_y, const double *rho, double *ex,
                double *ey, double *phi)
{
    size_t nb = (size_t)nx * ny;
    double *a = (double *)malloc(nb * sizeof(double));
    memcpy(a, rho, nb * sizeof(double));
    /* forward 2-D DCT (ddct2d, isgn=-1) then FFT/fft.cpp:200-216 scaling */
    transform_axis(a, nx, ny, 0, 0);
    transform_axis(a, nx, ny, 1, 0);
    for (int i = 0; i < nx; i++)
        a[(size_t)i * ny] *= 0.5;
    for (int j = 0; j < ny; j++)
        a[j] *= 0.5;
    for (size_t k = 0; k < nb; k++)
        a[k] *= 4.0 / nx / ny;
    /* spectral solve, FFT/fft.cpp:129-147,219-266 */
    double *sp = (double *)malloc(nb * sizeof(double));
    double *sx = (double *)malloc(nb * sizeof(double));
    double *sy = (double *)malloc(nb * sizeof(double));
    for (int u = 0; u < nx; u++)
    {
        double wx = OR_PI * u / nx;
        for (int v = 0; v < ny; v++)
        {
            double wy = OR_PI * v / ny * ((double)step_y / (double)step_x);
            size_t k = (size_t)u * ny + v;
            double p = (u == 0 && v == 0) ? 0.0 : a[k] / (wx * wx + wy * wy);
            sp[k] = p;
            sx[k] = p * wx;
            sy[k] = p * wy;
        }
    }
    /* inverse transforms: phi cos/cos, Ex sin/cos, Ey cos/sin (fft.cpp:272-282) */
    if (phi)
    {
        transform_axis(sp, nx, ny, 0, 1);
        transform_axis(sp, nx, ny, 1, 1);
        memcpy(phi, sp, nb * sizeof(double));
    }
    if (ex)
    {
        transform_axis(sx, nx, ny, 0, 2);
        transform_axis(sx, nx, ny, 1, 1);
        memcpy(ex, sx, nb * sizeof(double));
    }
    if (ey)
    {
        transform_axis(sy, nx, ny, 0, 1);
        transform_axis(sy, nx, ny, 1, 2);
        memcpy(ey, sy, nb * sizeof(double));
    }
    free(a);
    free(sp);
    free(sx);
    free(sy);
}

void or_gather(const or_grid *g, int n, const float *cx, const float *cy, const float *w,
               const float *h, const double *ex, const double *ey, double *grad_xy)
{
    for (int o = 0; o < n; o++)
    {
        float llx, lly, urx, ury, sx, sy;
        obj_rect(g, cx[o], cy[o], w[o], h[o], &llx, &lly, &urx, &ury, &sx, &sy);
        int i0, i1, j0, j1;
        bin_range(g, llx, lly, urx, ury, &i0, &i1, &j0, &j1);
        double gx = 0, gy = 0;
        for (int i = i0; i <= i1; i++)
            for (int j = j0; j <= j1; j++)
            {
                float bl, bb, br, bt;
                bin_box(g, i, j, &bl, &bb, &br, &bt);
                double ov = (double)(sx * sy) * overlap_area(bl, bb, br, bt, llx, lly, urx, ury);
                size_t k = (size_t)i * g->ny + j;
                gx += ov * ex[k];
                gy += ov * ey[k];
            }
        grad_xy[2 * o] = gx;
        grad_xy[2 * o + 1] = gy;
    }
}

double or_overflow(const or_grid *g, const double *node, const double *terminal,
                   const double *base, double std_area, double macro_area)
{
    double bin_area = (double)(g->step_x * g->step_y);
    double acc = 0;
    size_t nb = (size_t)g->nx * g->ny;
    for (size_t k = 0; k < nb; k++)
    {
        double d = (node[k] + terminal[k] + base[k]) / bin_area - g->target_density;
        if (d > 0)
            acc += d * bin_area;
    }
    return acc / (std_area + macro_area * g->target_density);
}

void or_inv_gamma(double tau, float step_x, float step_y, double *igx, double *igy)
{
    double bx = 0.125 / step_x, by = 0.125 / step_y;
    double s;
    if (tau > 1.0)
        s = 0.1;
    else if (tau < 0.1)
        s = 10.0;
    else
        s = 1.0 / pow(10.0, (tau - 0.1) * 20 / 9.0 - 1.0);
    *igx = bx * s;
    *igy = by * s;
}

static void pin_pos(int p, const int32_t *pin_owner, const float *pin_dx, const float *pin_dy,
                    int num_objects, const float *cx, const float *cy, const float *term_cx,
                    const float *term_cy, double *x, double *y)
{
    int o = pin_owner[p];
    /* Pin::calculateAbsolutePos: float centre + float offset, rounded to float */
    if (o < num_objects)
    {
        *x = (float)(cx[o] + pin_dx[p]);
        *y = (float)(cy[o] + pin_dy[p]);
    }
    else
    {
        *x = (float)(term_cx[o - num_objects] + pin_dx[p]);
        *y = (float)(term_cy[o - num_objects] + pin_dy[p]);
    }
}

double or_hpwl(int num_nets, const int32_t *net_start, const int32_t *pin_owner,
               const float *pin_dx, const float *pin_dy, int num_objects, const float *cx,
               const float *cy, const float *term_cx, const float *term_cy)
{
    double total = 0;
    for (int n = 0; n < num_nets; n++)
    {
        double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
        for (int p = net_start[n]; p < net_start[n + 1]; p++)
        {
            double x, y;
            pin_pos(p, pin_owner, pin_dx, pin_dy, num_objects, cx, cy, term_cx, term_cy, &x, &y);
            if (x < x0) x0 = x;
            if (x > x1) x1 = x;
            if (y < y0) y0 = y;
            if (y > y1) y1 = y;
        }
        total += (x1 - x0) + (y1 - y0);
    }
    return total;
}

double or_wirelength_grad(int num_nets, const int32_t *net_start, const int32_t *pin_owner,
                          const float *pin_dx, const float *pin_dy, int num_objects,
                          const float *cx, const float *cy, const float *term_cx,
                          const float *term_cy, double igx, double igy, int exp_mode, int lse,
                          double *grad_xy, double *hpwl)
{
    memset(grad_xy, 0, sizeof(double) * 2 * (size_t)num_objects);
    double total = 0, hp = 0;
    int cap = 0;
    double *px = NULL, *py = NULL, *emx = NULL, *enx = NULL, *emy = NULL, *eny = NULL;
    for (int n = 0; n < num_nets; n++)
    {
        int a = net_start[n], b = net_start[n + 1], d = b - a;
        if (d > cap)
        {
            cap = d;
            px = (double *)realloc(px, sizeof(double) * cap);
            py = (double *)realloc(py, sizeof(double) * cap);
            emx = (double *)realloc(emx, sizeof(double) * cap);
            enx = (double *)realloc(enx, sizeof(double) * cap);
            emy = (double *)realloc(emy, sizeof(double) * cap);
            eny = (double *)realloc(eny, sizeof(double) * cap);
        }
        double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
        for (int k = 0; k < d; k++)
        {
            pin_pos(a + k, pin_owner, pin_dx, pin_dy, num_objects, cx, cy, term_cx, term_cy,
                    &px[k], &py[k]);
            if (px[k] < x0) x0 = px[k];
            if (px[k] > x1) x1 = px[k];
            if (py[k] < y0) y0 = py[k];
            if (py[k] > y1) y1 = py[k];
        }
        hp += (x1 - x0) + (y1 - y0);
        double nmx = 0, dmx = 0, nnx = 0, dnx = 0, nmy = 0, dmy = 0, nny = 0, dny = 0;
        for (int k = 0; k < d; k++)
        {
            /* exponent arguments; <= -300 flags the term as zero */
            double amx = (px[k] - x1) * igx, anx = (x0 - px[k]) * igx;
            double amy = (py[k] - y1) * igy, any = (y0 - py[k]) * igy;
            emx[k] = amx > OR_NEG_MAX_EXP ? wl_exp(amx, exp_mode) : 0.0;
            enx[k] = anx > OR_NEG_MAX_EXP ? wl_exp(anx, exp_mode) : 0.0;
            emy[k] = amy > OR_NEG_MAX_EXP ? wl_exp(amy, exp_mode) : 0.0;
            eny[k] = any > OR_NEG_MAX_EXP ? wl_exp(any, exp_mode) : 0.0;
            nmx += px[k] * emx[k];
            dmx += emx[k];
            nnx += px[k] * enx[k];
            dnx += enx[k];
            nmy += py[k] * emy[k];
            dmy += emy[k];
            nny += py[k] * eny[k];
            dny += eny[k];
        }
        if (lse)
            total += (x1 - x0 + log(dmx) / igx + log(dnx) / igx) +
                     (y1 - y0 + log(dmy) / igy + log(dny) / igy);
        else
            total += (nmx / dmx - nnx / dnx) + (nmy / dmy - nny / dny);
        for (int k = 0; k < d; k++)
        {
            int o = pin_owner[a + k];
            if (o >= num_objects)
                continue;
            double gx, gy;
            if (lse)
            {
                gx = emx[k] / dmx - enx[k] / dnx;
                gy = emy[k] / dmy - eny[k] / dny;
            }
            else
            {
                double gmx = 0, gnx = 0, gmy = 0, gny = 0;
                if (emx[k] != 0)
                {
                    double dd = igx * emx[k], nd = emx[k] + px[k] * dd;
                    gmx = (nd * dmx - dd * nmx) / (dmx * dmx);
                }
                if (enx[k] != 0)
                {
                    double dd = igx * enx[k], nd = enx[k] - px[k] * dd;
                    gnx = (nd * dnx + dd * nnx) / (dnx * dnx);
                }
                if (emy[k] != 0)
                {
                    double dd = igy * emy[k], nd = emy[k] + py[k] * dd;
                    gmy = (nd * dmy - dd * nmy) / (dmy * dmy);
                }
                if (eny[k] != 0)
                {
                    double dd = igy * eny[k], nd = eny[k] - py[k] * dd;
                    gny = (nd * dny + dd * nny) / (dny * dny);
                }
                gx = gmx - gnx;
                gy = gmy - gny;
            }
            grad_xy[2 * o] += gx;
            grad_xy[2 * o + 1] += gy;
        }
    }
    free(px); free(py); free(emx); free(enx); free(emy); free(eny);
    if (hpwl)
        *hpwl = hp;
    return total;
}

void or_combine(int n, const int32_t *pins_per_object, const float *area, const uint8_t *flags,
                double lambda, const double *grad_density, const double *grad_wl, double *g)
{
    for (int o = 0; o < n; o++)
    {
        double pre = 1.0 / fmax(1.0, pins_per_object[o] + lambda * area[o]);
        if (flags[o] & OR_FILLER)
        {
            g[2 * o] = pre * lambda * grad_density[2 * o];
            g[2 * o + 1] = pre * lambda * grad_density[2 * o + 1];
        }
        else
        {
            g[2 * o] = pre * (lambda * grad_density[2 * o] - grad_wl[2 * o]);
            g[2 * o + 1] = pre * (lambda * grad_density[2 * o + 1] - grad_wl[2 * o + 1]);
        }
    }
}

double or_lambda0(int num_nodes, int num_objects, const double *grad_wl, const double *grad_density)
{
    double num = 0, den = 0;
    for (int o = 0; o < num_nodes; o++)
        num += fabs(grad_wl[2 * o]) + fabs(grad_wl[2 * o + 1]);
    for (int o = 0; o < num_objects; o++)
        den += fabs(grad_density[2 * o]) + fabs(grad_density[2 * o + 1]);
    return num / den;
}

double or_lambda_multiplier(double cur_hpwl, double last_hpwl)
{
    double delta = cur_hpwl - last_hpwl;
    double m = delta < 0.0 ? 1.05 : pow(1.05, -delta / 350000.0 + 1.0);
    if (m > 1.05) m = 1.05;
    if (m < 0.95) m = 0.95;
    return m;
}

void or_clamp(float *x, float *y, float w, float h, float core_llx, float core_lly,
              float core_urx, float core_ury)
{
    float cx = *x, cy = *y;
    if (cx - 0.5 * w < core_llx) cx = (float)(core_llx + 0.5 * w + OR_EPS);
    if (cx + 0.5 * w > core_urx) cx = (float)(core_urx - 0.5 * w - OR_EPS);
    if (cy - 0.5 * h < core_lly) cy = (float)(core_lly + 0.5 * h + OR_EPS);
    if (cy + 0.5 * h > core_ury) cy = (float)(core_ury - 0.5 * h - OR_EPS);
    *x = cx;
    *y = cy;
}

/* ----------------------------- mGP loop -------------------------------- */
typedef struct eval_buf {
    double *node, *filler, *rho, *ex, *ey, *gd, *gwl, *g, *term, *basem;
} eval_buf;

/* totalGradientUpdate at (cx, cy): returns tau; fills gd, gwl and g. */
static double or_eval(const or_design *d, const float *cx, const float *cy, double lambda,
                      eval_buf *b, double *hpwl)
{
    const or_grid *g = &d->grid;
    int n = d->num_nodes + d->num_fillers;
    size_t nb = (size_t)g->nx * g->ny;
    or_scatter(g, n, cx, cy, d->w, d->h, d->flags, 0.0, b->node, b->filler, NULL, NULL);
    double bin_area = (double)(g->step_x * g->step_y);
    for (size_t k = 0; k < nb; k++)
        b->rho[k] = (b->node[k] + b->basem[k] + b->filler[k] + b->term[k]) / bin_area;
    or_poisson(g->nx, g->ny, g->step_x, g->step_y, b->rho, b->ex, b->ey, NULL);
    or_gather(g, n, cx, cy, d->w, d->h, b->ex, b->ey, b->gd);
    double tau = or_overflow(g, b->node, b->term, b->basem, d->std_area, d->macro_area);
    double igx, igy;
    or_inv_gamma(tau, g->step_x, g->step_y, &igx, &igy);
    or_wirelength_grad(d->num_nets, d->net_start, d->pin_owner, d->pin_dx, d->pin_dy, n, cx, cy,
                       d->term_cx, d->term_cy, igx, igy, d->exp_mode, 0, b->gwl, hpwl);
    float *area = (float *)malloc(sizeof(float) * n);
    for (int o = 0; o < n; o++)
        area[o] = d->w[o] * d->h[o];
    or_combine(n, d->pins_per_object, area, d->flags, lambda, b->gd, b->gwl, b->g);
    free(area);
    return tau;
}

void or_mgp_run(const or_design *d, float *cx, float *cy, or_run_stats *stats)
{
    const or_grid *gr = &d->grid;
    int n = d->num_nodes + d->num_fillers;
    size_t nb = (size_t)gr->nx * gr->ny;
    eval_buf b;
    b.node = calloc(nb, sizeof(double));
    b.filler = calloc(nb, sizeof(double));
    b.rho = calloc(nb, sizeof(double));
    b.ex = calloc(nb, sizeof(double));
    b.ey = calloc(nb, sizeof(double));
    b.term = calloc(nb, sizeof(double));
    b.basem = calloc(nb, sizeof(double));
    for (size_t k = 0; k < nb; k++)
    {
        b.term[k] = d->terminal[k];
        b.basem[k] = d->base[k];
    }
    b.gd = calloc(2 * (size_t)n, sizeof(double));
    b.gwl = calloc(2 * (size_t)n, sizeof(double));
    b.g = calloc(2 * (size_t)n, sizeof(double));
    double *gprev = calloc(2 * (size_t)n, sizeof(double));
    float *x = malloc(sizeof(float) * 2 * n), *yprev = malloc(sizeof(float) * 2 * n);
    float *ycx = malloc(sizeof(float) * n), *ycy = malloc(sizeof(float) * n);

    for (int o = 0; o < n; o++)
        or_clamp(&cx[o], &cy[o], d->w[o], d->h[o], gr->core_llx, gr->core_lly, gr->core_urx,
                 gr->core_ury);
    double hp;
    /* initialization(): gradient with lambda = 0, then lambda_0 */
    double tau = or_eval(d, cx, cy, 0.0, &b, &hp);
    double lambda = or_lambda0(d->num_nodes, n, b.gwl, b.gd);
    double last_hpwl = hp;
    for (int o = 0; o < n; o++)
    {
        x[2 * o] = cx[o];
        x[2 * o + 1] = cy[o];
    }
    double a = 1.0;
    int iter = 0;
    while (!(tau < d->target_overflow || iter > d->max_iterations))
    {
        for (int o = 0; o < n; o++)
        {
            ycx[o] = cx[o];
            ycy[o] = cy[o];
        }
        tau = or_eval(d, ycx, ycy, lambda, &b, &hp);
        double step = 1.0;
        if (iter > 0)
        {
            double sg = 0, sy = 0;
            for (int o = 0; o < n; o++)
            {
                double dgx = b.g[2 * o] - gprev[2 * o], dgy = b.g[2 * o + 1] - gprev[2 * o + 1];
                double dyx = (double)ycx[o] - yprev[2 * o], dyy = (double)ycy[o] - yprev[2 * o + 1];
                sg += dgx * dgx + dgy * dgy;
                sy += dyx * dyx + dyy * dyy;
            }
            step = sqrt(sy) / sqrt(sg);
        }
        double a_new = (1.0 + sqrt(4.0 * a * a + 1.0)) / 2.0;
        double coef = (a - 1.0) / a_new;
        for (int o = 0; o < n; o++)
        {
            double nx_ = ycx[o] + b.g[2 * o] * step;
            double ny_ = ycy[o] + b.g[2 * o + 1] * step;
            float yx = (float)(nx_ + (nx_ - x[2 * o]) * coef);
            float yy = (float)(ny_ + (ny_ - x[2 * o + 1]) * coef);
            or_clamp(&yx, &yy, d->w[o], d->h[o], gr->core_llx, gr->core_lly, gr->core_urx,
                     gr->core_ury);
            x[2 * o] = (float)nx_;
            x[2 * o + 1] = (float)ny_;
            cx[o] = yx;
            cy[o] = yy;
            yprev[2 * o] = ycx[o];
            yprev[2 * o + 1] = ycy[o];
            gprev[2 * o] = b.g[2 * o];
            gprev[2 * o + 1] = b.g[2 * o + 1];
        }
        double cur = or_hpwl(d->num_nets, d->net_start, d->pin_owner, d->pin_dx, d->pin_dy, n, cx,
                             cy, d->term_cx, d->term_cy);
        lambda *= or_lambda_multiplier(cur, last_hpwl);
        last_hpwl = cur;
        a = a_new;
        iter++;
    }
    /* wrap_up: the main solution */
    for (int o = 0; o < n; o++)
    {
        cx[o] = x[2 * o];
        cy[o] = x[2 * o + 1];
        or_clamp(&cx[o], &cy[o], d->w[o], d->h[o], gr->core_llx, gr->core_lly, gr->core_urx,
                 gr->core_ury);
    }
    if (stats)
    {
        stats->iterations = iter;
        stats->overflow = tau;
        stats->hpwl = or_hpwl(d->num_nets, d->net_start, d->pin_owner, d->pin_dx, d->pin_dy, n, cx,
                              cy, d->term_cx, d->term_cy);
        stats->lambda = lambda;
    }
    free(b.node); free(b.filler); free(b.rho); free(b.ex); free(b.ey); free(b.term);
    free(b.basem); free(b.gd); free(b.gwl); free(b.g); free(gprev); free(x); free(yprev);
    free(ycx); free(ycy);
}
