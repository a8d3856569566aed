// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// A thin extern "C" driver around the UNMODIFIED reference sources of
// Xinyu-lumos/ePlace, compiled where they lie by oracle/Makefile into
// oracle/_ref/libeplace_ref.so.  Only tests/, __graft_entry__.smoke() and the
// CPU-baseline legs of bench.py load it.  It lets the tests
//   * build a reference PlaceDB from a Bookshelf design (Parser/parser.cpp:44)
//     or from plain arrays through PlaceDB's own add* API
//     (PlaceDB/placedb.cpp:96-153), exactly as the parser would;
//   * run EPlacer_2D::initialization (EPlace/eplace.cpp:39-50),
//     totalGradientUpdate (EPlace/eplace.cpp:687-738), updatePenaltyFactor
//     (EPlace/eplace.cpp:846-883), the stage switches (:887-904) and the
//     EplaceNesterovOpt loop (Optimization/nesterov.hpp:86-415) step by step;
//   * read back every intermediate the hot path produces (bin maps, field,
//     potential, density / wirelength / total gradients, tau, 1/gamma, lambda,
//     HPWL) at full float precision, bypassing the %.0f .pl writer;
//   * run the reference's CPU stages around global placement on whatever
//     positions were set: SAMacroLegalizer (mLG), AbacusLegalizer and
//     DetailedPlacer (main/ePlace_main.cpp:174-279).
// Nothing here re-implements reference arithmetic: every number comes from
// the reference's own functions.

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <unistd.h>
#include <fcntl.h>
#include <sys/time.h>

#include "global.h"
#include "objects.h"
#include "placedb.h"
#include "eplace.h"
#include "plot.h"
#include "optutils.hpp"
#include "opt.hpp"
#include "parser.h"
#include "qplace.h"
#include "legalizer.h"
#include "detailed.h"
#include "Eigen/Dense"

// The optimizer keeps its per-step methods private; the harness needs to call
// opt_step()/stop_condition() one at a time to time a bounded number of
// iterations.  Its dependencies are all included above, so only the
// EplaceNesterovOpt declaration sees the access change.
#define private public
#include "nesterov.hpp"
#undef private

namespace {

struct RefHandle
{
    PlaceDB *db = nullptr;
    EPlacer_2D *placer = nullptr;
    EplaceNesterovOpt<VECTOR_3D> *opt = nullptr;
    bool initialized = false;
};

int g_quiet = 1;

// Silence the reference's cout/printf chatter (it logs every iteration).
struct Quiet
{
    int saved_out = -1, saved_err = -1;
    Quiet()
    {
        if (!g_quiet)
            return;
        fflush(stdout);
        fflush(stderr);
        std::cout.flush();
        int devnull = open("/dev/null", O_WRONLY);
        if (devnull < 0)
            return;
        saved_out = dup(1);
        saved_err = dup(2);
        dup2(devnull, 1);
        dup2(devnull, 2);
        close(devnull);
    }
    ~Quiet()
    {
        if (saved_out < 0)
            return;
        fflush(stdout);
        fflush(stderr);
        std::cout.flush();
        dup2(saved_out, 1);
        dup2(saved_err, 2);
        close(saved_out);
        close(saved_err);
    }
};

double now_s()
{
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

} // namespace

extern "C" {

void ref_set_quiet(int quiet) { g_quiet = quiet; }

// gArg switches read on the hot path: "LSE", "bb", "bktrk", "targetOverflow".
void ref_set_flag(const char *name, const char *value) { gArg.Override(name, value ? value : "1"); }
void ref_clear_flag(const char *name) { gArg.RemoveOverride(name); }

void *ref_create_bookshelf(const char *aux_path)
{
    Quiet q;
    RefHandle *h = new RefHandle();
    h->db = new PlaceDB();
    std::string file(aux_path);
    std::string::size_type pos = file.rfind('/');
    gArg.Override("path", pos == std::string::npos ? std::string("./") : file.substr(0, pos + 1));
    BookshelfParser parser;
    parser.ReadFile(file, *h->db);
    return h;
}

// Build the PlaceDB through the same add* calls Parser/parser.cpp makes.
// Nodes are movable (macro iff height > row height, PlaceDB/placedb.cpp:96-114);
// terminals are fixed.  Pins are given net by net (CSR), offsets from the
// owner's centre (Pin::calculateAbsolutePos, PlaceCommon/objects.cpp:454-459).
// pin_owner < num_nodes names a node, otherwise terminal (pin_owner - num_nodes).
void *ref_create_arrays(int num_nodes, int num_terminals, int num_nets, int num_rows,
                        const float *node_w, const float *node_h,
                        const float *node_cx, const float *node_cy,
                        const float *term_llx, const float *term_lly,
                        const float *term_w, const float *term_h, const unsigned char *term_is_ni,
                        const int *net_start, const int *pin_owner,
                        const float *pin_dx, const float *pin_dy,
                        const float *row_llx, const float *row_lly, const float *row_urx,
                        const float *row_h, const float *row_site_w)
{
    Quiet q;
    RefHandle *h = new RefHandle();
    PlaceDB &db = *(h->db = new PlaceDB());
    for (int r = 0; r < num_rows; r++)
    {
        SiteRow row(row_lly[r], row_h[r], row_site_w[r]);
        row.start = POS_2D(row_llx[r], row_lly[r]);
        row.end = POS_2D(row_urx[r], row_lly[r]);
        row.intervals.push_back(Interval(row_llx[r], row_urx[r]));
        db.dbSiteRows.push_back(row);
    }
    db.commonRowHeight = db.dbSiteRows.back().height;
    db.setCoreRegion();

    db.allocateNodeMemory(num_nodes);
    db.allocateTerminalMemory(num_terminals);
    std::vector<Module *> owners(num_nodes + num_terminals);
    for (int i = 0; i < num_nodes; i++)
    {
        std::string name = "o" + std::to_string(i);
        owners[i] = db.addNode(i, name, node_w[i], node_h[i]);
        db.moduleMap[name] = owners[i];
    }
    for (int i = 0; i < num_terminals; i++)
    {
        std::string name = "t" + std::to_string(i);
        bool ni = term_is_ni ? term_is_ni[i] != 0 : false;
        owners[num_nodes + i] = db.addTerminal(i, name, term_w[i], term_h[i], true, ni);
        db.moduleMap[name] = owners[num_nodes + i];
    }
    db.moduleCount = num_nodes + num_terminals;

    db.allocateNetMemory(num_nets);
    db.allocatePinMemory(net_start[num_nets]);
    for (int n = 0; n < num_nets; n++)
    {
        Net *net = new Net(n);
        net->allocateMemoryForPin(net_start[n + 1] - net_start[n]);
        for (int p = net_start[n]; p < net_start[n + 1]; p++)
        {
            Module *m = owners[pin_owner[p]];
            int pinId = db.addPin(m, net, pin_dx[p], pin_dy[p]);
            m->addPin(db.dbPins[pinId]);
            net->addPin(db.dbPins[pinId]);
        }
        db.addNet(net);
    }
    db.pinCount = net_start[num_nets];
    db.netCount = num_nets;

    for (int i = 0; i < num_terminals; i++)
        db.setModuleLocation_2D(owners[num_nodes + i], term_llx[i], term_lly[i]);
    for (int i = 0; i < num_nodes; i++)
        db.setModuleCenter_2D(owners[i], node_cx[i], node_cy[i]);
    db.setChipRegion_2D();
    return h;
}

void ref_destroy(void *hp)
{
    // The reference leaks its bins, fillers and netlist objects by design
    // (raw owning pointers without destructors); only the handle is freed.
    delete static_cast<RefHandle *>(hp);
}

// QPPlacer::quadraticPlacement (QPlace/qplace.cpp:20-103).
double ref_qp(void *hp)
{
    Quiet q;
    RefHandle *h = static_cast<RefHandle *>(hp);
    QPPlacer qp(h->db);
    double t0 = now_s();
    qp.quadraticPlacement();
    return now_s() - t0;
}

// SAMacroLegalizer::legalization (Legalization/legalizer.cpp:701-845), as
// main/ePlace_main.cpp:176-181 runs it between mGP and FILLERONLY; returns
// its seconds.
double ref_macro_legalize(void *hp, float target_density)
{
    Quiet q;
    RefHandle *h = static_cast<RefHandle *>(hp);
    SAMacroLegalizer lg(h->db);
    lg.setTargetDensity(target_density);
    double t0 = now_s();
    lg.legalization();
    return now_s() - t0;
}

// AbacusLegalizer::legalization (Legalization/legalizer.cpp:58-183), the
// flow's internal legalizer (main/ePlace_main.cpp:251-262); returns its
// seconds.
double ref_abacus(void *hp)
{
    Quiet q;
    RefHandle *h = static_cast<RefHandle *>(hp);
    AbacusLegalizer lg(h->db);
    double t0 = now_s();
    lg.legalization();
    return now_s() - t0;
}

// DetailedPlacer::detailedPlacement (DetailedPlacement/detailed.cpp), run
// after the internal legalizer (main/ePlace_main.cpp:268-279); returns its
// seconds.
double ref_detailed(void *hp)
{
    Quiet q;
    RefHandle *h = static_cast<RefHandle *>(hp);
    DetailedPlacer dp(h->db);
    double t0 = now_s();
    dp.detailedPlacement();
    return now_s() - t0;
}

// Sizes known before initialization (netlist only).
void ref_netlist_counts(void *hp, int *out)
{
    RefHandle *h = static_cast<RefHandle *>(hp);
    out[0] = (int)h->db->dbNodes.size();
    out[1] = (int)h->db->dbTerminals.size();
    out[2] = (int)h->db->dbNets.size();
    out[3] = (int)h->db->dbPins.size();
    out[4] = (int)h->db->dbSiteRows.size();
    out[5] = h->db->dbMacroCount;
}

// Node centres (dbNodes order), e.g. after QP.
void ref_get_node_centers(void *hp, float *cx, float *cy)
{
    RefHandle *h = static_cast<RefHandle *>(hp);
    for (size_t i = 0; i < h->db->dbNodes.size(); i++)
    {
        cx[i] = h->db->dbNodes[i]->getCenter().x;
        cy[i] = h->db->dbNodes[i]->getCenter().y;
    }
}

void ref_set_node_centers(void *hp, const float *cx, const float *cy)
{
    RefHandle *h = static_cast<RefHandle *>(hp);
    for (size_t i = 0; i < h->db->dbNodes.size(); i++)
        h->db->setModuleCenter_2D(h->db->dbNodes[i], cx[i], cy[i]);
}

// EPlacer_2D::setTargetDensity + initialization (EPlace/eplace.cpp:27-50).
// srand(1) reproduces the unseeded glibc rand() of a fresh process, which is
// what places the fillers (PlaceDB/placedb.cpp:353-379).
double ref_init(void *hp, float target_density)
{
    Quiet q;
    RefHandle *h = static_cast<RefHandle *>(hp);
    srand(1);
    h->placer = new EPlacer_2D(h->db);
    h->placer->setTargetDensity(target_density);
    double t0 = now_s();
    h->placer->initialization();
    double dt = now_s() - t0;
    h->opt = new EplaceNesterovOpt<VECTOR_3D>(h->placer);
    h->initialized = true;
    return dt;
}

// Scalars: see the index list below.
void ref_get_info(void *hp, double *out)
{
    RefHandle *h = static_cast<RefHandle *>(hp);
    EPlacer_2D *p = h->placer;
    PlaceDB *db = h->db;
    out[0] = db->dbNodes.size();
    out[1] = p->ePlaceFillers.size();
    out[2] = p->binDimension.x;
    out[3] = p->binDimension.y;
    out[4] = p->binStep.x;
    out[5] = p->binStep.y;
    out[6] = db->coreRegion.ll.x;
    out[7] = db->coreRegion.ll.y;
    out[8] = db->coreRegion.ur.x;
    out[9] = db->coreRegion.ur.y;
    out[10] = p->ePlaceFillers.empty() ? 0.0 : p->ePlaceFillers[0]->getWidth();
    out[11] = p->ePlaceFillers.empty() ? 0.0 : p->ePlaceFillers[0]->getHeight();
    out[12] = p->ePlaceStdCellArea;
    out[13] = p->ePlaceMacroArea;
    out[14] = p->targetDensity;
    out[15] = p->globalDensityOverflow;
    out[16] = p->lambda;
    out[17] = p->invertedGamma.x;
    out[18] = p->invertedGamma.y;
    out[19] = p->lastHPWL;
    out[20] = p->placementStage;
    out[21] = p->mGPIterationCount;
    out[22] = db->totalRowArea;
    out[23] = p->ePlaceCellsAndFillers.size();
    out[24] = h->opt ? (double)h->opt->iter_count : 0.0;
    out[25] = h->opt ? (double)h->opt->NS_opt_param : 0.0;
}

// Centres of ePlaceNodesAndFillers (nodes, then fillers).
void ref_get_positions(void *hp, float *cx, float *cy)
{
    RefHandle *h = static_cast<RefHandle *>(hp);
    const std::vector<Module *> &all = h->placer->ePlaceNodesAndFillers;
    for (size_t i = 0; i < all.size(); i++)
    {
        cx[i] = all[i]->getCenter().x;
        cy[i] = all[i]->getCenter().y;
    }
}

// Write centres of ePlaceNodesAndFillers through PlaceDB::setModuleCenter_2D.
void ref_set_positions(void *hp, const float *cx, const float *cy)
{
    RefHandle *h = static_cast<RefHandle *>(hp);
    const std::vector<Module *> &all = h->placer->ePlaceNodesAndFillers;
    for (size_t i = 0; i < all.size(); i++)
        h->db->setModuleCenter_2D(all[i], cx[i], cy[i]);
}

// EPlacer_2D::totalGradientUpdate (EPlace/eplace.cpp:687-738).
double ref_eval(void *hp)
{
    Quiet q;
    RefHandle *h = static_cast<RefHandle *>(hp);
    double t0 = now_s();
    h->placer->totalGradientUpdate();
    return now_s() - t0;
}

void ref_set_lambda(void *hp, float lambda) { static_cast<RefHandle *>(hp)->placer->lambda = lambda; }
void ref_set_last_hpwl(void *hp, double v) { static_cast<RefHandle *>(hp)->placer->lastHPWL = v; }
void ref_penalty_init(void *hp) { static_cast<RefHandle *>(hp)->placer->penaltyFactorInitilization(); }
void ref_penalty_update(void *hp) { static_cast<RefHandle *>(hp)->placer->updatePenaltyFactor(); }
double ref_calc_hpwl(void *hp) { return static_cast<RefHandle *>(hp)->db->calcHPWL(); }

// Bin maps, x-major ([x][y] -> x*Ny + y).
void ref_get_bins(void *hp, float *node, float *filler, float *terminal, float *base,
                  float *ex, float *ey, float *phi)
{
    RefHandle *h = static_cast<RefHandle *>(hp);
    EPlacer_2D *p = h->placer;
    int nx = p->binDimension.x, ny = p->binDimension.y;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
        {
            Bin_2D *b = p->bins[i][j];
            size_t k = (size_t)i * ny + j;
            if (node) node[k] = b->nodeDensity;
            if (filler) filler[k] = b->fillerDensity;
            if (terminal) terminal[k] = b->terminalDensity;
            if (base) base[k] = b->baseDensity;
            if (ex) ex[k] = b->E.x;
            if (ey) ey[k] = b->E.y;
            if (phi) phi[k] = b->phi;
        }
}

// wirelengthGradient (nodes only), densityGradient and totalGradient
// (nodes + fillers), interleaved x,y.
void ref_get_gradients(void *hp, float *wl, float *dens, float *total)
{
    RefHandle *h = static_cast<RefHandle *>(hp);
    EPlacer_2D *p = h->placer;
    for (size_t i = 0; i < p->wirelengthGradient.size(); i++)
    {
        wl[2 * i] = p->wirelengthGradient[i].x;
        wl[2 * i + 1] = p->wirelengthGradient[i].y;
    }
    for (size_t i = 0; i < p->densityGradient.size(); i++)
    {
        dens[2 * i] = p->densityGradient[i].x;
        dens[2 * i + 1] = p->densityGradient[i].y;
        total[2 * i] = p->totalGradient[i].x;
        total[2 * i + 1] = p->totalGradient[i].y;
    }
}

// Stage-view gradient (getGradient, EPlace/eplace.cpp:742-756), interleaved.
int ref_get_stage_gradient(void *hp, float *g)
{
    RefHandle *h = static_cast<RefHandle *>(hp);
    std::vector<VECTOR_3D> v = h->placer->getGradient();
    for (size_t i = 0; i < v.size(); i++)
    {
        g[2 * i] = v[i].x;
        g[2 * i + 1] = v[i].y;
    }
    return (int)v.size();
}

// Whole stage: FirstOrderOptimizer::opt (Optimization/opt.hpp:30-36).
// Returns wall seconds; iterations via ref_get_info()[24].
double ref_opt_run(void *hp)
{
    Quiet q;
    RefHandle *h = static_cast<RefHandle *>(hp);
    double t0 = now_s();
    h->opt->opt();
    return now_s() - t0;
}

// Step-wise form of the same loop: begin = init(), step = one
// "if (!stop_condition()) opt_step()", end = wrap_up().
void ref_opt_begin(void *hp)
{
    Quiet q;
    static_cast<RefHandle *>(hp)->opt->init();
}

// Returns 1 if the loop stopped (no step taken), 0 after a step.
int ref_opt_step(void *hp, double *seconds)
{
    Quiet q;
    RefHandle *h = static_cast<RefHandle *>(hp);
    if (h->opt->stop_condition())
        return 1;
    double t0 = now_s();
    h->opt->opt_step();
    if (seconds)
        *seconds = now_s() - t0;
    return 0;
}

void ref_opt_end(void *hp)
{
    Quiet q;
    static_cast<RefHandle *>(hp)->opt->wrap_up();
}

// Optimizer vectors of the current stage view (interleaved x,y).
int ref_opt_state(void *hp, float *x, float *y, float *g, float *y_prev, float *g_prev)
{
    RefHandle *h = static_cast<RefHandle *>(hp);
    auto &c = h->opt->cur_iter;
    auto &l = h->opt->last_iter;
    size_t n = c.main_solution.size();
    for (size_t i = 0; i < n; i++)
    {
        if (x) { x[2 * i] = c.main_solution[i].x; x[2 * i + 1] = c.main_solution[i].y; }
        if (y && i < c.reference_solution.size()) { y[2 * i] = c.reference_solution[i].x; y[2 * i + 1] = c.reference_solution[i].y; }
        if (g && i < c.gradient.size()) { g[2 * i] = c.gradient[i].x; g[2 * i + 1] = c.gradient[i].y; }
        if (y_prev && i < l.reference_solution.size()) { y_prev[2 * i] = l.reference_solution[i].x; y_prev[2 * i + 1] = l.reference_solution[i].y; }
        if (g_prev && i < l.gradient.size()) { g_prev[2 * i] = l.gradient[i].x; g_prev[2 * i + 1] = l.gradient[i].y; }
    }
    return (int)n;
}

void ref_switch_filler_only(void *hp) { static_cast<RefHandle *>(hp)->placer->switch2FillerOnly(); }
void ref_switch_cgp(void *hp) { static_cast<RefHandle *>(hp)->placer->switch2cGP(); }

// Node flags: 1 = macro.  Filler flags are implicit (index >= nodes).
void ref_get_node_flags(void *hp, unsigned char *is_macro)
{
    RefHandle *h = static_cast<RefHandle *>(hp);
    for (size_t i = 0; i < h->db->dbNodes.size(); i++)
        is_macro[i] = h->db->dbNodes[i]->isMacro ? 1 : 0;
}

// Ooura 2-D transforms on a caller grid (x-major), for checking the dense
// restatement of FFT_2D::doFFT: kind 0 = ddct2d, 1 = ddsct2d, 2 = ddcst2d.
void ref_ooura_2d(int kind, int n1, int n2, int isgn, float *data)
{
    std::vector<float *> rows(n1);
    for (int i = 0; i < n1; i++)
        rows[i] = data + (size_t)i * n2;
    int nmax = std::max(n1, n2);
    std::vector<float> w(nmax * 3 / 2, 0.0f);
    std::vector<int> ip((int)round(sqrt((double)nmax)) + 2, 0);
    if (kind == 0)
        replace::ddct2d(n1, n2, isgn, rows.data(), nullptr, ip.data(), w.data());
    else if (kind == 1)
        replace::ddsct2d(n1, n2, isgn, rows.data(), nullptr, ip.data(), w.data());
    else
        replace::ddcst2d(n1, n2, isgn, rows.data(), nullptr, ip.data(), w.data());
}

} // extern "C"
