// eplace_b200.hpp -- header-only C++17 adapter over the C-ABI of eplace_gpu.h
// that keeps the call surface of the reference's EPlacer_2D
// (EPlace/eplace.h:95-200) and EplaceNesterovOpt (Optimization/nesterov.hpp:59-77),
// so a driver written against the reference (main/ePlace_main.cpp:141-211)
// keeps its calls.  Errors throw eplace_b200::Error (the reference exits).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "eplace_gpu.h"

namespace eplace_b200 {

struct Error : std::runtime_error {
    ep_status status;
    Error(ep_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

struct Vec2 {
    float x, y;
};

class EPlacer2D {
  public:
    EPlacer2D(const ep_netlist &nl, const ep_params &p) {
        ep_status s = ep_create(&nl, &p, &e_);
        if (s != EP_OK) {
            std::string m = e_ ? ep_last_error(e_) : "ep_create failed";
            ep_destroy(e_);
            e_ = nullptr;
            throw Error(s, m);
        }
        check(ep_get_info(e_, &info_));
    }
    ~EPlacer2D() { ep_destroy(e_); }
    EPlacer2D(const EPlacer2D &) = delete;
    EPlacer2D &operator=(const EPlacer2D &) = delete;

    // initialization(): fillers and bins were built by ep_create; this runs
    // the first totalGradientUpdate and penaltyFactorInitilization.
    void initialization() { check(ep_initialize(e_)); }
    void totalGradientUpdate() { check(ep_eval_gradient(e_)); }
    std::vector<Vec2> getGradient() { return view(ep_get_gradient); }
    std::vector<Vec2> getPosition() { return view(ep_get_positions); }
    void setPosition(const std::vector<Vec2> &xy) {
        check(ep_set_positions(e_, stage(), &xy[0].x, (int32_t)xy.size()));
    }
    void penaltyFactorInitilization() { check(ep_penalty_init(e_)); }
    void updatePenaltyFactor() { check(ep_penalty_update(e_)); }
    void switch2FillerOnly() { check(ep_switch_stage(e_, EP_STAGE_FILLERONLY, nullptr)); }
    void switch2cGP() { check(ep_switch_stage(e_, EP_STAGE_CGP, nullptr)); }

    // public fields of EPlacer_2D, read through ep_query
    float globalDensityOverflow() { return (float)scalars().overflow; }
    float lambda() { return (float)scalars().lambda; }
    int placementStage() { return scalars().stage; }
    int mGPIterationCount() { return scalars().mgp_iterations; }
    double calcHPWL() {
        double h = 0;
        check(ep_hpwl(e_, &h));
        return h;
    }
    const ep_info &info() const { return info_; }
    ep_engine *handle() { return e_; }

  private:
    ep_engine *e_ = nullptr;
    ep_info info_{};

    void check(ep_status s) {
        if (s != EP_OK) throw Error(s, ep_last_error(e_));
    }
    ep_scalars scalars() {
        ep_scalars s{};
        check(ep_query(e_, &s));
        return s;
    }
    int stage() { return scalars().stage; }
    int view_size(int st) const {
        return st == EP_STAGE_MGP ? info_.num_objects
                                  : st == EP_STAGE_FILLERONLY ? info_.num_fillers : info_.num_cells_and_fillers;
    }
    template <typename F>
    std::vector<Vec2> view(F fn) {
        int st = stage();
        std::vector<Vec2> v(view_size(st));
        if (!v.empty()) check(fn(e_, st, &v[0].x, (int32_t)v.size()));
        return v;
    }
};

// FirstOrderOptimizer<T>::opt with EplaceNesterovOpt's steps; the loop runs
// on the device.
class EplaceNesterovOpt {
  public:
    explicit EplaceNesterovOpt(EPlacer2D *placer) : p_(placer) {}
    ep_run_stats opt(int max_steps = 0) {
        ep_run_stats st{};
        ep_status s = ep_nesterov_run(p_->handle(), max_steps, &st);
        if (s != EP_OK) throw Error(s, ep_last_error(p_->handle()));
        return st;
    }

  private:
    EPlacer2D *p_;
};

}  // namespace eplace_b200
