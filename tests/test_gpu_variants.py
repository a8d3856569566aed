"""The engine's non-default options and later stages against the reference
(tests/golden/variants.npz, written by make_golden.py from the unmodified
reference) and the FP64 oracle:

  * LSE wirelength model (gArg "LSE", EPlace/eplace.cpp:512-549,
    PlaceCommon/objects.cpp:161-241,423-437): gradient at the initial
    positions within 1e-4 of the reference; whole mGP run within 10%
    iterations and 1% HPWL;
  * Barzilai-Borwein step (gArg "bb", Optimization/nesterov.hpp:231-302) and
    backtracking step (gArg "bktrk", :310-369): whole run within 10%
    iterations and 1% HPWL; backtracking one step at a time gives bitwise the
    run's positions;
  * exact exp instead of fastExp: wirelength gradient within 1e-4 of the FP64
    oracle evaluated with exp;
  * mixed-size stages (EPlace/eplace.cpp:887-904): FILLERONLY runs exactly 20
    steps and moves fillers only, lambda grows by 1.05 per step at constant
    HPWL, switch2cGP divides lambda by 1.1^(0.1 * mGP iterations), cGP keeps
    the macros fixed and reaches overflow < 0.07 within 25% of the reference's
    iterations and 2% of its HPWL;
  * failure detection: a non-finite position is reported as EP_ERR_NAN by the
    run, and the engine stays usable afterwards.
"""
import numpy as np
import pytest

from eplace_b200 import placer
from tests.helpers import OracleDesign, golden_netlist, load_golden, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def variants():
    return load_golden("variants")


def engine_at_reference_start(g, **kw):
    p = placer.default_params(target_density=float(g["target_density"]), keep_maps=1)
    for k, v in kw.items():
        setattr(p, k, v)
    e = placer.Engine(golden_netlist(g), p)
    e.set_positions(np.stack([g["init_cx"], g["init_cy"]], 1))
    return e


def test_lse_gradient_matches_reference(variants):
    g = load_golden("stdcell_2k")  # the same design and start as the LSE fixture
    e = engine_at_reference_start(g, wl_model=placer.WL_LSE)
    e.initialize()
    _, gw = e.component_gradients()
    n = int(g["info_num_nodes"])
    assert rel_err(gw[:n], variants["lse_init_grad_wl"]) < 1e-4


def test_lse_run_matches_reference(variants):
    g = load_golden("stdcell_2k")
    e = engine_at_reference_start(g, wl_model=placer.WL_LSE)
    e.initialize()
    st = e.nesterov_run()
    it = int(variants["lse_run_iterations"])
    assert abs(st["iterations"] - it) <= max(2, 0.1 * it), (st["iterations"], it)
    assert st["overflow"] < 0.1
    assert abs(st["hpwl"] / float(variants["lse_run_hpwl"]) - 1) < 0.01


def test_bb_run_matches_reference(variants):
    g = load_golden("stdcell_2k")
    e = engine_at_reference_start(g, step_rule=placer.STEP_BB)
    e.initialize()
    st = e.nesterov_run()
    it = int(variants["bb_run_iterations"])
    assert abs(st["iterations"] - it) <= max(2, 0.1 * it), (st["iterations"], it)
    assert st["overflow"] < 0.1
    assert abs(st["hpwl"] / float(variants["bb_run_hpwl"]) - 1) < 0.01


def test_bktrk_run_matches_reference(variants):
    g = load_golden("stdcell_2k")
    e = engine_at_reference_start(g, step_rule=placer.STEP_BKTRK)
    e.initialize()
    st = e.nesterov_run()
    it = int(variants["bktrk_run_iterations"])
    assert abs(st["iterations"] - it) <= max(2, 0.1 * it), (st["iterations"], it)
    assert st["overflow"] < 0.1
    assert abs(st["hpwl"] / float(variants["bktrk_run_hpwl"]) - 1) < 0.01


def test_bktrk_steps_one_at_a_time_match_the_run():
    g = load_golden("stdcell_2k")
    runs = []
    for stepwise in (False, True):
        e = engine_at_reference_start(g, step_rule=placer.STEP_BKTRK)
        e.initialize()
        if stepwise:
            e.nesterov_begin()
            for _ in range(6):
                assert not e.nesterov_step()
            e.nesterov_end()
        else:
            e.nesterov_run(max_steps=6)
        runs.append(e.get_positions())
    assert np.array_equal(runs[0], runs[1])


def test_exact_exp_gradient_matches_oracle():
    g = load_golden("stdcell_2k")
    e = engine_at_reference_start(g, exp_mode=placer.EXP_EXACT)
    e.initialize()
    _, gw = e.component_gradients()
    d = OracleDesign.from_golden(g)
    r = d.evaluate(g["init_cx"], g["init_cy"], 0.0, exp_mode=1, qscale=e.info.density_scale)
    n = int(g["info_num_nodes"])
    assert rel_err(gw[:n], r["gwl"][:n]) < 1e-4


def test_mixed_size_stage_sequence(variants):
    g = load_golden("mixed_5k")  # the design of the stage fixture
    e = engine_at_reference_start(g)
    assert np.array_equal(e.get_positions()[:, 0], variants["stage_init_cx"])
    e.initialize()
    mgp = e.nesterov_run()
    it_ref = int(variants["stage_mgp_iterations"])
    assert abs(mgp["iterations"] - it_ref) <= max(2, 0.1 * it_ref)
    it_mgp = int(e.query()["mgp_iterations"])
    assert it_mgp == mgp["iterations"]

    # continue from the reference's state at the switch: its mGP result and
    # its re-drawn fillers, its lambda
    e.switch_stage(placer.FILLERONLY)
    start = np.stack([variants["stage_fo_start_cx"], variants["stage_fo_start_cy"]], 1)
    e.set_positions(start)
    lam0 = float(variants["stage_mgp_lambda"])
    e.set_lambda(lam0)
    fo = e.nesterov_run()
    assert fo["iterations"] == 20 == int(variants["stage_fo_iterations"])
    after = e.get_positions()
    nn = int(g["info_num_nodes"])
    assert np.array_equal(after[:nn], start[:nn]), "FILLERONLY moved a cell"
    assert not np.array_equal(after[nn:], start[nn:])
    # cells fixed: HPWL constant, so updatePenaltyFactor multiplies by 1.05
    # each step (the first step compares with the engine's own last mGP HPWL,
    # a few 1e-5 away from exactly 1.05)
    assert abs(fo["hpwl"] / float(variants["stage_fo_hpwl"]) - 1) < 1e-6
    lam_fo = e.query()["lambda_"]
    assert abs(lam_fo / (lam0 * 1.05 ** 20) - 1) < 1e-4
    assert abs(lam_fo / float(variants["stage_fo_lam"]) - 1) < 1e-4

    e.switch_stage(placer.CGP)
    lam_c = e.query()["lambda_"]
    assert abs(lam_c / (lam_fo / 1.1 ** (0.1 * it_mgp)) - 1) < 1e-6
    assert abs(lam_c / float(variants["stage_cgp_start_lambda"]) - 1) < 1.1 ** (0.1 * abs(it_mgp - it_ref)) - 1 + 1e-6
    before = e.get_positions()
    cg = e.nesterov_run()
    final = e.get_positions()
    macro = np.asarray(g["node_is_macro"]).astype(bool)
    assert macro.any()
    assert np.array_equal(final[:nn][macro], before[:nn][macro]), "cGP moved a macro"
    assert cg["overflow"] < 0.07
    it_c = int(variants["stage_cgp_iterations"])
    assert abs(cg["iterations"] - it_c) <= max(3, 0.25 * it_c), (cg["iterations"], it_c)
    assert abs(cg["hpwl"] / float(variants["stage_cgp_hpwl"]) - 1) < 0.02


@pytest.mark.parametrize("design", ["stdcell_2k", "mixed_5k"])
def test_fused_update_scatter_loop_matches_separate_scatter(design):
    """Without kept maps the captured loop scatters inside the update kernel;
    with them it scatters at the start of each evaluation.  Same integer maps,
    so the runs agree bit for bit (mixed_5k has block-per-object objects).  A
    capped run must leave the maps clear: the next evaluation sees the same
    overflow either way."""
    g = load_golden(design)
    res = []
    for keep in (1, 0):
        e = engine_at_reference_start(g, keep_maps=keep)
        e.initialize()
        capped = e.nesterov_run(max_steps=7)
        e.eval_gradient()
        tau_after = e.query()["overflow"]
        st = e.nesterov_run()
        res.append((capped["iterations"], tau_after, st["iterations"], e.get_positions()))
    assert res[0][0] == res[1][0] == 7
    assert res[0][1] == res[1][1]
    assert res[0][2] == res[1][2]
    assert np.array_equal(res[0][3], res[1][3])


def test_nan_position_reported_and_engine_recovers():
    g = load_golden("stdcell_2k")
    e = engine_at_reference_start(g)
    e.initialize()
    xy = e.get_positions()
    bad = xy.copy()
    bad[7, 0] = np.nan
    e.set_positions(bad)
    with pytest.raises(placer.EPError) as ex:
        e.nesterov_run()
    assert ex.value.status == placer.EP_ERR_NAN
    # the context and the engine stay usable
    e.set_positions(xy)
    e.initialize()
    st = e.nesterov_run()
    assert st["overflow"] < 0.1


def test_run_batch_matches_single_runs():
    """ep_run_batch interleaves several engines' loops on their own streams;
    each ends exactly as its own ep_nesterov_run would (different designs,
    options and stop conditions in one batch)."""
    cases = [("stdcell_2k", {}), ("mixed_5k", {}), ("stdcell_2k", {"step_rule": placer.STEP_BB}),
             ("ref_smoke", {})]
    solo, batch = [], []
    for target in (solo, batch):
        for name, kw in cases:
            g = load_golden(name)
            p = placer.default_params(target_density=float(g["target_density"]), **kw)
            e = placer.Engine(golden_netlist(g), p)
            e.set_positions(np.stack([g["init_cx"], g["init_cy"]], 1))
            e.initialize()
            target.append(e)
    single = [e.nesterov_run() for e in solo]
    many = placer.run_batch(batch)
    for a, b, ea, eb in zip(single, many, solo, batch):
        assert a["iterations"] == b["iterations"]
        assert a["hpwl"] == b["hpwl"]
        assert np.array_equal(ea.get_positions(), eb.get_positions())
