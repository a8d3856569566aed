"""The C restatement (oracle/) pinned against the reference's own outputs.

Golden fixtures (tests/golden/*.npz) were produced by the unmodified
reference (tests/golden/make_golden.py); these tests need no GPU and no
reference tree.  Tolerances: exact for the integer-like setup (filler count,
bin grid, terminal / base maps, HPWL); 1e-5 relative for the float-accumulated
maps, field, gather and combine; 5e-3 for the float WA gradient against the
FP64 restatement (the reference forms the quotient-rule numerators in float,
which cancel for the clustered cells of a QP start)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import DESIGNS, OracleDesign, golden_netlist, load_golden, rel_err


@pytest.fixture(scope="module", params=DESIGNS)
def case(request):
    g = load_golden(request.param)
    return request.param, g, OracleDesign.from_golden(g)


def test_setup_matches_reference(case):
    name, g, d = case
    nl = golden_netlist(g)
    fs = O.filler_sizing(nl, g["node_is_macro"])
    assert fs["num_fillers"] == int(g["info_num_fillers"])
    assert np.float32(fs["filler_w"]) == np.float32(g["info_filler_w"])
    assert np.float32(fs["std_area"]) == np.float32(g["info_std_area"])
    bd = O.bin_dimension(fs["std_area"], fs["macro_area"], nl.num_nodes,
                         g["info_core_urx"] - g["info_core_llx"], g["info_core_ury"] - g["info_core_lly"],
                         float(g["target_density"]))
    if name != "ref_smoke":  # the smoke example is run with the automatic rule too
        assert bd == int(g["info_bins_x"])
    term, base = d.term, d.base
    assert np.array_equal(term, g["init_terminal"])
    assert np.array_equal(base, g["init_base"])


def test_evaluation_matches_reference(case):
    name, g, d = case
    r = d.evaluate(g["init_cx"], g["init_cy"], 0.0)
    assert rel_err(r["node"], g["init_node"]) < 1e-5
    assert rel_err(r["filler"], g["init_filler"]) < 1e-5
    assert abs(r["tau"] - g["info_overflow"]) < 1e-5 * max(1.0, g["info_overflow"])
    assert r["hpwl"] == pytest.approx(float(g["info_last_hpwl"]), rel=1e-12)
    # the Poisson solve against the reference's Ooura transforms
    binA = d.bin_area()
    rho = (g["init_node"].astype(np.float64) + g["init_base"] + g["init_filler"] + g["init_terminal"]) / binA
    ex, ey, phi = O.poisson(rho, d.grid.step_x, d.grid.step_y)
    assert rel_err(ex, g["init_ex"]) < 1e-5
    assert rel_err(ey, g["init_ey"]) < 1e-5
    assert rel_err(phi, g["init_phi"]) < 1e-5
    gd = O.gather(d.grid, g["init_cx"], g["init_cy"], d.w, d.h, g["init_ex"], g["init_ey"])
    assert rel_err(gd, g["init_grad_density"]) < 1e-5
    _, hp, gwl = O.wirelength_grad(d.nl_obj, g["init_cx"], g["init_cy"], d.tcx, d.tcy,
                                   g["info_inv_gamma_x"], g["info_inv_gamma_y"], 0)
    assert rel_err(gwl[:d.nl.num_nodes], g["init_grad_wl"]) < 5e-3
    lam0 = O.lambda0(d.nl.num_nodes, np.concatenate([g["init_grad_wl"], np.zeros((d.nf, 2))]),
                     g["init_grad_density"])
    assert lam0 == pytest.approx(float(g["eval2_lambda"]), rel=1e-5)
    tot = O.combine(d.ppo, d.area, d.flags, g["eval2_lambda"], g["init_grad_density"],
                    np.concatenate([g["init_grad_wl"], np.zeros((d.nf, 2))]))
    assert rel_err(tot, g["eval2_grad_total"]) < 1e-5


def test_inv_gamma_and_lambda_rules():
    # 1/gamma schedule branches (EPlace/eplace.cpp:482-498) and the lambda
    # multiplier clamp (EPlace/eplace.cpp:852-870)
    gx, _ = O.inv_gamma(1.5, 2.0, 2.0)
    assert gx == pytest.approx(0.125 / 2.0 * 0.1)
    gx, _ = O.inv_gamma(0.05, 2.0, 2.0)
    assert gx == pytest.approx(0.125 / 2.0 * 10.0)
    gx, _ = O.inv_gamma(0.55, 2.0, 2.0)
    assert gx == pytest.approx(0.125 / 2.0 / 10 ** ((0.55 - 0.1) * 20 / 9 - 1))
    assert O.lambda_multiplier(100.0, 200.0) == pytest.approx(1.05)
    assert O.lambda_multiplier(200.0, 100.0) == pytest.approx(1.05 ** (1 - 100 / 350000))
    assert O.lambda_multiplier(2e6, 0.0) == pytest.approx(0.95)


def test_mgp_loop_outcome_matches_reference():
    # the FP64 restatement of the whole loop lands on the reference's outcome
    g = load_golden("stdcell_2k")
    d = OracleDesign.from_golden(g)
    x, y, st = O.mgp_run(d.grid, d.nl_obj, d.w, d.h, d.flags, d.ppo, d.nf, d.tcx, d.tcy, d.term, d.base,
                         d.std_area(), d.macro_area(), g["init_cx"], g["init_cy"])
    assert st["overflow"] < 0.1
    assert abs(st["iterations"] - int(g["run_iterations"])) <= 0.1 * int(g["run_iterations"])
    assert st["hpwl"] == pytest.approx(float(g["run_hpwl"]), rel=0.01)
