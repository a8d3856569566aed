"""The engine's global placement inside the reference's whole flows, the
reference's CPU stages run on the engine's output through the compiled
reference (tests/ref_stages.py, a child process):

  * config 1 (synth.smoke: 100 cells, 16 x 16 bins, targetDensity 0.8, QP
    start, FP64): engine mGP (from the reference's start, and as the
    engine's own flow from its device QP), then the reference's
    AbacusLegalizer and DetailedPlacer (main/ePlace_main.cpp:248-279).  The
    exact-integer checker (eplace_b200/legality.py) passes after both;
    HPWL against the reference's own flow (tests/golden/flows.npz) as each
    test states;
  * mixed-size ePlace-MS (mixed_5k from its recorded start): engine mGP,
    the reference's SAMacroLegalizer on the engine's result (macros checked
    for overlap in integers), then the engine's FILLERONLY and cGP stages
    (main/ePlace_main.cpp:174-211): cGP ends below overflow 0.1 with macros
    fixed, HPWL within 3% of the reference's flow.
"""
import numpy as np
import pytest

from eplace_b200 import legality, placer, synth
from oracle import refharness as R
from tests import ref_stages
from tests.helpers import golden_netlist, load_golden

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="reference harness not built")]


@pytest.fixture(scope="module")
def flows():
    return load_golden("flows")


def _config1_engine(nl, bins):
    """bins 0: the reference's bin-count rule (8 x 8 on these designs)."""
    return placer.Engine(nl, placer.default_params(target_density=0.8, bins_x=bins, bins_y=bins,
                                                   precision=placer.PREC_FP64))


def _legalize_and_check(nl, seed, xy, tmp_path):
    rc, out = ref_stages.run(f"smoke:{seed}", xy[:, 0], xy[:, 1], 0.8, ["abacus", "detailed"], str(tmp_path))
    if rc < 0 and "abacus_cx" not in out:
        pytest.skip(f"the reference's legalizer or detailed placer ended its process (signal {-rc})")
    assert rc == 0
    r = legality.check(nl, out["abacus_cx"], out["abacus_cy"])
    assert r["legal"], r
    r = legality.check(nl, out["detailed_cx"], out["detailed_cy"])
    assert r["legal"], r
    assert out["detailed_hpwl"] <= out["abacus_hpwl"] + 1e-9
    return out


@pytest.mark.parametrize("seed", [1, 2, 4])
def test_config1_from_reference_start_then_reference_legalizer(flows, seed, tmp_path):
    """From the reference's own start (its QP result and fillers) on the
    reference's bin grid (its rule gives 8 x 8 here; the reference cannot be
    given another): the engine's mGP within 10% of the reference's
    iterations and 2% of its HPWL; after the reference's Abacus + detailed
    placement on it, legal and within 3% of the reference's flow."""
    nl = synth.smoke(seed)
    k = f"c1_{seed}_"
    e = _config1_engine(nl, 0)
    assert e.info.bins_x == e.info.bins_y == 8
    e.set_positions(np.stack([flows[k + "init_cx"], flows[k + "init_cy"]], 1))
    e.initialize()
    st = e.nesterov_run()
    assert st["overflow"] < 0.1
    it = int(flows[k + "gp_iterations"])
    assert abs(st["iterations"] - it) <= max(2, 0.1 * it), (st["iterations"], it)
    # 2%: on 100 cells one cell ending in another bin moves the HPWL by ~1%
    assert st["hpwl"] == pytest.approx(float(flows[k + "gp_hpwl"]), rel=0.02)
    xy = e.get_positions()[:nl.num_nodes]
    e.close()
    out = _legalize_and_check(nl, seed, xy, tmp_path)
    assert float(out["detailed_hpwl"]) == pytest.approx(float(flows[k + "dp_hpwl"]), rel=0.03)


@pytest.mark.parametrize("seed", [1, 2, 4])
def test_config1_engine_flow_then_reference_legalizer(flows, seed, tmp_path):
    """Config 1 as specified -- 16 x 16 bins -- with the engine's whole global
    placement (device QP, its own fillers, mGP), then the reference's Abacus
    + detailed placement: legal, and within 6% of the reference's flow (which
    ran on its own 8 x 8 grid; on 100 cells the grid and the fillers' random
    start move the result by a few percent)."""
    nl = synth.smoke(seed)
    e = _config1_engine(nl, 16)
    e.quadratic_placement()
    e.initialize()
    st = e.nesterov_run()
    assert st["overflow"] < 0.1
    xy = e.get_positions()[:nl.num_nodes]
    e.close()
    out = _legalize_and_check(nl, seed, xy, tmp_path)
    assert float(out["detailed_hpwl"]) == pytest.approx(float(flows[f"c1_{seed}_dp_hpwl"]), rel=0.06)


def test_mixed_size_flow_with_reference_macro_legalizer(flows, tmp_path):
    g = load_golden("mixed_5k")
    nl = golden_netlist(g)
    assert np.array_equal(nl.node_w, synth.blob_start(synth.mixed_size(5000, 6, 3, seed=5)).node_w)
    e = placer.Engine(nl, placer.default_params(target_density=float(g["target_density"])))
    e.set_positions(np.stack([g["init_cx"], g["init_cy"]], 1))
    e.initialize()
    mgp = e.nesterov_run()
    assert mgp["overflow"] < 0.1
    assert mgp["hpwl"] == pytest.approx(float(flows["mlg_mgp_hpwl"]), rel=0.03)
    nn = nl.num_nodes
    xy = e.get_positions()
    rc, out = ref_stages.run("mixed_5k", xy[:nn, 0], xy[:nn, 1], float(g["target_density"]), ["mlg"],
                             str(tmp_path))
    assert rc == 0
    macro = np.asarray(nl.node_h) > 1.0
    assert macro.sum() == 6
    r = legality.check(nl, out["mlg_cx"], out["mlg_cy"], macros_only=True)
    assert r["legal"], r
    # mLG moves macros only
    assert np.array_equal(out["mlg_cx"][~macro], xy[:nn, 0][~macro])
    e.switch_stage(placer.FILLERONLY)
    allp = e.get_positions()
    allp[:nn] = np.stack([out["mlg_cx"], out["mlg_cy"]], 1)
    e.set_positions(allp)
    fo = e.nesterov_run()
    assert fo["iterations"] == 20
    e.switch_stage(placer.CGP)
    before = e.get_positions()
    cg = e.nesterov_run()
    final = e.get_positions()
    assert np.array_equal(final[:nn][macro], before[:nn][macro]), "cGP moved a macro"
    assert cg["overflow"] < 0.1
    assert cg["hpwl"] == pytest.approx(float(flows["mlg_cgp_hpwl"]), rel=0.03)
    e.close()
