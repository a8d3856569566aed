"""Quadratic placement on the device (ep_quadratic_placement) against the
reference's QPPlacer::quadraticPlacement (QPlace/qplace.cpp:20-106), whose
results tests/golden/variants.npz holds (make_golden.py).

Both sides run BiCGSTAB capped at 100 iterations per solve, which on these
designs ends before the solve converges (|r|/|b| ~ 1e-7 .. 1e-6); what one
float iteration order leaves unconverged the other leaves slightly
differently, so individual weakly connected nodes can land apart.  The
checks are therefore on the outcome: HPWL within 1%, mean node displacement
below 1% of the die, the solver errors below the reference's 1e-6 round
criterion, bitwise repeatability, and the reference's own flow (QP, then
mGP) on its smoke example ending within 2% of the reference's HPWL.
"""
import numpy as np
import pytest

from eplace_b200 import placer, synth
from tests.helpers import golden_netlist, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def variants():
    return load_golden("variants")


def engine_for(g, **kw):
    p = placer.default_params(target_density=float(g["target_density"]), **kw)
    return placer.Engine(golden_netlist(g), p)


@pytest.mark.parametrize("design", ["stdcell_2k", "mixed_5k"])
def test_quadratic_placement_matches_reference(variants, design):
    g = load_golden(design)
    e = engine_for(g)
    st = e.quadratic_placement()
    nn = int(g["info_num_nodes"])
    xy = e.get_positions()[:nn]
    ref = np.stack([variants[f"qp_{design}_cx"], variants[f"qp_{design}_cy"]], 1)
    i = e.info
    die = max(i.core_urx - i.core_llx, i.core_ury - i.core_lly)
    assert abs(st["hpwl"] / float(variants[f"qp_{design}_hpwl"]) - 1) < 0.01
    assert np.abs(xy - ref).mean() / die < 0.01
    assert st["error_x"] < 1e-6 and st["error_y"] < 1e-6
    assert st["rounds"] >= 6  # the reference's "i > 4" before its error test


def test_quadratic_placement_is_repeatable():
    g = load_golden("stdcell_2k")
    e = engine_for(g)
    e.quadratic_placement()
    a = e.get_positions()
    e.quadratic_placement()  # starts from the core centre again
    assert np.array_equal(a, e.get_positions())


def test_qp_then_mgp_matches_reference_flow():
    # ref_smoke's reference run started from the reference's own QP
    g = load_golden("ref_smoke")
    e = engine_for(g, keep_maps=1)
    e.set_positions(np.stack([g["init_cx"], g["init_cy"]], 1))  # the reference's fillers
    e.quadratic_placement()
    e.initialize()
    st = e.nesterov_run()
    assert st["overflow"] < 0.1
    assert abs(st["hpwl"] / float(g["run_hpwl"]) - 1) < 0.02


def test_quadratic_refine_keeps_a_converged_placement_and_improves_a_blob():
    nl = synth.standard_cell(5_000, seed=3, every_cell_pinned=True, local_pads=True)
    e = placer.Engine(nl, placer.default_params(target_density=1.0))
    full = e.quadratic_placement()
    ref = e.get_positions()
    st = e.quadratic_refine(2)
    assert st["rounds"] == 2
    assert st["hpwl"] == pytest.approx(full["hpwl"], rel=0.005)
    core = max(e.info.core_urx - e.info.core_llx, e.info.core_ury - e.info.core_lly)
    assert np.abs(e.get_positions() - ref).mean() < 0.01 * core
    b = placer.Engine(synth.blob_start(nl, sigma_frac=0.2), placer.default_params(target_density=1.0))
    h0 = b.hpwl()
    assert b.quadratic_refine(3)["hpwl"] < 0.5 * h0
    with pytest.raises(placer.EPError):
        b.quadratic_refine(0)
    e.close()
    b.close()


def test_jacobi_refine_solves_the_same_system_in_fewer_iterations():
    """ep_quadratic_refine with the Jacobi preconditioner (Eigen's
    DiagonalPreconditioner form of BiCGSTAB): one round from a blob solves
    the same system -- with 100 iterations both forms land on the same
    placement -- and after 20 iterations its residual is below the
    unpreconditioned solver's."""
    nl = synth.blob_start(synth.standard_cell(20_000, seed=8, every_cell_pinned=True, local_pads=True),
                          sigma_frac=0.2)
    out = {}
    for its, jac in ((100, 0), (100, 1), (20, 0), (20, 1)):
        e = placer.Engine(nl, placer.default_params(target_density=1.0))
        st = e.quadratic_refine(1, its, jac)
        out[(its, jac)] = (st, e.get_positions()[:nl.num_nodes])
        core = max(e.info.core_urx - e.info.core_llx, e.info.core_ury - e.info.core_lly)
        e.close()
    (a, pa), (b, pb) = out[(100, 0)], out[(100, 1)]
    assert b["hpwl"] == pytest.approx(a["hpwl"], rel=0.002)
    assert np.abs(pa - pb).mean() < 0.002 * core
    e20, j20 = out[(20, 0)][0], out[(20, 1)][0]
    assert max(j20["error_x"], j20["error_y"]) < max(e20["error_x"], e20["error_y"])
    e = placer.Engine(nl, placer.default_params(target_density=1.0))
    with pytest.raises(placer.EPError):
        e.quadratic_refine(1, 20, 2)
    e.close()
