"""The 200k-cell design bench.py measures (bench.netlist(): 200k cells, 220k
nets, 2k pads, 512 x 512 bins, targetDensity 1.0) against the reference's
own runs on it (tests/golden/reference_runs.json, written by
tests/golden/make_golden.py --bench from the unmodified reference).

Tolerances:
  * from the seeded blob start (bench.design()): overflow below 0.1,
    iterations within 10% and HPWL within 0.5% of the reference's mGP run, in
    both the mixed-precision and the FP64 form;
  * quadratic placement round for round: stopped after the reference's
    number of rounds (or earlier, where its own stopping test passes), the
    engine's HPWL within 1% of the reference's HPWL after that many rounds
    (the reference's per-round log);
  * the reference flow, quadratic placement then mGP: the engine's device
    quadratic placement with its own stopping test within 2% of the
    reference's HPWL after QP, and the mGP run from it within 10% of the
    reference's iterations and 1% of its HPWL.  Both quadratic placements
    stop their BiCGSTAB at 100 iterations unconverged; the reference's last
    round ends with its error at the stopping threshold (1e-6), so float
    rounding decides between stopping there and one to three rounds more,
    each lowering HPWL by about 1%.
"""
import json
import os

import pytest

import bench
from eplace_b200 import placer

pytestmark = pytest.mark.gpu

RUNS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_runs.json")


def _ref(key):
    with open(RUNS) as f:
        return json.load(f)[key]


@pytest.mark.parametrize("precision", [placer.PREC_MIXED, placer.PREC_FP64])
def test_blob_start_mgp_matches_reference(precision):
    ref = _ref("stdcell_200k_blob_mgp")
    e = placer.Engine(bench.design(), placer.default_params(target_density=1.0, precision=precision))
    assert e.info.bins_x == ref["bins"] and e.info.num_fillers == ref["fillers"]
    e.initialize()
    st = e.nesterov_run()
    assert st["overflow"] < 0.1
    assert abs(st["iterations"] - ref["iterations"]) <= 0.1 * ref["iterations"], (st, ref)
    assert st["hpwl"] == pytest.approx(ref["hpwl"], rel=0.005)
    e.close()


def test_quadratic_placement_follows_reference_rounds():
    trace = _ref("stdcell_200k_qp_mgp")["qp_trace"]
    assert trace[-1][2] == pytest.approx(_ref("stdcell_200k_qp_mgp")["qp_hpwl"], rel=1e-9)
    e = placer.Engine(bench.netlist(), placer.default_params(target_density=1.0))
    st = e.quadratic_placement(max_iterations=len(trace) - 1)
    k = st["rounds"]
    assert 6 <= k <= len(trace)  # the stopping test counts from the sixth round
    assert st["hpwl"] == pytest.approx(trace[k - 1][2], rel=0.01), (k, st["hpwl"], trace[k - 1])
    e.close()


@pytest.mark.parametrize("precision", [placer.PREC_MIXED, placer.PREC_FP64])
def test_qp_then_mgp_flow_matches_reference(precision):
    ref = _ref("stdcell_200k_qp_mgp")
    e = placer.Engine(bench.netlist(), placer.default_params(target_density=1.0, precision=precision))
    qp = e.quadratic_placement()
    assert qp["hpwl"] == pytest.approx(ref["qp_hpwl"], rel=0.02)
    e.initialize()
    st = e.nesterov_run()
    assert st["overflow"] < 0.1
    assert abs(st["iterations"] - ref["iterations"]) <= 0.1 * ref["iterations"], (st, ref)
    assert st["hpwl"] == pytest.approx(ref["hpwl"], rel=0.01)
    e.close()
