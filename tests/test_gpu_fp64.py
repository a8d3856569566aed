"""The plain FP64 form of the loop (ep_params.precision = EP_PREC_FP64)
against the FP64 oracle and the reference's golden runs, through the C-ABI.

Tolerances (stated per check):
  * Poisson field and potential: 1e-11 of max|E| (max|phi|) against the FP64
    oracle, on the engine's own density read back exactly from its
    fixed-point maps (the FP64 rounding of the fast transforms);
  * on a design whose geometry is exact in float (sizes, pin offsets and
    centres on a 1/64 grid, bin steps powers of two), where the reference's
    float rectangles and pin positions lose nothing: cell node map 1e-11,
    cell density gradient 1e-10, WA gradient and HPWL 1e-9 (the engine's
    weighted-mean form of the gradient against the oracle's expanded
    quotient) with the exact exp and with fastExp;
  * whole mGP run on the golden designs: tau below target, iterations within
    10% and HPWL within 1% of the reference's run from the same start;
  * the FP64 and FP32 forms on one design: HPWL within 0.5%, iterations
    within 5%;
  * quadratic placement (FP32 in both forms): the FP64 engine's result equals
    the FP32 engine's bit for bit.
"""
import copy

import numpy as np
import pytest

from eplace_b200 import placer, synth
from oracle import oracle as O
from tests.helpers import DESIGNS, OracleDesign, golden_netlist, load_golden, rel_err

pytestmark = pytest.mark.gpu


def _q64(a):
    return (np.round(np.asarray(a, np.float64) * 64.0) / 64.0).astype(np.float32)


def dyadic_design(n=3000, seed=2, side=128.0):
    nl = synth.standard_cell(n, seed=seed, every_cell_pinned=True, local_pads=True)
    d = copy.copy(nl)
    for k, v in synth._rows(side).items():
        setattr(d, k, v)
    tx, ty = synth._pad_ring(nl.num_terminals, side)
    d.term_llx, d.term_lly = _q64(tx), _q64(ty)
    d.pin_dx, d.pin_dy = _q64(nl.pin_dx), _q64(nl.pin_dy)
    rng = np.random.default_rng(seed)
    d.node_cx = _q64(side / 2 + rng.normal(0, 0.12 * side, n).clip(-0.4 * side, 0.4 * side))
    d.node_cy = _q64(side / 2 + rng.normal(0, 0.12 * side, n).clip(-0.4 * side, 0.4 * side))
    return d


def fp64_engine(nl, **kw):
    p = placer.default_params(target_density=float(nl.target_density), keep_maps=1, precision=placer.PREC_FP64)
    for k, v in kw.items():
        setattr(p, k, v)
    return placer.Engine(nl, p)


def engine_rho(e):
    """The engine's density, rebuilt exactly as its prep kernel forms it from
    the fixed-point maps and the static terminal / base maps."""
    i = e.info
    nq, fq = e.density_fixed()
    st = e.bin_maps(("terminal", "base"))
    inv_q = 1.0 / i.density_scale
    bin_area = np.float32(np.float32(i.bin_step_x) * np.float32(i.bin_step_y))
    inv_bin_area = np.float64(np.float32(1.0 / np.float64(bin_area)))
    node, fill = nq.astype(np.float64) * inv_q, fq.astype(np.float64) * inv_q
    return (((node + st["base"].astype(np.float64)) + fill) + st["terminal"].astype(np.float64)) * inv_bin_area


@pytest.mark.parametrize("bins", [(64, 64), (128, 32), (512, 512)])
def test_fp64_poisson_field_to_fp64_rounding(bins):
    nl = synth.blob_start(synth.standard_cell(20_000, seed=5), sigma_frac=0.15)
    e = fp64_engine(nl, bins_x=bins[0], bins_y=bins[1])
    assert e.info.precision == placer.PREC_FP64 and e.info.dct_mode == placer.DCT_FFT
    e.eval_gradient()
    ex, ey, phi = O.poisson(engine_rho(e), e.info.bin_step_x, e.info.bin_step_y)
    f = e.field_f64()
    scale = max(np.abs(ex).max(), np.abs(ey).max())
    assert max(np.abs(f["ex"] - ex).max(), np.abs(f["ey"] - ey).max()) < 1e-11 * scale
    assert rel_err(f["phi"], phi) < 1e-11
    e.close()


@pytest.mark.parametrize("exp_mode", [placer.EXP_EXACT, placer.EXP_FAST])
def test_fp64_gradients_exact_on_float_exact_geometry(exp_mode):
    nl = dyadic_design()
    e = fp64_engine(nl, bins_x=32, bins_y=32, exp_mode=exp_mode)
    i = e.info
    assert i.bin_step_x == 4.0 and i.bin_step_y == 4.0
    e.set_positions(_q64(e.get_positions()))
    e.eval_gradient()
    xy = e.get_positions_f64()
    assert np.array_equal(xy, _q64(xy))  # centres stayed on the grid
    n = nl.num_nodes
    d = OracleDesign(nl, np.zeros(n, np.uint8), i.num_fillers, i.filler_w, i.filler_h,
                     (i.core_llx, i.core_lly, i.core_urx, i.core_ury), (32, 32), (4.0, 4.0), 1.0)
    # cell density map: the oracle's float contributions are exact here
    cells = d.flags.copy()
    cells[n:] = O.FILLER
    nd, _, _, _ = O.scatter(d.grid, xy[:, 0], xy[:, 1], d.w, d.h, cells)
    nq, _ = e.density_fixed()
    assert rel_err(nq * (1.0 / i.density_scale), nd) < 1e-11
    # density gradient of the cells on the engine's own field
    f = e.field_f64()
    gd_ref = O.gather(d.grid, xy[:, 0], xy[:, 1], d.w, d.h, f["ex"], f["ey"])
    gd, gw = e.component_gradients_f64()
    assert rel_err(gd[:n], gd_ref[:n]) < 1e-10
    # WA gradient and HPWL at the engine's 1/gamma
    s = e.query()
    _, hp, gw_ref = O.wirelength_grad(d.nl_obj, xy[:, 0], xy[:, 1], d.tcx, d.tcy, s["inv_gamma_x"],
                                      s["inv_gamma_y"], exp_mode=exp_mode)
    assert rel_err(gw[:n], gw_ref[:n]) < 1e-9
    assert s["hpwl"] == pytest.approx(hp, rel=1e-9)
    e.close()


@pytest.fixture(scope="module", params=DESIGNS)
def golden(request):
    return request.param, load_golden(request.param)


def test_fp64_whole_mgp_run_outcome(golden):
    name, g = golden
    nl = golden_netlist(g)
    e = fp64_engine(nl, keep_maps=0)
    e.set_positions(np.stack([g["init_cx"], g["init_cy"]], 1))
    e.initialize()
    st = e.nesterov_run()
    it_ref = int(g["run_iterations"])
    assert st["overflow"] < 0.1
    assert abs(st["iterations"] - it_ref) <= max(2, 0.1 * it_ref), (st, it_ref)
    assert st["hpwl"] == pytest.approx(float(g["run_hpwl"]), rel=0.01)
    e.close()


def test_fp64_and_mixed_forms_agree_on_a_run():
    nl = synth.blob_start(synth.standard_cell(20_000, seed=6, every_cell_pinned=True, local_pads=True))
    out = {}
    for prec in (placer.PREC_MIXED, placer.PREC_FP64):
        e = placer.Engine(nl, placer.default_params(target_density=1.0, precision=prec))
        e.initialize()
        out[prec] = e.nesterov_run()
        e.close()
    a, b = out[placer.PREC_MIXED], out[placer.PREC_FP64]
    assert a["overflow"] < 0.1 and b["overflow"] < 0.1
    assert abs(a["iterations"] - b["iterations"]) <= max(2, 0.05 * b["iterations"]), (a, b)
    assert a["hpwl"] == pytest.approx(b["hpwl"], rel=0.005)


def test_fp64_quadratic_placement_equals_fp32():
    nl = synth.standard_cell(5_000, seed=3, every_cell_pinned=True, local_pads=True)
    res = []
    for prec in (placer.PREC_MIXED, placer.PREC_FP64):
        e = placer.Engine(nl, placer.default_params(target_density=1.0, precision=prec))
        st = e.quadratic_placement()
        res.append((st, e.get_positions_f64()))
        e.close()
    assert res[0][0]["hpwl"] == res[1][0]["hpwl"]
    assert np.array_equal(res[0][1], res[1][1])


def test_fp64_stepwise_equals_graph_loop_and_bktrk_runs():
    g = load_golden("stdcell_2k")
    nl = golden_netlist(g)
    start = np.stack([g["init_cx"], g["init_cy"]], 1)
    a = fp64_engine(nl, keep_maps=0)
    a.set_positions(start)
    a.initialize()
    ra = a.nesterov_run(max_steps=12)
    b = fp64_engine(nl, keep_maps=0)
    b.set_positions(start)
    b.initialize()
    b.nesterov_begin()
    for _ in range(12):
        b.nesterov_step()
    b.nesterov_end()
    assert ra["iterations"] == 12
    assert np.array_equal(a.get_positions_f64(), b.get_positions_f64())
    c = fp64_engine(nl, keep_maps=0, step_rule=placer.STEP_BKTRK)
    c.set_positions(start)
    c.initialize()
    rc = c.nesterov_run(max_steps=10)
    assert rc["iterations"] == 10 and np.isfinite(rc["hpwl"])
    for x in (a, b, c):
        x.close()


def test_fp64_refuses_dense_poisson_grids():
    nl = synth.standard_cell(2_000, seed=1)
    with pytest.raises(placer.EPError) as ex:
        fp64_engine(nl, bins_x=96, bins_y=96)
    assert ex.value.status == placer.EP_ERR_UNSUPPORTED
