"""The give-up paths of the engine's bounded waits and retries, made to run
out through ep_set_limits (no GPU fault, trap or hang is involved: a wait
that runs out of polls records EP_ERR_TIMEOUT in the device status, drains
the copies and MMAs its CTA started, frees its TMEM and returns).

  * tensor-core Poisson GEMMs with zero pipeline polls: the evaluation and a
    captured optimizer run end with EP_ERR_TIMEOUT; with the default limit
    restored the same engine evaluates the field within 1e-4 of the FP64
    oracle and runs to overflow < 0.1;
  * backtracking steps that can accept no trial: the run ends with
    EP_ERR_TIMEOUT after the trial cap; with the defaults restored the engine
    takes its steps again.
"""
import numpy as np
import pytest

from eplace_b200 import placer, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DEFAULT_POLLS = 1 << 22


def _field_error(e):
    m = e.bin_maps()
    i = e.info
    bin_area = np.float64(np.float32(i.bin_step_x) * np.float32(i.bin_step_y))
    rho = (m["node"].astype(np.float64) + m["base"] + m["filler"] + m["terminal"]) / bin_area
    ex, ey, _ = O.poisson(rho, i.bin_step_x, i.bin_step_y)
    scale = max(np.abs(ex).max(), np.abs(ey).max())
    return max(np.abs(m["ex"] - ex).max(), np.abs(m["ey"] - ey).max()) / scale


def test_tensor_core_wait_gives_up_and_the_engine_recovers():
    nl = synth.blob_start(synth.standard_cell(20_000, seed=5), sigma_frac=0.15)
    e = placer.Engine(nl, placer.default_params(target_density=1.0, bins_x=256, bins_y=256,
                                                dct_mode=placer.DCT_BF16X3, keep_maps=1))
    assert e.limits()["wait_polls"] == DEFAULT_POLLS
    e.set_limits(wait_polls=0)
    with pytest.raises(placer.EPError) as ex:
        e.eval_gradient()
    assert ex.value.status == placer.EP_ERR_TIMEOUT
    e.set_limits(wait_polls=DEFAULT_POLLS)
    e.initialize()
    assert _field_error(e) < 1e-4
    e.close()


def test_tensor_core_wait_gives_up_inside_a_captured_run():
    nl = synth.blob_start(synth.standard_cell(20_000, seed=5), sigma_frac=0.15)
    e = placer.Engine(nl, placer.default_params(target_density=1.0, bins_x=128, bins_y=128,
                                                dct_mode=placer.DCT_BF16X3))
    e.save_positions()
    e.initialize()
    e.set_limits(wait_polls=0)
    with pytest.raises(placer.EPError) as ex:
        e.nesterov_run()
    assert ex.value.status == placer.EP_ERR_TIMEOUT
    e.set_limits(wait_polls=DEFAULT_POLLS)
    e.load_positions()
    e.initialize()
    st = e.nesterov_run()
    assert st["overflow"] < 0.1
    e.close()


def test_backtracking_trial_cap_ends_the_run():
    nl = synth.blob_start(synth.standard_cell(2_000, seed=3))
    e = placer.Engine(nl, placer.default_params(target_density=1.0, step_rule=placer.STEP_BKTRK))
    e.save_positions()
    e.initialize()
    e.set_limits(bktrk_trials=3, bktrk_accept=1e30)  # no trial can be accepted
    with pytest.raises(placer.EPError) as ex:
        e.nesterov_run()
    assert ex.value.status == placer.EP_ERR_TIMEOUT
    e.set_limits(bktrk_trials=64, bktrk_accept=0.95)
    e.load_positions()
    e.initialize()
    st = e.nesterov_run(max_steps=6)
    assert st["iterations"] == 6 and np.isfinite(st["hpwl"])
    e.close()


def test_limits_reject_bad_values():
    nl = synth.blob_start(synth.standard_cell(2_000, seed=3))
    e = placer.Engine(nl, placer.default_params(target_density=1.0))
    for kw in (dict(bktrk_trials=0), dict(bktrk_accept=0.0)):
        with pytest.raises(placer.EPError) as ex:
            e.set_limits(**kw)
        assert ex.value.status == placer.EP_ERR_ARG
    e.close()
