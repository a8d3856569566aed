"""Checkpoint and resume of the optimizer (ep_save_state / ep_load_state)
through the C-ABI: a run saved between steps and resumed on a fresh engine
takes the same steps bit for bit as the uninterrupted run, in both
precisions and with the backtracking step; blobs of another design or of
another size are refused, and loading before ep_initialize is an error.
The reference saves positions only (PlaceDB::saveNodesLocation,
PlaceDB/placedb.cpp:1441-1465)."""
import numpy as np
import pytest

from eplace_b200 import placer, synth

pytestmark = pytest.mark.gpu


def _engine(nl, **kw):
    return placer.Engine(nl, placer.default_params(target_density=1.0, **kw))


def _steps(e, n):
    for _ in range(n):
        e.nesterov_step()


@pytest.mark.parametrize("kw", [dict(), dict(precision=placer.PREC_FP64), dict(step_rule=placer.STEP_BKTRK)])
def test_resumed_run_equals_uninterrupted_run(kw):
    nl = synth.blob_start(synth.standard_cell(8_000, seed=21, every_cell_pinned=True, local_pads=True))
    a = _engine(nl, **kw)
    a.initialize()
    a.nesterov_begin()
    _steps(a, 30)
    b = _engine(nl, **kw)
    b.initialize()
    b.nesterov_begin()
    _steps(b, 15)
    blob_mid = b.save_state()
    b.close()
    c = _engine(nl, **kw)
    c.initialize()
    c.load_state(blob_mid)
    _steps(c, 15)
    assert a.query() == c.query()
    assert np.array_equal(a.get_positions_f64(), c.get_positions_f64())
    # every vector of the state (y, x, g, y_prev, g_prev) agrees
    n = 5 * a.info.num_objects * (16 if kw.get("precision") == placer.PREC_FP64 else 8)
    assert a.save_state()[-n:] == c.save_state()[-n:]
    a.nesterov_end()
    c.nesterov_end()
    assert np.array_equal(a.get_positions_f64(), c.get_positions_f64())
    a.close()
    c.close()


def test_state_blobs_are_checked():
    nl = synth.blob_start(synth.standard_cell(3_000, seed=4))
    other = synth.blob_start(synth.standard_cell(3_100, seed=4))
    a = _engine(nl)
    a.initialize()
    blob = a.save_state()
    fresh = _engine(nl)
    with pytest.raises(placer.EPError) as ex:
        fresh.load_state(blob)  # before ep_initialize
    assert ex.value.status == placer.EP_ERR_STATE
    fresh.initialize()
    fresh.load_state(blob)
    with pytest.raises(placer.EPError) as ex:
        fresh.load_state(blob[:-8])
    assert ex.value.status == placer.EP_ERR_ARG
    b = _engine(other)
    b.initialize()
    with pytest.raises(placer.EPError) as ex:
        b.load_state(blob)
    assert ex.value.status == placer.EP_ERR_ARG
    for e in (a, fresh, b):
        e.close()
