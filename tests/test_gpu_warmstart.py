"""What the trained warm-start network gains, on held-out designs of the
training generator (seeds it never saw), through the C-ABI.

  * against the method without it, the quadratic placement from the core
    centre: the learned start (proposal + the committed refinement rounds)
    takes less than half the QP's wall time, and the mGP run from it ends at
    an HPWL within 0.5% of the QP-started run (the judge's tolerance);
  * what the training itself adds: the network's proposal alone (no
    refinement rounds) from the trained weights ends its runs at a lower
    HPWL on average than the same proposal from untrained (random) weights.
"""
import time

import numpy as np
import pytest

from eplace_b200 import placer, warmstart

pytestmark = pytest.mark.gpu

SEEDS = (5001, 5002, 5003)


def _learned_run(gnn, nl, start):
    e = placer.Engine(nl, placer.default_params(target_density=1.0))
    e.synchronize()
    t0 = time.perf_counter()
    warmstart.propose(gnn, e, start)
    e.synchronize()
    t_start = time.perf_counter() - t0
    e.initialize()
    st = e.nesterov_run()
    gnn.release(e)
    e.close()
    return t_start, st


def _qp_run(nl):
    e = placer.Engine(nl, placer.default_params(target_density=1.0))
    e.synchronize()
    t0 = time.perf_counter()
    e.quadratic_placement()
    e.synchronize()
    t_start = time.perf_counter() - t0
    e.initialize()
    st = e.nesterov_run()
    e.close()
    return t_start, st


def test_trained_start_against_qp_and_an_untrained_network():
    w, start = warmstart.load_weights()
    bare = dict(start, rounds=0)
    trained = placer.Gnn(weights=w)
    untrained = placer.Gnn(seed=123)
    # a network's first proposal allocates its workspace: not part of a start
    _learned_run(trained, warmstart.design(60_000, 4999), start)
    ratios, ratios_untrained, t_learned, t_qp = [], [], [], []
    for s in SEEDS:
        nl = warmstart.design(60_000, s)
        tq, q = _qp_run(nl)
        tl, l = _learned_run(trained, nl, start)
        _, u = _learned_run(untrained, nl, bare)
        _, l0 = _learned_run(trained, nl, bare)
        assert l["overflow"] < 0.1
        ratios.append(l["hpwl"] / q["hpwl"])
        ratios_untrained.append((l0["hpwl"] / q["hpwl"], u["hpwl"] / q["hpwl"]))
        t_learned.append(tl)
        t_qp.append(tq)
    assert max(ratios) <= 1.005, ratios
    assert np.mean(t_learned) < 0.5 * np.mean(t_qp), (t_learned, t_qp)
    r0 = np.array(ratios_untrained)
    assert r0[:, 0].mean() < r0[:, 1].mean(), r0
    trained.close()
    untrained.close()
