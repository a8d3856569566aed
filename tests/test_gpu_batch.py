"""Many designs on one GPU: engines built on a pool of host threads
(placer.create_engines) are the engines built one after another -- after
ep_initialize and one ep_run_batch over all of them, every design's final
positions and run statistics agree bit for bit."""
import numpy as np
import pytest

from eplace_b200 import placer, synth

pytestmark = pytest.mark.gpu


def test_pooled_construction_equals_sequential():
    sizes = [2_000, 9_000, 3_500, 20_000, 5_000, 12_000, 2_500, 7_000]
    nls = [synth.blob_start(synth.standard_cell(n, seed=40 + i, every_cell_pinned=True, local_pads=True))
           for i, n in enumerate(sizes)]
    out = []
    for threads in (1, 8):
        params = [placer.default_params(target_density=1.0) for _ in nls]
        engines = placer.create_engines(nls, params, threads=threads)
        for e in engines:
            e.initialize()
        stats = placer.run_batch(engines)
        out.append(([e.get_positions() for e in engines], stats))
        for e in engines:
            e.close()
    for a, b in zip(out[0][0], out[1][0]):
        assert np.array_equal(a, b)
    for a, b in zip(out[0][1], out[1][1]):
        assert a["iterations"] == b["iterations"] and a["hpwl"] == b["hpwl"]
        assert a["overflow"] < 0.1
