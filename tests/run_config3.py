"""Config 3 end to end, the ePlace-MS flow at full size (synth.config3 from
its seeded blob): the engine's mGP, the reference's SAMacroLegalizer on the
engine's result (compiled reference, child process: minutes of CPU), the
engine's FILLERONLY and cGP; prints one JSON line with each stage's
iterations, overflow, HPWL and seconds, the macro legality after mLG, and
the reference's own flow from tests/golden/config3_flow.json beside it.
TEST INFRASTRUCTURE (it runs the compiled reference); not part of the
pytest suite because the reference's legalizer alone takes minutes.

    python tests/run_config3.py
"""
import json
import os
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from eplace_b200 import legality, placer, synth  # noqa: E402
from tests import ref_stages  # noqa: E402


def main():
    with open(os.path.join(ROOT, "tests", "golden", "config3_flow.json")) as f:
        ref = json.load(f)
    out = {"reference": ref}
    t0 = time.time()
    nl = synth.blob_start(synth.config3())
    out["generate_s"] = time.time() - t0
    t0 = time.time()
    e = placer.Engine(nl, placer.default_params(target_density=1.0, bins_x=1024, bins_y=1024))
    out["create_s"] = time.time() - t0
    out["fillers"], out["bins"] = e.info.num_fillers, e.info.bins_x
    e.initialize()
    st = e.nesterov_run()
    out["mgp"] = {k: st[k] for k in ("iterations", "overflow", "hpwl", "seconds")}
    nn = nl.num_nodes
    xy = e.get_positions()
    with tempfile.TemporaryDirectory() as tmp:
        t0 = time.time()
        rc, res = ref_stages.run("config3", xy[:nn, 0], xy[:nn, 1], 1.0, ["mlg"], tmp)
        out["mlg_wall_s"] = time.time() - t0
    out["mlg_rc"] = rc
    if rc == 0:
        out["mlg_seconds"] = float(res["mlg_seconds"])
        out["mlg_hpwl"] = float(res["mlg_hpwl"])
        r = legality.check(nl, res["mlg_cx"], res["mlg_cy"], macros_only=True, macros_vs_fixed=False)
        out["mlg_legal"] = {k: r[k] for k in ("legal", "macros", "macro_overlap", "outside_core",
                                                "macro_fixed_overlap")}
        macro = np.asarray(nl.node_h) > 1.0
        e.switch_stage(placer.FILLERONLY)
        allp = e.get_positions()
        allp[:nn] = np.stack([res["mlg_cx"], res["mlg_cy"]], 1)
        e.set_positions(allp)
        st = e.nesterov_run()
        out["fo"] = {k: st[k] for k in ("iterations", "overflow", "hpwl", "seconds")}
        e.switch_stage(placer.CGP)
        before = e.get_positions()
        st = e.nesterov_run()
        out["cgp"] = {k: st[k] for k in ("iterations", "overflow", "hpwl", "seconds")}
        out["cgp_macros_fixed"] = bool(np.array_equal(e.get_positions()[:nn][macro], before[:nn][macro]))
    e.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
