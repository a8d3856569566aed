"""Run the reference's CPU stages around global placement (through the
compiled reference, oracle/_ref) on given node centres, in a process of its
own: the reference's DetailedPlacer ends its process with a segmentation
fault on some inputs, and a child process keeps that from ending the test
run.  TEST INFRASTRUCTURE ONLY.

    python tests/ref_stages.py <design> <in.npz> <out.npz> <stage> [<stage> ...]

design: smoke:<seed> (synth.smoke), mixed_5k (the golden mixed-size
design) or config3 (synth.config3 from its seeded blob); in.npz holds cx, cy (movable-node centres) and target_density;
stages, in order: mlg (SAMacroLegalizer), abacus (AbacusLegalizer),
detailed (DetailedPlacer).  out.npz gets <stage>_cx, <stage>_cy,
<stage>_hpwl and <stage>_seconds after each stage.
"""
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def design(name):
    sys.path.insert(0, ROOT)
    from eplace_b200 import synth
    if name.startswith("smoke:"):
        return synth.smoke(int(name.split(":")[1]))
    if name == "mixed_5k":
        return synth.blob_start(synth.mixed_size(5000, 6, 3, seed=5))
    if name == "config3":
        return synth.blob_start(synth.config3())
    raise ValueError(name)


def run(design_name, cx, cy, target_density, stages, tmpdir):
    """Run the stages in a child process; returns (returncode, results)."""
    src = os.path.join(tmpdir, "stages_in.npz")
    dst = os.path.join(tmpdir, "stages_out.npz")
    np.savez(src, cx=np.asarray(cx, np.float32), cy=np.asarray(cy, np.float32),
             target_density=np.float32(target_density))
    r = subprocess.run([sys.executable, os.path.abspath(__file__), design_name, src, dst, *stages],
                       cwd=ROOT, capture_output=True, text=True, timeout=1800)
    out = dict(np.load(dst)) if r.returncode == 0 and os.path.exists(dst) else {}
    return r.returncode, out


def main():
    name, src, dst, *stages = sys.argv[1:]
    sys.path.insert(0, ROOT)
    from oracle import refharness as R
    nl = design(name)
    z = np.load(src)
    ref = R.RefPlacer(nl)
    ref.set_node_centers(z["cx"], z["cy"])
    out = {}
    for st in stages:
        if st == "mlg":
            t = ref.macro_legalize(float(z["target_density"]))
        elif st == "abacus":
            t = ref.abacus()
        elif st == "detailed":
            t = ref.detailed()
        else:
            raise ValueError(st)
        cx, cy = ref.node_centers()
        out[st + "_cx"], out[st + "_cy"] = cx, cy
        out[st + "_hpwl"] = np.float64(ref.hpwl())
        out[st + "_seconds"] = np.float64(t)
    ref.close()
    np.savez(dst, **out)


if __name__ == "__main__":
    main()
