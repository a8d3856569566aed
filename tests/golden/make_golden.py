"""Generate the golden fixtures of tests/golden/ from the REFERENCE itself.

Runs where the reference sources are (their directory in the environment
variable EPLACE_REF_SRC) with the harness library oracle/_ref/libeplace_ref.so
built by `make -C oracle`.  For each
design it records, at full float precision, what the unmodified reference
computes on the same netlist and starting positions:

  * initialization(): filler count / size, bin grid, every bin map
    (node, filler, terminal, base density, E_x, E_y, phi), density /
    wirelength / total gradients, tau, 1/gamma, HPWL and lambda_0;
  * a second totalGradientUpdate with lambda_0 (the preconditioned direction);
  * the first optimizer steps (positions, tau, lambda after each);
  * the whole mGP run (iterations, final tau, HPWL);
  * variants.npz: the LSE and BB options and the mixed-size stage sequence
    (record_variants);
  * flows.npz: the CPU stages around global placement, the macro legalizer
    between mGP and cGP and Abacus + detailed placement on config 1
    (record_flows);
  * reference_runs.json (--bench): the whole runs on bench.py's design.

    python tests/golden/make_golden.py [--variants-only] [--bench] [--config3]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from eplace_b200 import bookshelf, synth  # noqa: E402
from oracle import refharness as R  # noqa: E402

REF_SRC = os.environ.get("EPLACE_REF_SRC", "")
REF_SMOKE = os.path.join(REF_SRC, "examples", "smoke", "smoke.aux")
TRAJ_STEPS = 5
C1_SEEDS = (1, 2, 4)


def designs():
    # the reference's own example, started from the reference's QP like its flow
    yield "ref_smoke", bookshelf.read_aux(REF_SMOKE, target_density=0.8), True
    yield "stdcell_2k", synth.blob_start(synth.standard_cell(2000, seed=3)), False
    yield "mixed_5k", synth.blob_start(synth.mixed_size(5000, 6, 3, seed=5)), False


def netlist_arrays(nl):
    keys = ("node_w", "node_h", "node_cx", "node_cy", "term_llx", "term_lly", "term_w", "term_h",
            "term_is_ni", "net_start", "pin_owner", "pin_dx", "pin_dy", "row_llx", "row_lly",
            "row_urx", "row_h", "row_site_w")
    return {"nl_" + k: getattr(nl, k) for k in keys}


def record(name, nl, use_qp):
    ref = R.RefPlacer(nl)
    if use_qp:
        ref.qp()
        cx, cy = ref.node_centers()
        nl = nl.with_positions(cx, cy)
    out = dict(netlist_arrays(nl))
    out["target_density"] = np.float32(nl.target_density)
    out["node_is_macro"] = ref.node_is_macro()
    ref.initialization(nl.target_density)
    info = ref.info()
    for k, v in info.items():
        out["info_" + k] = np.float64(v)
    cx, cy = ref.positions()
    out["init_cx"], out["init_cy"] = cx, cy
    maps = ref.bins()
    for k, v in maps.items():
        out["init_" + k] = v
    wl, dens, tot = ref.gradients()
    out["init_grad_wl"], out["init_grad_density"], out["init_grad_total"] = wl, dens, tot
    # second evaluation at the same positions, now with lambda_0
    ref.total_gradient_update()
    wl2, dens2, tot2 = ref.gradients()
    out["eval2_grad_total"] = tot2
    out["eval2_lambda"] = np.float64(ref.info()["lambda"])
    # optimizer: first steps, then the rest of the stage
    ref.opt_begin()
    tcx, tcy, tlam, ttau, thp = [], [], [], [], []
    for _ in range(TRAJ_STEPS):
        stopped, _ = ref.opt_step()
        if stopped:
            break
        x, y = ref.positions()
        i = ref.info()
        tcx.append(x)
        tcy.append(y)
        tlam.append(i["lambda"])
        ttau.append(i["overflow"])
        thp.append(i["last_hpwl"])
    out["traj_cx"], out["traj_cy"] = np.array(tcx), np.array(tcy)
    out["traj_lambda"], out["traj_tau"], out["traj_hpwl"] = np.array(tlam), np.array(ttau), np.array(thp)
    while True:
        stopped, _ = ref.opt_step()
        if stopped:
            break
    ref.opt_end()
    i = ref.info()
    out["run_iterations"] = np.int64(i["iter_count"])
    out["run_overflow"] = np.float64(i["overflow"])
    out["run_hpwl"] = np.float64(ref.hpwl())
    out["run_lambda"] = np.float64(i["lambda"])
    fx, fy = ref.positions()
    out["run_cx"], out["run_cy"] = fx, fy
    ref.close()
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: {i['num_nodes']:.0f} nodes, {i['num_fillers']:.0f} fillers, bins {i['bins_x']:.0f}, "
          f"{int(out['run_iterations'])} iterations, tau {float(out['run_overflow']):.6f}, "
          f"HPWL {float(out['run_hpwl']):.3f} -> {os.path.getsize(path) // 1024} KB")


def check_reader():
    """The array netlist read by eplace_b200.bookshelf drives the reference to
    the same state as the reference's own Bookshelf parser."""
    a = R.RefPlacer(aux=REF_SMOKE)
    b = R.RefPlacer(bookshelf.read_aux(REF_SMOKE, target_density=0.8))
    for p in (a, b):
        p.qp()
        p.initialization(0.8)
    ia, ib = a.info(), b.info()
    assert ia["num_fillers"] == ib["num_fillers"] and ia["last_hpwl"] == ib["last_hpwl"], (ia, ib)
    assert np.array_equal(a.gradients()[2], b.gradients()[2])


def run_stage(ref):
    """One EplaceNesterovOpt::opt of the current stage; returns its summary."""
    ref.opt_run()
    i = ref.info()
    x, y = ref.positions()
    return dict(iterations=np.int64(i["iter_count"]), overflow=np.float64(i["overflow"]),
                hpwl=np.float64(ref.hpwl()), lam=np.float64(i["lambda"]), cx=x, cy=y)


def record_variants():
    """Reference runs under the non-default options and the later stages:
      * gArg "LSE": the wirelength gradient at the initial positions and the
        whole mGP run with the log-sum-exp model (EPlace/eplace.cpp:512-549);
      * gArg "bb": the whole mGP run with the Barzilai-Borwein step
        (Optimization/nesterov.hpp:231-302);
      * gArg "bktrk": the whole mGP run with the backtracking step
        (Optimization/nesterov.hpp:310-369);
      * mixed-size stages: mGP, switch2FillerOnly (the reference re-draws the
        fillers with rand(); their new centres are recorded), 20 FILLERONLY
        steps, switch2cGP and the cGP run (EPlace/eplace.cpp:887-904);
      * quadratic placement (QPPlacer::quadraticPlacement,
        QPlace/qplace.cpp:20-106): the node centres it produces.
    Written to variants.npz."""
    out = {}
    nl = synth.blob_start(synth.standard_cell(2000, seed=3))
    for flag in ("LSE", "bb", "bktrk"):
        R.set_flag(flag)
        try:
            ref = R.RefPlacer(nl)
            ref.initialization(nl.target_density)
            if flag == "LSE":
                out["lse_init_grad_wl"] = ref.gradients()[0]
            s = run_stage(ref)
            for k in ("iterations", "overflow", "hpwl", "lam"):
                out[f"{flag.lower()}_run_{k}"] = s[k]
            ref.close()
        finally:
            R.clear_flag(flag)
    mx = synth.blob_start(synth.mixed_size(5000, 6, 3, seed=5))
    ref = R.RefPlacer(mx)
    ref.initialization(mx.target_density)
    cx, cy = ref.positions()
    out["stage_init_cx"], out["stage_init_cy"] = cx, cy
    mgp = run_stage(ref)
    out["stage_mgp_iterations"], out["stage_mgp_lambda"] = mgp["iterations"], mgp["lam"]
    ref.switch_filler_only()
    x, y = ref.positions()
    out["stage_fo_start_cx"], out["stage_fo_start_cy"] = x, y
    fo = run_stage(ref)
    for k in ("iterations", "overflow", "hpwl", "lam", "cx", "cy"):
        out["stage_fo_" + k] = fo[k]
    ref.switch_cgp()
    out["stage_cgp_start_lambda"] = np.float64(ref.info()["lambda"])
    cg = run_stage(ref)
    for k in ("iterations", "overflow", "hpwl", "lam", "cx", "cy"):
        out["stage_cgp_" + k] = cg[k]
    ref.close()
    # quadratic placement (QPPlacer::quadraticPlacement) from the netlist alone
    for name, d in (("stdcell_2k", nl), ("mixed_5k", mx)):
        ref = R.RefPlacer(d)
        t = ref.qp()
        cx, cy = ref.node_centers()
        out[f"qp_{name}_cx"], out[f"qp_{name}_cy"] = cx, cy
        out[f"qp_{name}_hpwl"] = np.float64(ref.hpwl())
        out[f"qp_{name}_seconds"] = np.float64(t)
        ref.close()
    path = os.path.join(HERE, "variants.npz")
    np.savez_compressed(path, **out)
    print("variants:", {k: (v if np.ndim(v) == 0 else np.shape(v)) for k, v in out.items()})


def record_flows():
    """The reference's CPU stages around global placement, on designs the
    GPU flow tests rerun with the engine in place of its global placement:
      * mlg_*: mixed_5k from its recorded start: initialization, mGP, the SA
        macro legalizer (SAMacroLegalizer), FILLERONLY and cGP, as
        main/ePlace_main.cpp:174-211 runs them (node centres after mGP and
        after mLG, HPWL after each stage, the cGP outcome);
      * c1_<seed>_*: config 1 (synth.smoke) from the netlist: QPPlacer,
        initialization, mGP, AbacusLegalizer, DetailedPlacer
        (main/ePlace_main.cpp:248-279): every object's centre after
        initialization (the QP result and the reference's fillers), HPWL
        and iterations after GP, HPWL after legalization and detailed
        placement, and the final centres.  The reference's
        DetailedPlacer ends the process with a segmentation fault on smoke
        seeds 3 and 7 (after its own QP, mGP and Abacus); C1_SEEDS leaves
        them out.
    Written to flows.npz."""
    out = {}
    g = np.load(os.path.join(HERE, "mixed_5k.npz"))
    mx = synth.blob_start(synth.mixed_size(5000, 6, 3, seed=5))
    assert np.array_equal(np.asarray(g["nl_node_w"]), mx.node_w)
    ref = R.RefPlacer(mx)
    ref.initialization(mx.target_density)
    ref.opt_run()
    cx, cy = ref.node_centers()
    out["mlg_mgp_cx"], out["mlg_mgp_cy"], out["mlg_mgp_hpwl"] = cx, cy, np.float64(ref.hpwl())
    out["mlg_seconds"] = np.float64(ref.macro_legalize(mx.target_density))
    cx, cy = ref.node_centers()
    out["mlg_cx"], out["mlg_cy"], out["mlg_hpwl"] = cx, cy, np.float64(ref.hpwl())
    ref.switch_filler_only()
    fo = run_stage(ref)
    ref.switch_cgp()
    cg = run_stage(ref)
    out["mlg_fo_hpwl"] = fo["hpwl"]
    for k in ("iterations", "overflow", "hpwl"):
        out["mlg_cgp_" + k] = cg[k]
    out["mlg_cgp_cx"], out["mlg_cgp_cy"] = ref.node_centers()
    ref.close()
    for seed in C1_SEEDS:
        nl = synth.smoke(seed)
        ref = R.RefPlacer(nl)
        ref.qp()
        ref.initialization(nl.target_density)
        k = f"c1_{seed}_"
        out[k + "init_cx"], out[k + "init_cy"] = ref.positions()  # QP result and the fillers
        ref.opt_run()
        out[k + "gp_hpwl"] = np.float64(ref.hpwl())
        out[k + "gp_iterations"] = np.int64(ref.info()["iter_count"])
        out[k + "gp_overflow"] = np.float64(ref.info()["overflow"])
        ref.abacus()
        out[k + "lg_hpwl"] = np.float64(ref.hpwl())
        ref.detailed()
        out[k + "dp_hpwl"] = np.float64(ref.hpwl())
        out[k + "cx"], out[k + "cy"] = ref.node_centers()
        ref.close()
    path = os.path.join(HERE, "flows.npz")
    np.savez_compressed(path, **out)
    print("flows:", {k: (float(v) if np.ndim(v) == 0 else np.shape(v)) for k, v in out.items()})


def record_config3():
    """The reference's mixed-size flow on config 3 (synth.config3: 1M cells,
    300 movable + 50 fixed macros, 1024 x 1024 bins) from a seeded blob
    start: initialization, mGP, SAMacroLegalizer, FILLERONLY, cGP
    (main/ePlace_main.cpp:174-211), with each stage's iterations, overflow,
    HPWL and seconds.  Half an hour of CPU; written to config3_flow.json."""
    import json
    import time
    nl = synth.blob_start(synth.config3())
    ref = R.RefPlacer(nl)
    out = {}
    t0 = time.time()
    ref.initialization(nl.target_density)
    out["init_seconds"] = time.time() - t0
    i = ref.info()
    out.update(fillers=int(i["num_fillers"]), bins=int(i["bins_x"]))
    for stage, run in (("mgp", None), ("mlg", None), ("fo", None), ("cgp", None)):
        t0 = time.time()
        if stage == "mlg":
            ref.macro_legalize(nl.target_density)
            out["mlg_seconds"] = time.time() - t0
            out["mlg_hpwl"] = float(ref.hpwl())
            continue
        if stage == "fo":
            ref.switch_filler_only()
        elif stage == "cgp":
            ref.switch_cgp()
        r = run_stage(ref)
        out[stage] = dict(iterations=int(r["iterations"]), overflow=float(r["overflow"]), hpwl=float(r["hpwl"]),
                          seconds=time.time() - t0)
        print(stage, out[stage], flush=True)
    ref.close()
    out["note"] = "reference CPU path, 1 thread, from synth.blob_start(synth.config3())"
    with open(os.path.join(HERE, "config3_flow.json"), "w") as f:
        json.dump(out, f, indent=1)


def qp_with_trace(ref):
    """QPPlacer::quadraticPlacement with its per-round log line captured:
    [(round, max(xError, yError) as printed, HPWL after the round)]."""
    import ctypes
    import re
    import tempfile
    R.lib().ref_set_quiet(0)
    saved = os.dup(1)
    with tempfile.TemporaryFile() as tmp:
        sys.stdout.flush()
        os.dup2(tmp.fileno(), 1)
        try:
            ref.qp()
            ctypes.CDLL(None).fflush(None)
        finally:
            os.dup2(saved, 1)
            os.close(saved)
            R.lib().ref_set_quiet(1)
        tmp.seek(0)
        text = tmp.read().decode(errors="replace")
    rows = re.findall(r"at iteration number\s+(\d+),\s+CG Error ([-\d.e+]+),\s+HPWL ([\d.]+)", text)
    return [(int(a), float(b), float(c)) for a, b, c in rows]


def record_bench_reference():
    """The reference's whole runs on bench.py's 200k-cell design (a few
    minutes of CPU): from its own quadratic placement (QPPlacer, as its flow
    starts) and from bench.design()'s seeded blob; iterations to overflow
    < 0.1, final overflow and HPWL, and the stage times; for the quadratic
    placement also its per-round log (error as printed, HPWL)."""
    import json
    import time
    sys.path.insert(0, ROOT)
    import bench
    out = {}
    for key, nl, qp in (("stdcell_200k_qp_mgp", bench.netlist(), True),
                        ("stdcell_200k_blob_mgp", bench.design(), False)):
        ref = R.RefPlacer(nl)
        t_qp = 0.0
        rec = {}
        if qp:
            t0 = time.time()
            rec["qp_trace"] = qp_with_trace(ref)
            t_qp = time.time() - t0
            rec["qp_hpwl"] = float(ref.hpwl())
        t0 = time.time()
        ref.initialization(1.0)
        t_init = time.time() - t0
        t0 = time.time()
        ref.opt_run()
        t_mgp = time.time() - t0
        i = ref.info()
        rec.update(iterations=int(i["iter_count"]), overflow=float(i["overflow"]), hpwl=float(ref.hpwl()),
                   fillers=int(i["num_fillers"]), bins=int(i["bins_x"]), qp_seconds=t_qp, init_seconds=t_init,
                   mgp_seconds=t_mgp, note="reference CPU path, 1 thread")
        out[key] = rec
        ref.close()
        print(key, rec, flush=True)
    with open(os.path.join(HERE, "reference_runs.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    if not REF_SRC or not os.path.exists(REF_SMOKE) or not R.available():
        sys.exit("make_golden.py needs EPLACE_REF_SRC (the reference sources) and oracle/_ref built")
    if "--variants-only" not in sys.argv:
        check_reader()
        for name, nl, qp in designs():
            record(name, nl, qp)
    record_variants()
    record_flows()
    if "--bench" in sys.argv:
        record_bench_reference()
    if "--config3" in sys.argv:
        record_config3()
