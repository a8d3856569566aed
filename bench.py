#!/usr/bin/env python3
"""Benchmark: seconds for the ePlace mGP stage to reach overflow <= 0.1 on a
200k-cell synthetic standard-cell design (220k nets, 2k I/O pads, 512x512
bins, targetDensity 1.0), on one B200 per rank.

A "step" is one whole mGP solve from the same start: load the start
positions (device-resident snapshot), the first gradient evaluation and
lambda_0 (initialization tail), then the Nesterov loop until overflow < 0.1.

  value  device time of one solve (CUDA events on the engine's stream, L2
         flushed before every step by a 256 MiB write), max over ranks
  e2e    the same solve through the C-ABI with pinned HOST buffers: start
         positions copied in and final positions copied out inside the
         timed region
  roofline  the dominant kernel group, timed alone with CUDA events by
         ep_time_kernels, against MEASURED_PEAKS.json
  cpu_baseline / --impl reference  the reference's own CPU implementation
         (oracle/_ref, compiled from the reference sources; single-threaded
         by construction) timed on a bounded sample of optimizer steps and
         scaled by the reference's iteration count on this design

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s to overflow≤0.1, 200k cells: learned+mixed vs plain GPU, HPWL within 0.5%"
DESIGN = dict(cells=200_000, seed=7, start_seed=3, start_sigma=0.05)
REF_RUNS = os.path.join(ROOT, "tests", "golden", "reference_runs.json")
SAMPLE_ITERS = 8  # reference optimizer steps per CPU sample


def netlist():
    """The 200k-cell standard-cell design: every cell on a net, pads attached
    near their cluster (synth.standard_cell's every_cell_pinned / local_pads)."""
    from eplace_b200 import synth
    return synth.standard_cell(DESIGN["cells"], seed=DESIGN["seed"], every_cell_pinned=True, local_pads=True)


def design():
    """The same design started from a seeded blob at the core centre."""
    from eplace_b200 import synth
    return synth.blob_start(netlist(), seed=DESIGN["start_seed"], sigma_frac=DESIGN["start_sigma"])


def workload_config(nl, extra=None):
    c = dict(workload="stdcell_200k_mgp_to_overflow_0.1", cells=nl.num_nodes, nets=nl.num_nets,
             pins=nl.num_pins, pads=nl.num_terminals, bins="512x512 (reference rule)",
             target_density=1.0, target_overflow=0.1,
             start=f"all cells at the die centre + N(0, {DESIGN['start_sigma']} die) jitter, seed {DESIGN['start_seed']}",
             generator=f"synth.standard_cell(seed={DESIGN['seed']}): lognormal widths mean 3, power-law degree mean 3.6 (alpha fitted), Rent p=0.6",
             l2="flushed before every timed step (256 MiB write)")
    if extra:
        c.update(extra)
    return c


def reference_iterations():
    with open(REF_RUNS) as f:
        return json.load(f)["stdcell_200k_blob_mgp"]["iterations"]


def cpu_sample(warmup, steps, iters_per_step=SAMPLE_ITERS):
    """Time the reference's optimizer loop on the bench design (rank 0 only).
    Returns (seconds per step of the metric, list of per-iteration seconds, info)."""
    from oracle import refharness as R
    nl = design()
    ref = R.RefPlacer(nl)
    ref.initialization(1.0)
    ref.opt_begin()
    per_iter = []
    for k in range(warmup + steps):
        tt = []
        for _ in range(iters_per_step):
            stopped, dt = ref.opt_step()
            if stopped:
                break
            tt.append(dt)
        if k >= warmup and tt:
            per_iter.append(sum(tt) / len(tt))
    ref.close()
    return per_iter


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return dict(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=max(mx) if mx else None,
                    reasons=reasons, samples=len(rows))


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def ncu_traffic():
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def group_rate(t, hbm, tf):
    """(achieved, fraction of peak) of one kernel group: FLOP/s against the
    bf16 tensor peak when it has flops, else bytes/s against HBM."""
    if t["flops"] > 0:
        a = t["flops"] / (t["ms"] * 1e-3) / 1e12
        return a, a / tf
    a = t["bytes"] / (t["ms"] * 1e-3) / 1e9
    return a, a / hbm


def roofline(times, iterations):
    """Dominant kernel group by time per iteration; its achieved rate vs peak."""
    hbm, tf, src = peaks()
    dom = max(times, key=lambda t: t["ms"])
    traffic = ncu_traffic().get(dom["name"])
    if dom["flops"] > 0:
        ach = dom["flops"] / (dom["ms"] * 1e-3) / 1e12
        r = dict(bound="tensor", achieved=ach, peak=tf, unit="TFLOP/s", frac=ach / tf)
    else:
        ach = dom["bytes"] / (dom["ms"] * 1e-3) / 1e9
        r = dict(bound="hbm", achieved=ach, peak=hbm, unit="GB/s", frac=ach / hbm)
    r.update(kernel=dom["name"], ms_per_launch=dom["ms"], traffic=traffic, peak_source=src,
             groups={t["name"]: round(t["ms"] * 1e3, 2) for t in times},
             group_frac={t["name"]: round(group_rate(t, hbm, tf)[1], 4) for t in times if t["bytes"] or t["flops"]})
    return r


def max_over_ranks(dist, values, device):
    """Element-wise maximum of `values` over all ranks (each rank's device
    times; the job takes as long as its slowest replica).  `dist` is None for
    a single process."""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def run_reference(args, rank):
    if rank != 0:
        return 0
    from oracle import refharness as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libeplace_ref.so was not built"}))
        return 0
    nl = design()
    iters = reference_iterations()
    per_iter = cpu_sample(args.warmup, args.steps)
    s_per_iter = statistics.mean(per_iter)
    value = s_per_iter * iters
    sample = (f"{args.steps} samples of {SAMPLE_ITERS} EplaceNesterovOpt steps each (after {args.warmup} warm-up samples) "
              f"of the reference on the same design; value = mean s/step x {iters} reference steps to overflow<0.1")
    out = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
           "config": workload_config(nl, dict(reference_iterations=iters, s_per_iteration=s_per_iter)),
           "cpu_baseline": {"value": value, "unit": "s", "cores": 1, "kind": "reference", "sample": sample},
           "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--dct", default="auto", choices=["auto", "fp32", "bf16x3", "fft"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from eplace_b200 import placer
    nl = design()
    dct_mode = {"fp32": placer.DCT_FP32, "bf16x3": placer.DCT_BF16X3, "fft": placer.DCT_FFT}.get(args.dct, placer.DCT_AUTO)
    eng = placer.Engine(nl, placer.default_params(target_density=1.0, dct_mode=dct_mode, device=local))
    dct_mode = eng.info.dct_mode
    stream = torch.cuda.current_stream()
    eng.set_stream(stream.cuda_stream)
    eng.save_positions()
    n_obj = eng.info.num_objects
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def solve():
        eng.load_positions()
        eng.initialize()
        return eng.nesterov_run()

    # the clock sampler starts before the warm-up, so it is already reading
    # when the timed region begins (nvidia-smi takes a moment to start)
    sampler = ClockSampler(local)
    sampler.start()
    for _ in range(args.warmup):
        solve()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    times, runs = [], []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = solve()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
        runs.append(st)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    if dist:
        dist.barrier()
    ms = statistics.mean(times)
    launches = int(sum(r["kernel_launches"] for r in runs)) + args.steps * 0

    # end to end through the C-ABI with pinned host buffers
    host_in = torch.empty((n_obj, 2), dtype=torch.float32, pin_memory=True)
    host_out = torch.empty((n_obj, 2), dtype=torch.float32, pin_memory=True)
    eng.load_positions()
    host_in.numpy()[:] = eng.get_positions()
    e2e_times = []
    for k in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.set_positions_ptr(host_in.data_ptr(), n_obj)
        eng.initialize()
        eng.nesterov_run()
        eng.get_positions_ptr(host_out.data_ptr(), n_obj)
        t1 = time.perf_counter()
        if k >= args.warmup:
            e2e_times.append((t1 - t0) * 1e3)
    e2e_ms = statistics.mean(e2e_times)

    kt = eng.time_kernels(reps=20)
    ms, e2e_ms = max_over_ranks(dist, [ms, e2e_ms], "cuda")
    last = runs[-1]
    if rank == 0:
        out = {"metric": METRIC, "value": ms * 1e-3, "unit": "s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32", "data": "synthetic",
               "config": workload_config(nl, dict(
                   fillers=eng.info.num_fillers, parallelism=f"replicas x{world}" if world > 1 else "1 GPU",
                   dct={placer.DCT_BF16X3: "3xBF16 tcgen05 GEMMs, FP32 accumulate",
                        placer.DCT_FFT: "FP32 fast transforms (shared-memory FFTs)"}.get(dct_mode, "FP32 CUDA-core GEMMs"),
                   density="int64 fixed-point scatter", reductions="FP64")),
               "iterations": last["iterations"], "overflow": last["overflow"], "hpwl": last["hpwl"],
               "e2e": {"value": e2e_ms * 1e-3, "unit": "s", "h2d_bytes_per_step": 8 * n_obj,
                       "d2h_bytes_per_step": 8 * n_obj},
               "gpu_launches": launches,
               "roofline": roofline(kt, last["iterations"]),
               "clocks": clocks}
        if not args.no_cpu_baseline and world == 1:
            try:
                from oracle import refharness as R
                if R.available():
                    per_iter = cpu_sample(0, 1, SAMPLE_ITERS)
                    iters = reference_iterations()
                    v = statistics.mean(per_iter) * iters
                    out["cpu_baseline"] = {
                        "value": v, "unit": "s", "cores": 1, "kind": "reference",
                        "sample": f"{SAMPLE_ITERS} EplaceNesterovOpt steps of the reference (oracle/_ref) on the "
                                  f"same design after initialization(); mean s/step x {iters} reference steps"}
            except Exception as ex:  # the baseline is reported, never required
                out["cpu_baseline"] = {"value": None, "error": str(ex)[:200]}
        print(json.dumps(out))
    eng.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
