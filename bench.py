#!/usr/bin/env python3
"""Benchmark of the metric: seconds until the ePlace mGP stage reaches
overflow <= 0.1 on a 200k-cell synthetic standard-cell design (220k nets,
2k I/O pads, 512x512 bins, targetDensity 1.0), learned warm start + mixed
precision against the plain FP64 form, HPWL within 0.5%; one B200 per rank.

A "step" is one placement of the design from its netlist, resident on the
device, to overflow < 0.1:
  learned+mixed (the product; `value`)  the network's proposal (graph,
         pad-anchored diffusion features, forward pass; ep_gnn_propose with
         the committed weights and alpha), the committed number of rounds of
         the quadratic model from it (ep_quadratic_refine), then mGP in the
         mixed-precision form;
  plain  the device quadratic placement (the reference flow's start, run
         for the reference's own number of rounds on this design, whose last
         round ends at its stopping test's threshold) then mGP with every
         vector, map and wirelength term in FP64.
Both are timed with CUDA events on the engines' stream around the whole
step (host work inside it shows as elapsed time), L2 flushed (256 MiB write)
before each; the line carries both arms, their HPWL ratio and the GP-only
times.

  e2e    the product step through the C-ABI from HOST arrays: ep_create
         (netlist upload, fillers, bins), proposal, initialize, mGP, final
         positions read back (pinned buffer); the plain arm's the same way
  roofline  the dominant kernel group of the mixed loop (ep_time_kernels,
         CUDA events) on the algorithmic bytes of the hot-path table (WA:
         12 P + 4 (nets + 1) + 16 cells), and the whole-iteration fraction
  cpu_baseline  the reference's own CPU flow (oracle/_ref, 1 thread): its
         quadratic placement and initialization in full, then a sample of
         its optimizer steps scaled by its iteration count on this design
  --impl reference  one complete run of the reference's CPU flow on the
         same design (QPPlacer::quadraticPlacement, EPlacer_2D::initialization,
         EplaceNesterovOpt::opt to overflow < 0.1), timed, not extrapolated

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
SAMPLE_ITERS = 8  # reference optimizer steps of the cpu_baseline sample
# kernels one ep_gnn_propose launches on a netlist it has not bound: the
# features (initial values, terminal pin counts and feature, 1/degree, the
# aggregation indices, 128 diffusion steps of 2 kernels, 3 feature stores),
# the forward pass (input layer, 3 x (net mean, node mean, dense), output),
# the proposal and the position store
GNN_LAUNCHES = 5 + 2 * 128 + 3 + 1 + 3 * 3 + 1 + 2


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
    c = dict(workload="stdcell_200k_place_to_overflow_0.1", cells=nl.num_nodes, nets=nl.num_nets,
             pins=nl.num_pins, pads=nl.num_terminals, bins="512x512 (reference rule)",
             target_density=1.0, target_overflow=0.1,
             generator=(f"synth.standard_cell(200000, seed={DESIGN['seed']}, every_cell_pinned=True, "
                        "local_pads=True): lognormal widths mean 3, power-law degree mean 3.6 (alpha fitted), "
                        "Rent p=0.6, pads attached near their cluster"),
             l2="flushed before every timed step (256 MiB write)")
    if extra:
        c.update(extra)
    return c


def reference_iterations():
    with open(REF_RUNS) as f:
        return json.load(f)["stdcell_200k_qp_mgp"]["iterations"]


def reference_qp_rounds():
    """Rounds of the reference's quadratic placement on this design (its log).
    Its last round ends with the solver error at the stopping threshold
    (1e-6), where float rounding decides between stopping and a round or two
    more; the plain arm runs the same number of rounds as the reference."""
    with open(REF_RUNS) as f:
        return len(json.load(f)["stdcell_200k_qp_mgp"]["qp_trace"])


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


def survey_bytes(info, iterations_per_solve=None):
    """Algorithmic bytes of the hot-path table (FP32 words, int64 bins):
    WA value + gradient 12 P + 4 (nets + 1) + 16 cells per launch, and the
    whole iteration: scatter 20 N_o + 16 B, gather 28 N_o + 8 B, WA, combine
    + Nesterov + Lipschitz 80 N_o, DCT I/O 16 B (HPWL and overflow fused)."""
    no, p, nets, cells = info.num_objects, info.num_pins, info.num_nets, info.num_nodes
    b = info.bins_x * info.bins_y
    wa = 12.0 * p + 4.0 * (nets + 1) + 16.0 * cells
    iteration = (20.0 + 28.0 + 80.0) * no + (16.0 + 8.0 + 16.0) * b + wa
    return wa, iteration


def roofline(times, info, iterations, solve_ms):
    """Dominant kernel group by time per launch, on the algorithmic bytes."""
    hbm, tf, src = peaks()
    dom = max(times, key=lambda t: t["ms"])
    wa, iteration = survey_bytes(info)
    traffic = ncu_traffic().get(dom["name"])
    if dom["name"] == "wirelength":
        alg = wa
    else:
        alg = dom["bytes"]
    ach = alg / (dom["ms"] * 1e-3) / 1e9
    it_ach = iteration * iterations / (solve_ms * 1e-3) / 1e9
    return dict(bound="hbm", achieved=ach, peak=hbm, unit="GB/s", frac=ach / hbm, traffic=traffic,
                kernel=dom["name"], ms_per_launch=dom["ms"], algorithmic_bytes_per_launch=alg,
                peak_source=src + " (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else src,
                whole_iteration=dict(bytes_per_iteration=iteration, iterations=iterations, achieved=it_ach,
                                     frac=it_ach / hbm),
                groups_us={t["name"]: round(t["ms"] * 1e3, 2) for t in times},
                group_frac_own_bytes={t["name"]: round(group_rate(t, hbm, tf)[1], 4) for t in times
                                      if t["bytes"] or t["flops"]})


def max_over_ranks(dist, values, device):
    """Element-wise maximum of `values` over all ranks (each rank's device
    times; the job takes as long as its slowest replica).  `dist` is None for
    a single process."""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def reference_flow(nl):
    """One complete run of the reference's CPU flow; returns its times."""
    from oracle import refharness as R
    R.lib().ref_set_quiet(1)
    ref = R.RefPlacer(nl)
    t0 = time.perf_counter()
    ref.qp()
    t1 = time.perf_counter()
    ref.initialization(1.0)
    t2 = time.perf_counter()
    ref.opt_run()
    t3 = time.perf_counter()
    i = ref.info()
    out = dict(qp_s=t1 - t0, init_s=t2 - t1, mgp_s=t3 - t2, total_s=t3 - t0, iterations=int(i["iter_count"]),
               overflow=float(i["overflow"]), hpwl=float(ref.hpwl()))
    ref.close()
    return out


def cpu_sample(nl, iters_per_sample=SAMPLE_ITERS):
    """The reference's QP and initialization in full, then a few optimizer
    steps, scaled by the reference's iteration count on this design."""
    from oracle import refharness as R
    R.lib().ref_set_quiet(1)
    ref = R.RefPlacer(nl)
    t0 = time.perf_counter()
    ref.qp()
    ref.initialization(1.0)
    t_pre = time.perf_counter() - t0
    ref.opt_begin()
    tt = []
    for _ in range(iters_per_sample):
        stopped, dt = ref.opt_step()
        if stopped:
            break
        tt.append(dt)
    ref.close()
    iters = reference_iterations()
    return t_pre + statistics.mean(tt) * iters, t_pre, statistics.mean(tt), iters


def run_reference(args, rank):
    if rank != 0:
        return 0
    from oracle import refharness as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libeplace_ref.so was not built"}))
        return 0
    nl = netlist()
    r = reference_flow(nl)
    value = r["total_s"]
    sample = ("one complete run of the reference's CPU flow on the same design: QPPlacer::quadraticPlacement, "
              "EPlacer_2D::initialization, EplaceNesterovOpt::opt until overflow < 0.1 (single thread; "
              "the reference has no OpenMP); ms_per_step = the run's time / steps")
    out = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": 0, "ms_per_step": value * 1e3 / max(1, args.steps), "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
           "config": workload_config(nl, dict(reference_run=r)),
           "cpu_baseline": {"value": value, "unit": "s", "cores": 1, "kind": "reference", "sample": sample},
           "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import torch
    torch.cuda.set_device(local)
    # the engines, the network and the timing events share this stream (the
    # legacy default stream does not order against the engines' own streams)
    torch.cuda.set_stream(torch.cuda.Stream())
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from eplace_b200 import placer, warmstart
    nl = netlist()
    stream = torch.cuda.current_stream()
    weights, start = warmstart.load_weights()
    gnn = placer.Gnn(device=local, weights=weights)

    def engine(precision):
        e = placer.Engine(nl, placer.default_params(target_density=1.0, precision=precision, device=local))
        e.set_stream(stream.cuda_stream)
        e.save_positions()
        return e

    mixed, plain = engine(placer.PREC_MIXED), engine(placer.PREC_FP64)
    qp_rounds = reference_qp_rounds()
    info = mixed.info
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed(fn):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    def learned_step():
        mixed.load_positions()
        gnn.release(mixed)  # the proposal builds the graph and features afresh
        t0 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        ref = warmstart.propose(gnn, mixed, start)
        t1 = torch.cuda.Event(enable_timing=True)
        t1.record(stream)
        mixed.initialize()
        st = mixed.nesterov_run()
        t1.synchronize()
        st["start_ms"] = t0.elapsed_time(t1)
        st["start_launches"] = GNN_LAUNCHES + (ref["kernel_launches"] if ref else 0)
        return st

    def plain_step():
        plain.load_positions()
        qp = plain.quadratic_placement(max_iterations=qp_rounds - 1)
        plain.initialize()
        st = plain.nesterov_run()
        st["start_ms"] = qp["seconds"] * 1e3
        return st

    sampler = ClockSampler(local)
    sampler.start()
    for _ in range(args.warmup):
        learned_step()
        plain_step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    lt, pt, lruns, pruns = [], [], [], []
    for _ in range(args.steps):
        ms, st = timed(learned_step)
        lt.append(ms)
        lruns.append(st)
        ms, st = timed(plain_step)
        pt.append(ms)
        pruns.append(st)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    if dist:
        dist.barrier()
    l_ms, p_ms = statistics.mean(lt), statistics.mean(pt)

    # GP only: the mixed form from the plain arm's start (the QP result)
    plain.load_positions()
    plain.quadratic_placement(max_iterations=qp_rounds - 1)
    qp_xy = plain.get_positions()
    mixed.set_positions(qp_xy)
    gp_mixed_ms, gp_mixed = timed(lambda: (mixed.initialize(), mixed.nesterov_run())[1])

    # end to end from host arrays through the C-ABI
    host_out = torch.empty((info.num_objects, 2), dtype=torch.float32, pin_memory=True)
    h2d = sum(int(getattr(nl, k).nbytes) for k in ("node_w", "node_h", "node_cx", "node_cy", "term_llx",
                                                   "term_lly", "term_w", "term_h", "term_is_ni", "net_start",
                                                   "pin_owner", "pin_dx", "pin_dy", "row_llx", "row_lly",
                                                   "row_urx", "row_h"))

    def e2e(precision, how):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e = placer.Engine(nl, placer.default_params(target_density=1.0, precision=precision, device=local))
        if how == "gnn":
            warmstart.propose(gnn, e, start)
        else:
            e.quadratic_placement(max_iterations=qp_rounds - 1)
        e.initialize()
        st = e.nesterov_run()
        n = e.info.num_objects
        e.get_positions_ptr(host_out.data_ptr(), n)
        t1 = time.perf_counter()
        if how == "gnn":
            gnn.release(e)
        e.close()
        return (t1 - t0) * 1e3, st, n

    e2e_l, e2e_p = [], []
    for k in range(args.warmup + args.steps):
        a = e2e(placer.PREC_MIXED, "gnn")
        b = e2e(placer.PREC_FP64, "qp")
        if k >= args.warmup:
            e2e_l.append(a[0])
            e2e_p.append(b[0])
    n_obj = a[2]
    e2e_lms, e2e_pms = statistics.mean(e2e_l), statistics.mean(e2e_p)

    # kernel groups at the placement the last product step ended at (the
    # start is a clump, where the scatter's atomics all meet in a few bins)
    kt = mixed.time_kernels(reps=20)
    l_ms, p_ms, e2e_lms, e2e_pms = max_over_ranks(dist, [l_ms, p_ms, e2e_lms, e2e_pms], "cuda")
    ll, pl = lruns[-1], pruns[-1]
    ratio_hpwl = ll["hpwl"] / pl["hpwl"]
    if rank == 0:
        launches = int(sum(r["kernel_launches"] + r["start_launches"] for r in lruns))
        gp_ms = statistics.mean(r["seconds"] for r in lruns) * 1e3
        out = {"metric": METRIC, "value": l_ms * 1e-3, "unit": "s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": l_ms, "higher_is_better": False, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32", "data": "synthetic",
               "config": workload_config(nl, dict(
                   fillers=info.num_fillers, parallelism=f"replicas x{world}" if world > 1 else "1 GPU",
                   product=("learned warm start (ep_gnn_propose, alpha %.2f, then %d rounds of ep_quadratic_refine"
                            " of at most %d%s solver iterations) + mixed-precision mGP"
                            % (start["alpha"], start["rounds"], start["iters"],
                               " Jacobi-preconditioned" if start.get("jacobi") else "")),
                   plain="device quadratic placement (%d rounds, the reference's count) + FP64 mGP" % qp_rounds,
                   mixed_precision="FP32 positions, FFT Poisson, gather and WA; int64 fixed-point density; "
                                   "FP64 reductions; network BF16 weights, FP32 accumulate",
                   plain_precision="FP64 positions, FFT Poisson, gather and WA; int64 fixed-point density")),
               "learned_mixed": dict(ms=l_ms, start_ms=statistics.mean(r["start_ms"] for r in lruns),
                                     gp_ms=gp_ms, iterations=ll["iterations"], overflow=ll["overflow"],
                                     hpwl=ll["hpwl"]),
               "plain_fp64": dict(ms=p_ms, start_ms=statistics.mean(r["start_ms"] for r in pruns),
                                  gp_ms=statistics.mean(r["seconds"] for r in pruns) * 1e3,
                                  iterations=pl["iterations"], overflow=pl["overflow"], hpwl=pl["hpwl"]),
               "mixed_from_qp": dict(gp_ms=gp_mixed_ms, iterations=gp_mixed["iterations"], hpwl=gp_mixed["hpwl"]),
               "speedup_vs_plain": p_ms / l_ms, "gp_only_speedup_vs_plain":
                   statistics.mean(r["seconds"] for r in pruns) * 1e3 / gp_ms,
               "hpwl_ratio_vs_plain": ratio_hpwl, "hpwl_within_0_5pct": bool(abs(ratio_hpwl - 1.0) <= 0.005),
               "e2e": {"value": e2e_lms * 1e-3, "unit": "s", "h2d_bytes_per_step": h2d,
                       "d2h_bytes_per_step": 8 * n_obj, "plain_fp64_s": e2e_pms * 1e-3,
                       "includes": "ep_create from host arrays, proposal (or QP), initialize, mGP, read-back"},
               "gpu_launches": launches,
               "roofline": roofline(kt, info, ll["iterations"], gp_ms),
               "clocks": clocks}
        if not args.no_cpu_baseline and world == 1:
            try:
                from oracle import refharness as R
                if R.available():
                    v, t_pre, s_it, iters = cpu_sample(nl)
                    out["cpu_baseline"] = {
                        "value": v, "unit": "s", "cores": 1, "kind": "reference",
                        "sample": f"the reference's QP + initialization in full ({t_pre:.1f} s), then "
                                  f"{SAMPLE_ITERS} EplaceNesterovOpt steps ({s_it:.3f} s each) x {iters} "
                                  f"reference steps to overflow<0.1 on this design"}
            except Exception as ex:  # the baseline is reported, never required
                out["cpu_baseline"] = {"value": None, "error": str(ex)[:200]}
        print(json.dumps(out))
    mixed.close()
    plain.close()
    gnn.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
