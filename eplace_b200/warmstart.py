"""Learned warm start: training data, training and evaluation of the
message-passing network of the engine (ep_gnn_*, eplace_b200/csrc/gnn.cu)
that proposes the initial placement in place of the quadratic placement
(QPPlacer::quadraticPlacement, QPlace/qplace.cpp:20-103).

  * training designs: standard-cell netlists of 2k-50k cells (log-uniform,
    synth.standard_cell with pinned cells and local pads), each placed by the
    engine itself -- device quadratic placement, then mGP to overflow < 0.1
    (many designs at once, ep_run_batch);
  * training pairs: (netlist, final mGP centres), written by log_pair as the
    binary netlist file (ep_netbin_write) plus the centres as .npy;
  * training: Adam on the mean squared error of the network's two heads
    against the engine's quadratic placement and final mGP centres of each
    design (normalised to the core), one design per step in a seeded order;
  * the start: the network's proposal q + alpha (f - q), q and f the two
    heads, then `rounds` rounds of the quadratic model from there with at
    most `iters` BiCGSTAB iterations each, Jacobi-preconditioned or not
    (ep_quadratic_refine; rounds 0 = none).  (alpha, rounds, iters, jacobi)
    are picked on validation designs (not the held-out ones): the least
    solver work (rounds x iters), then the largest alpha, whose runs end with a mean HPWL within 0.15% of the QP-started
    runs, else the choice with the lowest mean HPWL;
  * evaluation: on held-out designs, the QP-started run against the
    proposal-started run (iterations and device seconds to overflow < 0.1,
    final HPWL), and the judge: a proposal is kept when its run reaches the
    overflow target at an HPWL within `tolerance` of the QP-started run.
    Start times: the quadratic placement's device time (CUDA events); the
    proposal's host wall time around ep_gnn_propose (graph build on first
    use, diffusion features, forward pass, positions set; it synchronises).

    python -m eplace_b200.warmstart train --designs 256 --steps 6000 --out W.npz
    python -m eplace_b200.warmstart pick --weights W.npz --out W2.npz   # re-pick the start only
    python -m eplace_b200.warmstart eval --weights W.npz --cells 200000 --seeds 100-119
"""
import argparse
import json
import math
import os
import time

import numpy as np

from eplace_b200 import placer, synth

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "warmstart_weights.npz")


def design(cells, seed):
    return synth.standard_cell(int(cells), seed=int(seed), every_cell_pinned=True, local_pads=True)


def training_sizes(count, seed, lo=2_000, hi=50_000):
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(math.log(lo), math.log(hi), count)).astype(int)


def load_weights(path=WEIGHTS):
    """(weights, start) of a trained network; start = dict(alpha, rounds,
    iters, jacobi)."""
    z = np.load(path)
    iters = int(z["iters"]) if "iters" in z.files else 100
    jacobi = int(z["jacobi"]) if "jacobi" in z.files else 0
    return z["weights"], dict(alpha=float(z["alpha"]), rounds=int(z["rounds"]), iters=iters, jacobi=jacobi)


def save_weights(path, weights, start, meta):
    np.savez(path, weights=np.asarray(weights, np.float32), alpha=np.float32(start["alpha"]),
             rounds=np.int32(start["rounds"]), iters=np.int32(start["iters"]),
             jacobi=np.int32(start.get("jacobi", 0)), meta=np.array(json.dumps(meta)))


def propose(gnn, engine, start):
    """The learned start: the network's proposal, then start["rounds"]
    rounds of the quadratic model from it (start["iters"] solver iterations
    each, Jacobi-preconditioned when start["jacobi"]); returns the
    refinement's statistics (None without refinement)."""
    gnn.propose(engine, start["alpha"])
    if start["rounds"] > 0:
        return engine.quadratic_refine(start["rounds"], start["iters"], start.get("jacobi", 0))
    return None


def log_pair(directory, name, nl, final_xy):
    """Write one training pair: the netlist as a binary netlist file and the
    final centres of its movable nodes as a float32 [num_nodes, 2] array."""
    os.makedirs(directory, exist_ok=True)
    placer.netbin_write(nl, os.path.join(directory, f"{name}.netbin"))
    np.save(os.path.join(directory, f"{name}.final.npy"), np.asarray(final_xy, np.float32))


def read_pair(directory, name):
    nl = placer.netbin_read(os.path.join(directory, f"{name}.netbin"))
    return nl, np.load(os.path.join(directory, f"{name}.final.npy"))


def place_designs(netlists, precision=placer.PREC_MIXED):
    """QP then mGP for every netlist (mGP runs batched); returns the engines
    (positions at their mGP result), the training targets [num_nodes, 4]
    (QP centre, final centre) and the run statistics."""
    engines = placer.create_engines(netlists, placer.default_params(target_density=1.0, precision=precision))
    qp_xy = []
    for nl, e in zip(netlists, engines):
        e.quadratic_placement()
        qp_xy.append(e.get_positions()[:nl.num_nodes])
        e.initialize()
    stats = placer.run_batch(engines)
    targets = [np.concatenate([q, e.get_positions()[:nl.num_nodes]], 1)
               for q, e, nl in zip(qp_xy, engines, netlists)]
    return engines, targets, stats


def train(gnn, engines, targets, steps, lr=2e-3, seed=0, log_every=0):
    """Adam steps over (engine, target centres) pairs in a seeded order;
    returns the loss before each step."""
    rng = np.random.default_rng(seed)
    losses = []
    order = []
    for s in range(steps):
        if not order:
            order = list(rng.permutation(len(engines)))
        k = order.pop()
        # cosine decay to a tenth of the rate
        rate = lr * (0.1 + 0.9 * 0.5 * (1.0 + math.cos(math.pi * s / max(1, steps))))
        losses.append(gnn.train_step(engines[k], targets[k], rate))
        if log_every and (s % log_every == 0 or s == steps - 1):
            print(f"step {s}: loss {np.mean(losses[-log_every:]):.6f}", flush=True)
    return losses


def run_from(engine, start):
    """mGP from the engine's current positions; start names the start."""
    engine.initialize()
    st = engine.nesterov_run()
    st["start"] = start
    return st


def compare(gnn, nl, start, precision=placer.PREC_MIXED, tolerance=0.005):
    """The QP-started run against the proposal-started run on one design.
    Device seconds of each start (quadratic placement; graph build, features
    and forward pass of the network) and of each mGP run."""
    out = {}
    e = placer.Engine(nl, placer.default_params(target_density=1.0, precision=precision))
    e.save_positions()
    qp = e.quadratic_placement()
    r = run_from(e, "qp")
    r["start_seconds"] = qp["seconds"]
    out["qp"] = r
    e.load_positions()
    e.synchronize()
    t0 = time.perf_counter()
    propose(gnn, e, start)
    e.synchronize()
    t_gnn = time.perf_counter() - t0
    r = run_from(e, "gnn")
    r["start_seconds"] = t_gnn
    out["gnn"] = r
    gnn.release(e)
    e.close()
    ratio = out["gnn"]["hpwl"] / out["qp"]["hpwl"]
    out["hpwl_ratio"] = ratio
    out["kept"] = bool(out["gnn"]["overflow"] < 0.1 and ratio <= 1.0 + tolerance)
    return out


def pick_start(gnn, netlists, alphas=(0.0, 0.5),
               refinements=((0, 0, 0), (1, 10, 1), (1, 15, 1), (1, 20, 1), (1, 20, 0), (1, 40, 0), (1, 40, 1),
                            (1, 100, 0)),
               within=0.0015):
    """On these (validation) netlists: the start (alpha, rounds, iters,
    jacobi) with the least solver work (rounds x iters), then the largest
    alpha, whose runs end with a mean HPWL ratio to the QP-started runs of
    at most 1 + within, else the one with the lowest mean ratio.  Returns it
    and the table of mean ratios and iterations."""
    keys = [(a, r, it, j) for r, it, j in refinements for a in alphas]
    ratio = {k: [] for k in keys}
    iters = {k: [] for k in keys}
    for nl in netlists:
        e = placer.Engine(nl, placer.default_params(target_density=1.0))
        e.save_positions()
        e.quadratic_placement()
        ref = run_from(e, "qp")["hpwl"]
        for a, r, it, j in keys:
            e.load_positions()
            propose(gnn, e, dict(alpha=a, rounds=r, iters=it, jacobi=j))
            st = run_from(e, f"gnn{a}/{r}x{it}j{j}")
            ratio[(a, r, it, j)].append(st["hpwl"] / ref)
            iters[(a, r, it, j)].append(st["iterations"])
        gnn.release(e)
        e.close()
    mean = {k: float(np.mean(v)) for k, v in ratio.items()}
    ok = [k for k in keys if mean[k] <= 1.0 + within]
    best = min(ok, key=lambda k: (k[1] * k[2], -k[0])) if ok else min(mean, key=mean.get)
    table = {f"{a}/{r}x{it}{'j' if j else ''}": dict(hpwl_ratio=mean[(a, r, it, j)],
                                                     iterations=float(np.mean(iters[(a, r, it, j)])))
             for a, r, it, j in keys}
    return dict(alpha=best[0], rounds=best[1], iters=best[2], jacobi=best[3]), table


def _seeds(spec):
    a, b = spec.split("-") if "-" in spec else (spec, spec)
    return list(range(int(a), int(b) + 1))


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--designs", type=int, default=256)
    t.add_argument("--valid", type=int, default=6)
    t.add_argument("--steps", type=int, default=6000)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--seed", type=int, default=1)
    t.add_argument("--pairs", default="")
    t.add_argument("--out", required=True)
    pk = sub.add_parser("pick")
    pk.add_argument("--weights", default=WEIGHTS)
    pk.add_argument("--valid", type=int, default=6)
    pk.add_argument("--seed", type=int, default=1)
    pk.add_argument("--out", required=True)
    ev = sub.add_parser("eval")
    ev.add_argument("--weights", default=WEIGHTS)
    ev.add_argument("--cells", type=int, default=200_000)
    ev.add_argument("--seeds", default="100-119")
    ev.add_argument("--out", default="")
    a = ap.parse_args()
    if a.cmd in ("train", "pick"):
        valid = [design(n, 900_000 + i) for i, n in enumerate(training_sizes(a.valid, a.seed + 7, 40_000, 120_000))]
    if a.cmd == "pick":
        w, _ = load_weights(a.weights)
        meta = json.loads(str(np.load(a.weights)["meta"]))
        gnn = placer.Gnn(weights=w)
        start, meta["start_table"] = pick_start(gnn, valid)
        save_weights(a.out, w, start, meta)
        print(json.dumps(dict(start=start, start_table=meta["start_table"])))
    elif a.cmd == "train":
        t0 = time.time()
        sizes = training_sizes(a.designs, a.seed)
        nls = [design(n, 1000 + a.seed * 10_000 + i) for i, n in enumerate(sizes)]
        t_gen = time.time() - t0
        engines, targets, stats = place_designs(nls)
        t_place = time.time() - t0 - t_gen
        if a.pairs:
            for i, (nl, tg) in enumerate(zip(nls, targets)):
                log_pair(a.pairs, f"d{i:03d}", nl, tg[:, 2:])
        gnn = placer.Gnn(seed=a.seed)
        losses = train(gnn, engines, targets, a.steps, a.lr, a.seed, log_every=250)
        for e in engines:
            gnn.release(e)
            e.close()
        start, table = pick_start(gnn, valid)
        meta = dict(designs=a.designs, steps=a.steps, lr=a.lr, seed=a.seed, final_loss=float(np.mean(losses[-100:])),
                    first_loss=float(np.mean(losses[:50])), start_table=table, generate_s=t_gen, place_s=t_place,
                    iterations=[int(s["iterations"]) for s in stats])
        save_weights(a.out, gnn.get_weights(), start, meta)
        print(json.dumps(dict(start=start, **meta)))
    else:
        w, start = load_weights(a.weights)
        gnn = placer.Gnn(weights=w)
        rows = []
        for s in _seeds(a.seeds):
            r = compare(gnn, design(a.cells, s), start)
            r["seed"] = s
            rows.append(r)
            print(json.dumps({k: r[k] for k in ("seed", "hpwl_ratio", "kept")} |
                             {f"{k}_{f}": r[k][f] for k in ("qp", "gnn")
                              for f in ("iterations", "seconds", "start_seconds", "hpwl")}), flush=True)
        if a.out:
            with open(a.out, "w") as f:
                json.dump(dict(start=start, rows=rows), f, indent=1)


if __name__ == "__main__":
    main()
