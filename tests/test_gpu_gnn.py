"""The learned warm start's kernels (ep_gnn_*) through the C-ABI, against a
float64 restatement on the CPU (numpy for the features, PyTorch autograd for
the network -- test-side only).

Tolerances:
  * diffusion features: 1e-5 absolute (core-normalised coordinates) against
    the same 8/32/128 mean-aggregation steps in float64;
  * both heads' predictions and the loss: 1e-5 relative; every weight
    gradient: 1e-4 of the largest gradient entry, against autograd on the
    BF16-rounded weights (the forward pass uses BF16 weights and FP32
    accumulation; its hidden layers run on the tensor cores with each FP32
    input split into two BF16 planes, 2^-17 relative);
  * a training step is bitwise repeatable, and 60 Adam steps on one design
    lower its loss by at least a fifth;
  * a proposal puts the movable nodes at q + alpha (f - q) of the forward
    pass (to float rounding of the core mapping, and the core clamp).
"""
import numpy as np
import pytest

from eplace_b200 import placer, synth

pytestmark = pytest.mark.gpu

H, F = 64, 9


def small_design(n=400, seed=3):
    return synth.blob_start(synth.standard_cell(n, seed=seed, every_cell_pinned=True, local_pads=True))


def graph(nl):
    """Mean-aggregation matrices over movable nodes + terminals, float64."""
    nn, nt = nl.num_nodes, nl.num_terminals
    N, nnet = nn + nt, nl.num_nets
    deg = np.diff(nl.net_start)
    net = np.repeat(np.arange(nnet), deg)
    node = np.asarray(nl.pin_owner, np.int64)  # terminals follow the nodes
    inc = np.zeros((nnet, N))
    np.add.at(inc, (net, node), 1.0)
    net_mean = inc / deg[:, None]
    pins = inc.sum(0)
    node_mean = inc.T / np.maximum(pins, 1)[:, None]
    node_mean[nn:] = 0.0
    return net_mean, node_mean, pins


def features_ref(nl):
    nn = nl.num_nodes
    net_mean, node_mean, pins = graph(nl)
    llx, lly, urx, ury = nl.core()
    tcx = (nl.term_llx + 0.5 * nl.term_w - llx) / (urx - llx)
    tcy = (nl.term_lly + 0.5 * nl.term_h - lly) / (ury - lly)
    v = np.concatenate([np.full((nn, 2), 0.5), np.stack([tcx, tcy], 1)]).astype(np.float64)
    has = pins[:nn] > 0
    cols = []
    for k in range(1, 129):
        new = node_mean @ (net_mean @ v)
        v[:nn][has] = new[:nn][has]
        if k in (8, 32, 128):
            cols.append(v.copy())
    return cols


def test_features_match_float64_diffusion():
    nl = small_design(3000, 5)
    e = placer.Engine(nl, placer.default_params(target_density=1.0))
    g = placer.Gnn(seed=2)
    x = g.features(e)
    nn = nl.num_nodes
    assert x.shape == (nn + nl.num_terminals, F)
    area = nl.node_w.astype(np.float64) * nl.node_h
    assert np.allclose(x[:nn, 0], np.log1p(area) / 4, atol=1e-6)
    assert np.all(x[:nn, 2] == 0) and np.all(x[nn:, 2] == 1)
    for j, ref in enumerate(features_ref(nl)):
        assert np.abs(x[:, 3 + 2 * j: 5 + 2 * j] - ref).max() < 1e-5, j
    g.close()
    e.close()


def torch_loss(x, w, nl, target, nn):
    import torch
    net_mean, node_mean, _ = graph(nl)
    A = torch.tensor(net_mean)
    M = torch.tensor(node_mean)
    X = torch.tensor(x, dtype=torch.float64)
    wb = torch.tensor(w).to(torch.bfloat16).to(torch.float64)  # the forward pass's weights
    wf = torch.tensor(w, dtype=torch.float64)
    p = {}
    o = 0

    def take(name, rows, cols, bf16):
        nonlocal o
        n = rows * cols
        src = wb if bf16 else wf
        p[name] = src[o:o + n].reshape(rows, cols).clone().requires_grad_(True)
        o += n

    take("W0", H, F, True)
    take("b0", 1, H, False)
    for l in (1, 2, 3):
        take(f"W{l}", H, 2 * H, True)
        take(f"b{l}", 1, H, False)
    take("W4", 4, H, True)
    take("b4", 1, 4, False)
    h = torch.relu(X @ p["W0"].T + p["b0"])
    for l in (1, 2, 3):
        m = M @ (A @ h)
        h = torch.relu(torch.cat([h, m], 1) @ p[f"W{l}"].T + p[f"b{l}"])
    raw = h @ p["W4"].T + p["b4"]
    d = X[:, 7:9]
    pred = torch.cat([d, d], 1) + 0.25 * torch.tanh(raw)
    t = torch.tensor(target, dtype=torch.float64)
    loss = ((pred[:nn] - t) ** 2).sum() / (2 * nn)
    loss.backward()
    grad = torch.cat([p[k].grad.reshape(-1) for k in
                      ("W0", "b0", "W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4")]).numpy()
    return loss.item(), pred.detach().numpy(), grad


def test_forward_loss_and_gradients_match_autograd():
    nl = small_design()
    e = placer.Engine(nl, placer.default_params(target_density=1.0))
    g = placer.Gnn(seed=4)
    w = g.get_weights()
    # larger output weights so every layer carries gradient
    w[-(4 * H + 4):] = np.random.default_rng(1).uniform(-0.5, 0.5, 4 * H + 4).astype(np.float32)
    g.set_weights(w)
    x = g.features(e)
    i = e.info
    rng = np.random.default_rng(7)
    nn = nl.num_nodes
    tgt = rng.uniform(0.05, 0.95, (nn, 4))
    core_w, core_h = i.core_urx - i.core_llx, i.core_ury - i.core_lly
    lo = np.array([i.core_llx, i.core_lly] * 2)
    size = np.array([core_w, core_h] * 2)
    target4 = (lo + tgt * size).astype(np.float32)
    tgt_norm = (target4.astype(np.float64) - lo) / size
    loss, grad = g.loss_grad(e, target4)
    rl, rpred, rgrad = torch_loss(x, w, nl, tgt_norm, nn)
    assert loss == pytest.approx(rl, rel=1e-5)
    pred = g.forward(e)
    ref = lo + rpred[:nn] * size
    assert np.abs(pred - ref).max() < 1e-5 * max(core_w, core_h)
    assert np.abs(grad - rgrad).max() < 1e-4 * np.abs(rgrad).max()
    # every block of weights receives gradient
    assert np.abs(grad[:H * F]).max() > 0 and np.abs(grad[-(4 * H + 4):]).max() > 0
    g.close()
    e.close()


def test_training_is_repeatable_and_learns():
    nl = small_design(2000, 9)
    e = placer.Engine(nl, placer.default_params(target_density=1.0))
    e.quadratic_placement()
    qp = e.get_positions()[:nl.num_nodes]
    e.initialize()
    e.nesterov_run()
    target = np.concatenate([qp, e.get_positions()[:nl.num_nodes]], 1)
    runs = []
    for _ in range(2):
        g = placer.Gnn(seed=11)
        losses = [g.train_step(e, target, 3e-3) for _ in range(60)]
        runs.append((losses, g.get_weights()))
        g.close()
    assert runs[0][0] == runs[1][0] and np.array_equal(runs[0][1], runs[1][1])
    losses = runs[0][0]
    assert np.mean(losses[-5:]) < 0.8 * np.mean(losses[:3]), (losses[:3], losses[-5:])
    e.close()


@pytest.mark.parametrize("alpha", [0.0, 0.4, 1.0])
def test_proposal_blends_the_two_heads(alpha):
    nl = small_design(3000, 5)
    e = placer.Engine(nl, placer.default_params(target_density=1.0))
    g = placer.Gnn(seed=2)
    p = g.forward(e).astype(np.float64)
    g.propose(e, alpha)
    i = e.info
    xy = e.get_positions()[:nl.num_nodes]
    ref = p[:, :2] + alpha * (p[:, 2:] - p[:, :2])
    # the core clamp keeps a node's box inside the core
    hw = nl.node_w.astype(np.float64) / 2
    inside = (ref[:, 0] - hw > i.core_llx + 1e-3) & (ref[:, 0] + hw < i.core_urx - 1e-3) & \
             (ref[:, 1] - 0.5 > i.core_lly + 1e-3) & (ref[:, 1] + 0.5 < i.core_ury - 1e-3)
    assert inside.mean() > 0.9
    assert np.abs(xy[inside] - ref[inside]).max() < 1e-3
    g.close()
    e.close()


def test_bad_arguments():
    nl = small_design()
    e = placer.Engine(nl, placer.default_params(target_density=1.0))
    g = placer.Gnn()
    with pytest.raises(placer.EPError):
        g.propose(e, 1.5)
    with pytest.raises(ValueError):
        g.set_weights(np.zeros(3, np.float32))
    g.close()
    e.close()


def test_forward_at_many_tiles_per_cta():
    """The forward pass on a design whose tensor-core dense layers take
    several 128-row tiles per persistent CTA (60k nodes: 470 tiles over at
    most two CTAs per SM), against a float64 forward pass with sparse
    aggregations on the same features; 1e-5 of the core, as above."""
    import scipy.sparse as sp
    nl = small_design(60000, 12)
    e = placer.Engine(nl, placer.default_params(target_density=1.0))
    g = placer.Gnn(seed=6)
    w = g.get_weights()
    w[-(4 * H + 4):] = np.random.default_rng(2).uniform(-0.5, 0.5, 4 * H + 4).astype(np.float32)
    g.set_weights(w)
    x = g.features(e).astype(np.float64)
    pred = g.forward(e)
    nn, N, nnet = nl.num_nodes, nl.num_nodes + nl.num_terminals, nl.num_nets
    deg = np.diff(nl.net_start)
    inc = sp.csr_matrix((np.ones(len(nl.pin_owner)), (np.repeat(np.arange(nnet), deg),
                                                        np.asarray(nl.pin_owner, np.int64))), shape=(nnet, N))
    pins = np.asarray(inc.sum(0)).ravel()
    A = sp.diags(1.0 / np.maximum(deg, 1)) @ inc
    scale = np.where(np.arange(N) < nn, 1.0 / np.maximum(pins, 1), 0.0)
    M = sp.diags(scale) @ inc.T.tocsr()
    import torch
    wb = torch.tensor(w).to(torch.bfloat16).to(torch.float64).numpy()
    o = 0

    def take(rows, cols, bf16):
        nonlocal o
        v = (wb if bf16 else w.astype(np.float64))[o:o + rows * cols].reshape(rows, cols)
        o += rows * cols
        return v

    W0, b0 = take(H, F, True), take(1, H, False)
    h = np.maximum(x @ W0.T + b0, 0)
    for _ in range(3):
        Wl, bl = take(H, 2 * H, True), take(1, H, False)
        h = np.maximum(np.concatenate([h, M @ (A @ h)], 1) @ Wl.T + bl, 0)
    W4, b4 = take(4, H, True), take(1, 4, False)
    d = x[:, 7:9]
    ref = np.concatenate([d, d], 1) + 0.25 * np.tanh(h @ W4.T + b4)
    i = e.info
    core_w, core_h = i.core_urx - i.core_llx, i.core_ury - i.core_lly
    lo = np.array([i.core_llx, i.core_lly] * 2)
    size = np.array([core_w, core_h] * 2)
    assert np.abs(pred - (lo + ref[:nn] * size)).max() < 1e-5 * max(core_w, core_h)
    g.close()
    e.close()


def test_dense_layer_wait_gives_up_and_recovers():
    """The tensor-core layers' mbarrier wait, bounded: with no polls allowed
    every wait gives up, the forward pass reports EP_ERR_TIMEOUT (the CTA
    still waits for its own MMAs before it frees its tensor memory), and with
    the default limit restored the next pass gives the same predictions as
    before, bit for bit."""
    nl = small_design(3000, 5)
    e = placer.Engine(nl, placer.default_params(target_density=1.0))
    g = placer.Gnn(seed=2)
    ref = g.forward(e)
    g.set_wait_limit(0)
    with pytest.raises(placer.EPError) as err:
        g.forward(e)
    assert err.value.status == placer.EP_ERR_TIMEOUT
    g.set_wait_limit()
    assert np.array_equal(g.forward(e), ref)
    g.close()
    e.close()
