"""The density scatter that allocates nothing (ep_density_scatter_noalloc),
checked against the engine's own allocating scatter through the C-ABI.

Some callers of this library cannot call cudaMalloc: a host tool whose
allocator reserves all device memory up front and forbids plugins from
allocating, or a caller that must keep the device-wide synchronisation of a
cudaMalloc / cudaFree pair out of its stream work.  The no-allocation entry
point serves them with a fixed 512 x 512-bin scratch array inside the
library.  Its maps must equal the engine's node / filler maps within the
1e-5 relative tolerance the other density tests use, on two calls in a row
(the second call proves the shared scratch is cleared between calls).

The file name sorts last so that a run stopping at the first failure has
already run every other test."""
import numpy as np
import pytest

from eplace_b200 import placer, synth
from tests.helpers import golden_netlist, load_golden, rel_err


def _device_inputs(engine, nl):
    import torch
    i = engine.info
    xy = engine.get_positions()
    nf = i.num_fillers
    row_h = float(nl.row_h[-1])
    w = np.concatenate([nl.node_w, np.full(nf, i.filler_w, np.float32)]).astype(np.float32)
    h = np.concatenate([nl.node_h, np.full(nf, i.filler_h, np.float32)]).astype(np.float32)
    macro = (np.asarray(nl.node_h, np.float64) - row_h > 1e-15).astype(np.uint8)
    flags = np.concatenate([macro, np.full(nf, 2, np.uint8)]).astype(np.uint8)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return dict(cx=t(xy[:, 0]), cy=t(xy[:, 1]), w=t(w), h=t(h), flags=t(flags))


def _grid(engine, td):
    i = engine.info
    return placer.ScatterGrid(i.bins_x, i.bins_y, i.core_llx, i.core_lly, i.bin_step_x, i.bin_step_y, td)


def _noalloc(engine, nl, td):
    import torch
    d = _device_inputs(engine, nl)
    i = engine.info
    node = torch.empty((i.bins_x, i.bins_y), dtype=torch.float32, device="cuda")
    filler = torch.empty_like(node)
    rc, msg = placer.density_scatter_noalloc(_grid(engine, td), i.num_objects, d["cx"].data_ptr(),
                                             d["cy"].data_ptr(), d["w"].data_ptr(), d["h"].data_ptr(),
                                             d["flags"].data_ptr(), node.data_ptr(), filler.data_ptr(),
                                             torch.cuda.current_stream().cuda_stream)
    assert rc == placer.EP_OK, msg
    torch.cuda.synchronize()
    return node.cpu().numpy(), filler.cpu().numpy()


@pytest.mark.gpu
def test_noalloc_equals_engine_scatter_on_two_calls():
    g = load_golden("mixed_5k")  # macros, fixed blocks and fillers on 64 x 64 bins
    nl = golden_netlist(g)
    td = float(g["target_density"])
    e = placer.Engine(nl, placer.default_params(target_density=td, keep_maps=1))
    starts = [np.stack([g["init_cx"], g["init_cy"]], 1), np.stack([g["traj_cx"][-1], g["traj_cy"][-1]], 1)]
    for xy in starts:
        e.set_positions(xy)
        e.eval_gradient()
        ref = e.bin_maps(("node", "filler"))
        node, filler = _noalloc(e, nl, td)
        assert rel_err(node, ref["node"]) < 1e-5
        assert rel_err(filler, ref["filler"]) < 1e-5
    e.close()


@pytest.mark.gpu
def test_noalloc_at_its_largest_grid():
    nl = synth.blob_start(synth.standard_cell(20_000, seed=4))
    e = placer.Engine(nl, placer.default_params(target_density=1.0, bins_x=512, bins_y=512, keep_maps=1))
    e.eval_gradient()
    ref = e.bin_maps(("node", "filler"))
    for _ in range(2):
        node, filler = _noalloc(e, nl, 1.0)
        assert rel_err(node, ref["node"]) < 1e-5
        assert rel_err(filler, ref["filler"]) < 1e-5
    e.close()


def test_noalloc_rejects_a_grid_beyond_its_scratch():
    # the size check comes before any CUDA call, so this runs without a GPU too
    big = placer.ScatterGrid(513, 512, 0.0, 0.0, 1.0, 1.0, 1.0)
    rc, msg = placer.density_scatter_noalloc(big, 0, 0, 0, 0, 0, 0, 1, 0)
    assert rc == placer.EP_ERR_ARG and "512 x 512" in msg
