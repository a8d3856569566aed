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

The maps are also held bit for bit to the oracle's scatter quantised at the
fixed-point scale the header states (2^k units per area unit, k chosen from
the object count and the bin area so that no bin sum can pass int64), on
the golden design and on a design drawn in fine units (a thousand units per
site), whose bin area would have wrapped a fixed 2^32 scale.

The file name sorts last so that a run stopping at the first failure has
already run every other test."""
import math

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
    d = _device_inputs(engine, nl)
    i = engine.info
    return _noalloc_raw(_grid(engine, td), i.num_objects, d, i.bins_x, i.bins_y)


def _noalloc_raw(grid, n, d, nx, ny):
    import torch
    node = torch.empty((nx, ny), dtype=torch.float32, device="cuda")
    filler = torch.empty_like(node)
    rc, msg = placer.density_scatter_noalloc(grid, n, d["cx"].data_ptr(),
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


def _scale_bits(num_objects, step_x, step_y):
    """k of the header: 2^k fixed-point units per area unit."""
    bin_area = float(np.float32(step_x)) * float(np.float32(step_y))
    return min(40, math.floor(62.0 - math.log2(1.05 * num_objects * bin_area + 1.0)))


def _oracle_maps(e, nl, td, xy):
    from oracle import oracle as O
    from tests.helpers import OracleDesign
    i = e.info
    od = OracleDesign(nl, (np.asarray(nl.node_h, np.float64) - float(nl.row_h[-1]) > 1e-15).astype(np.uint8),
                      i.num_fillers, i.filler_w, i.filler_h, (i.core_llx, i.core_lly, i.core_urx, i.core_ury),
                      (i.bins_x, i.bins_y), (i.bin_step_x, i.bin_step_y), td)
    k = _scale_bits(i.num_objects, i.bin_step_x, i.bin_step_y)
    _, _, nq, fq = O.scatter(od.grid, xy[:, 0], xy[:, 1], od.w, od.h, od.flags, math.ldexp(1.0, k))
    to_f = lambda q: (q.astype(np.float64) * math.ldexp(1.0, -k)).astype(np.float32)
    return to_f(nq), to_f(fq), k


@pytest.mark.gpu
def test_noalloc_bit_exact_against_the_oracle_at_its_scale():
    g = load_golden("mixed_5k")
    nl = golden_netlist(g)
    td = float(g["target_density"])
    e = placer.Engine(nl, placer.default_params(target_density=td, keep_maps=1))
    for xy in (np.stack([g["init_cx"], g["init_cy"]], 1), np.stack([g["traj_cx"][-1], g["traj_cy"][-1]], 1)):
        e.set_positions(xy)
        xy = e.get_positions()
        node, filler = _noalloc(e, nl, td)
        on, of, _ = _oracle_maps(e, nl, td, xy)
        assert np.array_equal(node, on) and np.array_equal(filler, of)
    e.close()


def _fine_units(nl, f):
    """The same design drawn with f units per site (sizes, offsets, rows, pads)."""
    import copy
    n = copy.copy(nl)
    for k in ("node_w", "node_h", "node_cx", "node_cy", "term_llx", "term_lly", "term_w", "term_h",
              "pin_dx", "pin_dy", "row_llx", "row_lly", "row_urx", "row_h", "row_site_w"):
        setattr(n, k, np.ascontiguousarray(getattr(nl, k) * np.float32(f), np.float32))
    return n


@pytest.mark.gpu
def test_noalloc_fine_unit_design_keeps_its_sums():
    # a macro-heavy design in 1000 units per site: bins of ~1.6e7 area units,
    # where 2^32 units per area unit would have wrapped the int64 sums
    base = synth.blob_start(synth.mixed_size(3000, 6, 3, seed=8))
    nl = _fine_units(base, 1000.0)
    e = placer.Engine(nl, placer.default_params(target_density=1.0, bins_x=64, bins_y=64, keep_maps=1))
    i = e.info
    assert _scale_bits(i.num_objects, i.bin_step_x, i.bin_step_y) < 32
    xy = e.get_positions()
    node, filler = _noalloc(e, nl, 1.0)
    on, of, _ = _oracle_maps(e, nl, 1.0, xy)
    assert np.array_equal(node, on) and np.array_equal(filler, of)
    assert node.min() >= 0 and filler.min() >= 0
    e.eval_gradient()
    ref = e.bin_maps(("node", "filler"))
    assert rel_err(node, ref["node"]) < 1e-5 and rel_err(filler, ref["filler"]) < 1e-5
    e.close()


def test_noalloc_rejects_bins_its_int64_sums_cannot_hold():
    # checked before any CUDA call, so this runs without a GPU too
    g = placer.ScatterGrid(64, 64, 0.0, 0.0, 3.0e9, 3.0e9, 1.0)
    rc, msg = placer.density_scatter_noalloc(g, 1000, 1, 1, 1, 1, 0, 1, 0)
    assert rc == placer.EP_ERR_ARG and "int64" in msg
    bad_td = placer.ScatterGrid(64, 64, 0.0, 0.0, 1.0, 1.0, 1.5)
    rc, msg = placer.density_scatter_noalloc(bad_td, 10, 1, 1, 1, 1, 0, 1, 0)
    assert rc == placer.EP_ERR_ARG and "target_density" in msg
