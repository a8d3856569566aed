"""CPU checks of the C-ABI library and the host-side helpers (no GPU needed)."""
import os
import re

import numpy as np
import pytest

from eplace_b200 import bookshelf, placer, synth
from tests.conftest import HAS_GPU

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "eplace_gpu.h")).read()
    return sorted(set(re.findall(r"\b(ep_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = placer.load()
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(placer.EXPORTS)


def test_abi_version_and_defaults():
    L = placer.load()
    assert L.ep_abi_version() == placer.ABI_VERSION == 3
    p = placer.default_params()
    assert p.target_density == pytest.approx(1.0)
    assert p.target_overflow == pytest.approx(0.10)
    assert p.max_iterations == 1000
    assert p.dct_mode == placer.DCT_AUTO and p.exp_mode == placer.EXP_FAST
    assert p.precision == placer.PREC_MIXED


def _bad_netlist(mutate):
    nl = synth.smoke(1)
    mutate(nl)
    return nl


@pytest.mark.parametrize("mutate,needle", [
    (lambda nl: setattr(nl, "net_start", np.concatenate([[0], nl.net_start[1:2], nl.net_start[1:]]).astype(np.int32)),
     "empty net"),
    (lambda nl: nl.pin_owner.__setitem__(0, 10_000), "pin_owner"),
    (lambda nl: nl.node_w.__setitem__(3, 0.0), "node sizes"),
    (lambda nl: nl.node_cx.__setitem__(3, np.nan), "node sizes"),
])
def test_netlist_validation_returns_arg_error(mutate, needle):
    nl = _bad_netlist(mutate)
    with pytest.raises(placer.EPError) as ex:
        placer.Engine(nl)
    assert ex.value.status == placer.EP_ERR_ARG
    assert needle in str(ex.value)


@pytest.mark.skipif(HAS_GPU, reason="checks the no-GPU error path")
def test_no_gpu_is_a_loud_error_not_a_fallback():
    with pytest.raises(placer.EPError) as ex:
        placer.Engine(synth.smoke(1))
    assert ex.value.status == placer.EP_ERR_CUDA
    assert "no CPU fallback" in str(ex.value)


def test_bookshelf_round_trip(tmp_path):
    nl = synth.mixed_size(800, 3, 2, seed=2)
    aux = synth.write_bookshelf(nl, str(tmp_path))
    rd = bookshelf.read_aux(aux, target_density=nl.target_density)
    for k in ("node_w", "node_h", "node_cx", "node_cy", "term_llx", "term_lly", "term_w", "term_h",
              "term_is_ni", "net_start", "pin_owner", "pin_dx", "pin_dy", "row_llx", "row_lly",
              "row_urx", "row_h"):
        a, b = getattr(nl, k), getattr(rd, k)
        assert np.array_equal(np.asarray(a, b.dtype), b), k


def test_standard_cell_generator_shape():
    nl = synth.standard_cell(20_000, seed=9)
    nl.validate()
    deg = np.diff(nl.net_start)
    assert nl.num_nets == 22_000 and nl.num_terminals == 200
    assert 3.3 < deg.mean() < 3.9 and deg.max() <= 500 and deg.min() >= 2
    w = nl.node_w
    assert w.min() >= 1 and w.max() <= 20 and 2.6 < w.mean() < 3.4
    # pins of a net are distinct cells
    for n in range(0, nl.num_nets, 997):
        o = nl.pin_owner[nl.net_start[n]:nl.net_start[n + 1]]
        assert len(set(o.tolist())) == len(o)
    # Rent-style locality: most nets span a small index window
    span = [np.ptp(nl.pin_owner[nl.net_start[n]:nl.net_start[n + 1]][
        nl.pin_owner[nl.net_start[n]:nl.net_start[n + 1]] < nl.num_nodes]) for n in range(0, nl.num_nets, 11)]
    assert np.median(span) < 200


def test_generators_are_seeded():
    a = synth.standard_cell(3000, seed=5)
    b = synth.standard_cell(3000, seed=5)
    c = synth.standard_cell(3000, seed=6)
    assert np.array_equal(a.pin_owner, b.pin_owner) and np.array_equal(a.node_w, b.node_w)
    assert not np.array_equal(a.pin_owner, c.pin_owner)


def test_powerlaw_alpha_fit():
    a = synth.fit_powerlaw_alpha(3.6, 2, 500)
    d = np.arange(2, 501, dtype=np.float64)
    w = d ** -a
    assert (d * w).sum() / w.sum() == pytest.approx(3.6, rel=1e-6)
