"""Binary netlist file (row f3 of the hot-path table: a fast, lossless
netlist format; the reference's Bookshelf text path is its slow, lossy
I/O).  The C writer / mapper (ep_netbin_write, ep_netbin_open) and the numpy
implementation (eplace_b200.netbin) are written independently and must agree
byte for byte on the arrays; both round-trip every array exactly.  CPU only:
no CUDA call is involved."""
import time

import numpy as np

from eplace_b200 import bookshelf, netbin, placer, synth

FIELDS = ("node_w", "node_h", "node_cx", "node_cy", "term_llx", "term_lly", "term_w", "term_h",
          "term_is_ni", "net_start", "pin_owner", "pin_dx", "pin_dy", "row_llx", "row_lly", "row_urx",
          "row_h")


def same(a, b, with_site=True):
    for k in FIELDS + (("row_site_w",) if with_site else ()):
        x, y = np.asarray(getattr(a, k)), np.asarray(getattr(b, k))
        assert x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8)), k
    assert np.float32(a.target_density) == np.float32(b.target_density)
    assert int(a.bins) == int(b.bins)


def test_numpy_round_trip(tmp_path):
    nl = synth.blob_start(synth.mixed_size(3000, 4, 2, seed=9))
    p = netbin.write(nl, str(tmp_path / "d.epn"))
    same(nl, netbin.read(p))
    same(nl, netbin.read(p, mmap=False))


def test_c_and_numpy_agree(tmp_path):
    nl = synth.blob_start(synth.standard_cell(5000, seed=4))
    a = netbin.write(nl, str(tmp_path / "py.epn"))
    b = placer.netbin_write(nl, str(tmp_path / "c.epn"))
    same(nl, placer.netbin_read(a), with_site=False)   # numpy file, C reader
    r = netbin.read(b)                                  # C file, numpy reader
    same(nl, r, with_site=False)
    assert np.all(r.row_site_w == 1.0)


def test_rejects_bad_files(tmp_path):
    p = tmp_path / "bad.epn"
    p.write_bytes(b"NOTANETL" + b"\0" * 400)
    try:
        placer.netbin_read(str(p))
    except placer.EPError as ex:
        assert ex.status == placer.EP_ERR_ARG
    else:
        raise AssertionError("accepted a file without the magic")
    nl = synth.smoke()
    good = netbin.write(nl, str(tmp_path / "good.epn"))
    raw = bytearray(open(good, "rb").read())
    raw = raw[: len(raw) // 2]  # truncated: arrays past the end
    (tmp_path / "short.epn").write_bytes(bytes(raw))
    try:
        placer.netbin_read(str(tmp_path / "short.epn"))
    except placer.EPError as ex:
        assert ex.status == placer.EP_ERR_ARG
    else:
        raise AssertionError("accepted a truncated file")


def test_faster_than_bookshelf_text(tmp_path):
    nl = synth.blob_start(synth.standard_cell(20000, seed=6))
    aux = synth.write_bookshelf(nl, str(tmp_path / "bs"))
    p = netbin.write(nl, str(tmp_path / "d.epn"))
    t0 = time.perf_counter()
    bookshelf.read_aux(aux, target_density=nl.target_density)
    t_text = time.perf_counter() - t0
    t0 = time.perf_counter()
    placer.netbin_read(p)
    t_bin = time.perf_counter() - t0
    assert t_bin * 10 < t_text, (t_bin, t_text)
