"""The native Bookshelf reader and .pl writer (ep_bookshelf_read /
ep_bookshelf_write_pl, csrc/bookshelf.cu) on the CPU: array for array equal
to the Python reader (eplace_b200/bookshelf.py, which states the rules of
Parser/parser.cpp:44-819 the placer depends on) on generated designs and on a
hand-written one with the format's corner cases; errors reported, not
crashed on; .pl positions written at full precision read back as the same
floats; faster than the Python reader."""
import time

import numpy as np
import pytest

from eplace_b200 import bookshelf, placer, synth

ARRAYS = ("node_w", "node_h", "node_cx", "node_cy", "term_llx", "term_lly", "term_w", "term_h", "term_is_ni",
          "net_start", "pin_owner", "pin_dx", "pin_dy", "row_llx", "row_lly", "row_urx", "row_h", "row_site_w")


def assert_same(a, b):
    for k in ARRAYS:
        x, y = np.asarray(getattr(a, k)), np.asarray(getattr(b, k))
        assert x.shape == y.shape, k
        assert np.array_equal(x.astype(y.dtype), y), k


@pytest.mark.parametrize("make", [lambda: synth.mixed_size(1500, 4, 6, seed=3),
                                  lambda: synth.standard_cell(5000, seed=11)])
def test_native_reader_matches_python_reader(tmp_path, make):
    nl = make()
    aux = synth.write_bookshelf(nl, str(tmp_path))
    with placer.BookshelfDesign(aux) as bd:
        assert_same(bd.netlist, bookshelf.read_aux(aux))
        assert_same(bd.netlist, nl)


def _write(d, name, text):
    (d / name).write_text(text)


CORNER = dict(
    aux="RowBasedPlacement :  c.nodes  c.nets c.wts c.pl c.scl\n",
    nodes="UCLA nodes 1.0\n# comment\n\nNumNodes : 6\nNumTerminals : 2\n"
          "  a   4 12\nb 2.5 12\r\nP1 1 1 terminal\nc 3e0 +12\nP2 2 3 terminal_NI\nd 8 24\n",
    nets="UCLA nets 1.0\nNumNets : 3\nNumPins : 7\n\n"
         "NetDegree : 3 n0\n a I : 0.5 -1.25\n b O:1 2\n P1 B\n"
         "NetDegree : 2\nc B : -0.75 0\nd I : 1\n"
         "# comment between nets\nNetDegree : 2 n2\nP2 O : 0 0\na B : 2 3\n",
    pl="UCLA pl 1.0\n\na 10 24 : N\nb\t20.5   0 : FS\nc (30,36) : N\nP1 = 0, 0 : N /FIXED\n"
       "P2 50 60 : N /FIXED_NI\nghost 1 2 : N\n# d is not placed: it stays at 0 0\n",
    scl="UCLA scl 1.0\nNumRows : 3\n\nCoreRow Horizontal\n Coordinate : 0\n Height : 12\n Sitewidth : 0.5\n"
        " Sitespacing : 0.5\n SubrowOrigin : 2 Numsites : 100\nEnd\nCoreRow Horizontal\n Coordinate : 12\n"
        " Height : 12\n SubrowOrigin : 2 NumSites : 90\nEnd\nCoreRow Horizontal\n Coordinate : 24\n Height : 12\n"
        " Sitewidth : 1\n SubrowOrigin : 0 Numsites : 40\nEnd\n",
    wts="UCLA wts 1.0\n")


def test_native_reader_format_corner_cases(tmp_path):
    for ext, text in CORNER.items():
        _write(tmp_path, "c." + ext, text)
    aux = str(tmp_path / "c.aux")
    py = bookshelf.read_aux(aux)
    with placer.BookshelfDesign(aux) as bd:
        nl = bd.netlist
        assert_same(nl, py)
    # the values the rules give, spelled out
    assert nl.num_nodes == 4 and nl.num_terminals == 2 and nl.num_nets == 3
    assert list(nl.term_is_ni) == [0, 1]
    assert list(nl.net_start) == [0, 3, 5, 7]
    assert list(nl.pin_owner) == [0, 1, 4, 2, 3, 5, 0]
    assert list(nl.pin_dx) == [0.5, 1, 0, -0.75, 1, 0, 2] and list(nl.pin_dy) == [-1.25, 2, 0, 0, 0, 0, 3]
    assert list(nl.node_cx) == [12, 21.75, 31.5, 4] and list(nl.node_cy) == [30, 6, 42, 12]
    assert list(nl.term_llx) == [0, 50] and list(nl.term_lly) == [0, 60]
    assert list(nl.row_llx) == [2, 2, 0] and list(nl.row_urx) == [52, 47, 40]  # site width 0.5 carried over
    assert list(nl.row_lly) == [0, 12, 24] and list(nl.row_h) == [12, 12, 12]


@pytest.mark.parametrize("ext,text,needle", [
    ("nets", "UCLA nets 1.0\nNetDegree : 1\nnobody B : 0 0\n", "unknown node 'nobody'"),
    ("nets", "UCLA nets 1.0\nNetDegree : 3\na B\nb B\n", "ends before"),
    ("nets", "UCLA nets 1.0\nbogus line\n", "unsupported line"),
    ("nodes", "UCLA nodes 1.0\na 4 x12\n", "bad number 'x12'"),
    ("scl", "UCLA scl 1.0\n Height : 12\n", "before the first CoreRow"),
])
def test_native_reader_reports_errors(tmp_path, ext, text, needle):
    for e, t in CORNER.items():
        _write(tmp_path, "c." + e, text if e == ext else t)
    with pytest.raises(placer.EPError) as ex:
        placer.BookshelfDesign(str(tmp_path / "c.aux"))
    assert ex.value.status == placer.EP_ERR_ARG
    assert needle in str(ex.value)


def test_native_reader_missing_files(tmp_path):
    with pytest.raises(placer.EPError) as ex:
        placer.BookshelfDesign(str(tmp_path / "none.aux"))
    assert "cannot read" in str(ex.value)
    _write(tmp_path, "c.aux", "RowBasedPlacement : c.nodes c.pl c.scl\n")
    with pytest.raises(placer.EPError) as ex:
        placer.BookshelfDesign(str(tmp_path / "c.aux"))
    assert "no .nets file" in str(ex.value)


def test_write_pl_round_trips_floats(tmp_path):
    nl = synth.mixed_size(1200, 3, 4, seed=5)
    aux = synth.write_bookshelf(nl, str(tmp_path))
    rng = np.random.default_rng(1)
    cx = (rng.random(nl.num_nodes) * 1e4 + 1 / 3).astype(np.float32)
    cy = (rng.random(nl.num_nodes) * 1e4 + 1 / 7).astype(np.float32)
    with placer.BookshelfDesign(aux) as bd:
        bd.write_pl(str(tmp_path / (nl.name + ".pl")), cx, cy)  # replaces the design's .pl
    with placer.BookshelfDesign(aux) as bd:
        back = bd.netlist
    half_w, half_h = np.float32(0.5) * nl.node_w, np.float32(0.5) * nl.node_h
    # the corner written is cx - w/2 in float; read back, + w/2 in float
    assert np.array_equal(back.node_cx, (cx - half_w) + half_w)
    assert np.array_equal(back.node_cy, (cy - half_h) + half_h)
    assert np.array_equal(back.term_llx, nl.term_llx) and np.array_equal(back.term_lly, nl.term_lly)
    text = (tmp_path / (nl.name + ".pl")).read_text()
    assert "/FIXED_NI" in text or not nl.term_is_ni.any()


def test_native_reader_faster_than_python(tmp_path):
    nl = synth.standard_cell(40_000, seed=4)
    aux = synth.write_bookshelf(nl, str(tmp_path))
    t0 = time.perf_counter()
    bookshelf.read_aux(aux)
    t_py = time.perf_counter() - t0
    t0 = time.perf_counter()
    with placer.BookshelfDesign(aux):
        pass
    t_native = time.perf_counter() - t0
    assert t_native * 3 < t_py, (t_native, t_py)


def test_native_writer_matches_python_writer(tmp_path):
    nl = synth.mixed_size(1500, 4, 6, seed=8)
    synth.write_bookshelf(nl, str(tmp_path / "py"))
    placer.bookshelf_write(nl, str(tmp_path / "native"))
    for ext in ("aux", "nodes", "nets", "wts", "pl", "scl"):
        f = f"{nl.name}.{ext}"
        assert (tmp_path / "native" / f).read_bytes() == (tmp_path / "py" / f).read_bytes(), ext


def test_read_write_round_trip_keeps_names_and_site_widths(tmp_path):
    for ext, text in CORNER.items():
        _write(tmp_path, "c." + ext, text)
    with placer.BookshelfDesign(str(tmp_path / "c.aux")) as bd:
        first = bd.netlist
        aux = bd.write(str(tmp_path / "out"), "c")
    with placer.BookshelfDesign(aux) as bd:
        assert_same(bd.netlist, first)
    nodes = (tmp_path / "out" / "c.nodes").read_text().split("\n")
    assert nodes[3:9] == ["a 4 12", "b 2.5 12", "c 3 12", "d 8 24", "P1 1 1 terminal", "P2 2 3 terminal_NI"]
    scl = (tmp_path / "out" / "c.scl").read_text()
    assert scl.count("Sitewidth : 0.5") == 2 and scl.count("Sitewidth : 1\n") == 1
    assert "SubrowOrigin : 2 Numsites : 90" in scl


def test_native_writer_faster_than_python(tmp_path):
    nl = synth.standard_cell(40_000, seed=4)
    t0 = time.perf_counter()
    synth.write_bookshelf(nl, str(tmp_path / "py"))
    t_py = time.perf_counter() - t0
    t0 = time.perf_counter()
    placer.bookshelf_write(nl, str(tmp_path / "native"))
    t_native = time.perf_counter() - t0
    assert t_native * 3 < t_py, (t_native, t_py)


def test_native_reader_agrees_with_reference_parser(tmp_path):
    """Against BookshelfParser::ReadFile itself (the reference compiled from
    its sources into oracle/_ref): the same counts, node centres bit for bit,
    and the same HPWL (PlaceDB::calcHPWL) as pins at owner centre + offset on
    the native arrays."""
    from oracle import refharness as R
    if not R.available():
        pytest.skip("the reference build (oracle/_ref) is not present")
    nl = synth.mixed_size(3000, 5, 8, seed=2)
    aux = synth.write_bookshelf(nl, str(tmp_path))
    ref = R.RefPlacer(aux=aux)
    with placer.BookshelfDesign(aux) as bd:
        n = bd.netlist
    assert (ref.num_nodes, ref.num_terminals, ref.num_nets, ref.num_pins, ref.num_rows) == \
        (n.num_nodes, n.num_terminals, n.num_nets, n.num_pins, n.num_rows)
    cx, cy = ref.node_centers()
    assert np.array_equal(cx, n.node_cx) and np.array_equal(cy, n.node_cy)
    tcx = n.term_llx + np.float32(0.5) * n.term_w
    tcy = n.term_lly + np.float32(0.5) * n.term_h
    ox, oy = np.concatenate([n.node_cx, tcx]), np.concatenate([n.node_cy, tcy])
    px = (ox[n.pin_owner] + n.pin_dx).astype(np.float64)
    py = (oy[n.pin_owner] + n.pin_dy).astype(np.float64)
    seg = n.net_start[:-1]
    deg = np.diff(n.net_start)
    hp = ((np.maximum.reduceat(px, seg) - np.minimum.reduceat(px, seg)) +
          (np.maximum.reduceat(py, seg) - np.minimum.reduceat(py, seg)))[deg >= 2].sum()
    assert hp == pytest.approx(ref.hpwl(), rel=1e-7)
    ref.close()
