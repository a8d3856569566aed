"""The C-ABI as C and C++ callers see it: small programs compiled against
include/ and linked with the built library.

* A C99 program (include/eplace_gpu.h only) reads a Bookshelf design with
  ep_bookshelf_read, stores and maps it as a binary netlist
  (ep_netbin_write / ep_netbin_open), writes a .pl (ep_bookshelf_write_pl)
  and prints what it saw; these entry points are host code, so it runs
  without a GPU.
* A C++17 program uses the adapter include/eplace_b200.hpp with the
  reference's call sequence (EPlacer2D, initialization, EplaceNesterovOpt::opt,
  getPosition); without a GPU the constructor throws the engine's
  EP_ERR_CUDA error (no CPU fallback), with one it places the design."""
import os
import subprocess

import numpy as np
import pytest

from eplace_b200 import placer, synth
from tests.conftest import HAS_GPU

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "eplace_b200")

C_PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include "eplace_gpu.h"

int main(int argc, char **argv) {
    ep_netlist nl, nb;
    void *design = NULL, *bin = NULL;
    char err[256];
    float td = 0.f;
    int32_t bins = -1;
    ep_status s;
    float *cx, *cy;
    int k;
    if (argc < 4) return 2;
    if (ep_abi_version() < 1) return 3;
    s = ep_bookshelf_read(argv[1], &nl, &design, err, (int32_t)sizeof err);
    if (s != EP_OK) { printf("read failed %d: %s\n", (int)s, err); return 4; }
    printf("nodes %d terminals %d nets %d rows %d pins %d\n", nl.num_nodes, nl.num_terminals, nl.num_nets,
           nl.num_rows, nl.net_start[nl.num_nets]);
    if (ep_netbin_write(argv[2], &nl, 0.9f, 0) != EP_OK) return 5;
    if (ep_netbin_open(argv[2], &nb, &td, &bins, &bin) != EP_OK) return 6;
    for (k = 0; k < nl.num_nodes; k++)
        if (nb.node_cx[k] != nl.node_cx[k] || nb.node_w[k] != nl.node_w[k]) return 7;
    printf("netbin density %.2f bins %d\n", td, bins);
    cx = (float *)malloc(sizeof(float) * (size_t)nl.num_nodes);
    cy = (float *)malloc(sizeof(float) * (size_t)nl.num_nodes);
    for (k = 0; k < nl.num_nodes; k++) { cx[k] = nl.node_cx[k] + 1.0f; cy[k] = nl.node_cy[k]; }
    s = ep_bookshelf_write_pl(design, argv[3], cx, cy);
    ep_netbin_close(bin);
    ep_bookshelf_close(design);
    free(cx);
    free(cy);
    printf("pl written %d\n", (int)s);
    return s == EP_OK ? 0 : 8;
}
"""

CPP_PROGRAM = r"""
#include <cstdio>
#include "eplace_b200.hpp"

int main(int argc, char **argv) {
    ep_netlist nl;
    void *design = nullptr;
    char err[256];
    if (ep_bookshelf_read(argv[1], &nl, &design, err, sizeof err) != EP_OK) return 4;
    ep_params prm;
    ep_default_params(&prm);
    int rc = 0;
    try {
        eplace_b200::EPlacer2D eplacer(nl, prm);
        eplacer.initialization();
        eplace_b200::EplaceNesterovOpt opt(&eplacer);
        ep_run_stats st = opt.opt();
        std::vector<eplace_b200::Vec2> xy = eplacer.getPosition();
        std::printf("placed %d iterations, overflow %.3f, %zu positions\n", st.iterations, st.overflow, xy.size());
    } catch (const eplace_b200::Error &e) {
        std::printf("engine error %d: %s\n", (int)e.status, e.what());
        rc = e.status == EP_ERR_CUDA ? 0 : 9;
    }
    ep_bookshelf_close(design);
    return rc;
}
"""


def _build(tmp_path, src, name, compiler, std):
    path = tmp_path / name
    (tmp_path / (name + (".c" if compiler == "gcc" else ".cpp"))).write_text(src)
    cmd = [compiler, f"-std={std}", "-Wall", "-Werror", "-I" + INC, str(path) + (".c" if compiler == "gcc" else ".cpp"),
           "-L" + LIBDIR, "-leplace_b200", "-Wl,-rpath," + LIBDIR, "-o", str(path)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return str(path)


@pytest.fixture(scope="module")
def design(tmp_path_factory):
    placer.load()  # the built library
    d = tmp_path_factory.mktemp("cabi")
    nl = synth.mixed_size(600, 2, 2, seed=4)
    return nl, synth.write_bookshelf(nl, str(d)), d


def test_c_program_reads_stores_and_writes(design, tmp_path):
    nl, aux, d = design
    exe = _build(tmp_path, C_PROGRAM, "cprog", "gcc", "c99")
    out_pl = tmp_path / "moved.pl"
    r = subprocess.run([exe, aux, str(tmp_path / "x.netbin"), str(out_pl)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert f"nodes {nl.num_nodes} terminals {nl.num_terminals} nets {nl.num_nets}" in r.stdout
    assert "netbin density 0.90 bins 0" in r.stdout
    lines = out_pl.read_text().splitlines()
    assert lines[0] == "UCLA pl 1.0" and len(lines) == 2 + nl.num_nodes + nl.num_terminals
    name, x, y = lines[2].split()[:3]
    assert name == "o0"
    assert np.float32(float(x)) == (nl.node_cx[0] + np.float32(1)) - np.float32(0.5) * nl.node_w[0]


def test_cpp_adapter_follows_the_reference_call_sequence(design, tmp_path):
    nl, aux, d = design
    exe = _build(tmp_path, CPP_PROGRAM, "cppprog", "g++", "c++17")
    r = subprocess.run([exe, aux], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    if HAS_GPU:
        assert "placed" in r.stdout
    else:
        assert "engine error 2" in r.stdout and "no CPU fallback" in r.stdout
