"""The exact-integer legality checker (eplace_b200/legality.py): placements
built by hand, legal and with one planted violation of each kind, and the
reference's own CPU flow on the config-1 smoke design -- QPPlacer, mGP,
AbacusLegalizer, DetailedPlacer (main/ePlace_main.cpp:174-279, through the
compiled reference) -- whose legalized output the checker must accept."""
import copy

import numpy as np
import pytest

from eplace_b200 import legality, synth
from oracle import refharness as R


def packed(nl):
    """Cells packed left to right, row by row, one site apart."""
    cx, cy = np.zeros(nl.num_nodes, np.float32), np.zeros(nl.num_nodes, np.float32)
    r, x = 0, 0.0
    for i in range(nl.num_nodes):
        w = float(nl.node_w[i])
        if x + w > float(nl.row_urx[r]):
            r, x = r + 1, 0.0
        cx[i], cy[i] = x + w / 2, float(nl.row_lly[r]) + 0.5
        x += w + 1.0
    return cx, cy


def test_hand_built_legal_placement():
    nl = synth.smoke(3)
    cx, cy = packed(nl)
    r = legality.check(nl, cx, cy)
    assert r["legal"], r
    assert r["cells"] == nl.num_nodes and r["macros"] == 0


@pytest.mark.parametrize("kind", ["off_site", "off_row", "overlap", "outside_row", "fixed_overlap"])
def test_each_planted_violation_is_found(kind):
    nl = copy.copy(synth.smoke(3))
    cx, cy = packed(nl)
    if kind == "off_site":
        cx[5] += 0.5
    elif kind == "off_row":
        cy[5] += 0.25
    elif kind == "overlap":
        # cell 6 starts on cell 5's last site (same row, still on sites)
        x5 = cx[5] - float(nl.node_w[5]) / 2
        cx[6], cy[6] = x5 + float(nl.node_w[5]) - 1.0 + float(nl.node_w[6]) / 2, cy[5]
    elif kind == "outside_row":
        cx[5] = float(nl.row_urx[0]) - float(nl.node_w[5]) / 2 + 1.0
    elif kind == "fixed_overlap":
        # a 2 x 2 fixed block where cell 5 sits
        nl.term_w = nl.term_w.copy()
        nl.term_h = nl.term_h.copy()
        nl.term_llx = nl.term_llx.copy()
        nl.term_lly = nl.term_lly.copy()
        nl.term_w[0], nl.term_h[0] = 2.0, 2.0
        nl.term_llx[0], nl.term_lly[0] = cx[5] - 1.0, cy[5] - 1.0
    r = legality.check(nl, cx, cy)
    assert not r["legal"] and r[kind] >= 1, r
    others = [k for k in ("off_site", "off_row", "overlap", "outside_row", "fixed_overlap", "macro_overlap",
                          "outside_core", "row_height", "width_sites") if k != kind and r[k]]
    if kind != "outside_row":
        assert not others, r


def test_inexact_coordinates_are_refused():
    nl = synth.smoke(3)
    cx, cy = packed(nl)
    cx[0] = np.float32(1e-30)  # no exact int64 scale keeps the die below 2^60
    assert cx[0] != packed(nl)[0][0]
    with pytest.raises(ValueError):
        legality.check(nl, cx, cy)


@pytest.mark.skipif(not R.available(), reason="reference harness not built")
def test_reference_flow_output_is_legal():
    nl = synth.smoke(1)
    ref = R.RefPlacer(nl)
    ref.qp()
    ref.initialization(nl.target_density)
    ref.opt_run()
    hpwl_gp = ref.hpwl()
    ref.abacus()
    cx, cy = ref.node_centers()
    r = legality.check(nl, cx, cy)
    assert r["legal"], r
    hpwl_lg = ref.hpwl()
    ref.detailed()
    cx, cy = ref.node_centers()
    assert legality.check(nl, cx, cy)["legal"]
    assert ref.hpwl() <= hpwl_lg  # detailed placement only improves
    assert hpwl_lg >= hpwl_gp * 0.9
    ref.close()
