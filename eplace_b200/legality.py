"""Exact-integer legality check of a placement after legalization.

The reference legalizes on the CPU (SAMacroLegalizer for macros,
AbacusLegalizer + DetailedPlacer for standard cells, main/ePlace_main.cpp:
174-279) and places every object on float coordinates.  This checker turns
every coordinate into an integer exactly -- all values are float32, hence
dyadic rationals, so one power-of-two scale makes each of them an integer in
int64 without rounding (it refuses values for which no scale up to 2^40
keeps every scaled value below 2^60) -- and then tests, in integers only:

  * row membership: a standard cell's bottom edge equals the bottom of a
    site row, its height the row's height, and its extent lies inside the
    row's [llx, urx);
  * site alignment: (x - row.llx) is a whole number of sites, and so is the
    cell's width;
  * no overlap: inside each row, cells sorted by x have x_i + w_i <= x_(i+1);
    no standard cell overlaps a fixed object (a terminal of non-zero area or
    a macro given as fixed) or a macro; no two macros overlap;
  * macros (cells taller than one row) lie inside the core.

Overlap of two rectangles is the usual strict test (they may touch).
"""
import numpy as np

MAX_SCALE_BITS = 40
MAX_SCALED = 2.0 ** 60


class Rects:
    """Axis-aligned rectangles as exact int64 (x0, y0, x1, y1) after scaling."""

    def __init__(self, x0, y0, x1, y1):
        self.x0, self.y0, self.x1, self.y1 = x0, y0, x1, y1

    def __len__(self):
        return len(self.x0)


def _scale_bits(*arrays):
    """Smallest s <= MAX_SCALE_BITS such that every value times 2^s is an
    integer below 2^60 in magnitude (int64 holds it and sums of two)."""
    vals = np.concatenate([np.asarray(a, np.float64).ravel() for a in arrays if np.size(a)])
    if not np.all(np.isfinite(vals)):
        raise ValueError("non-finite coordinate")
    for s in range(MAX_SCALE_BITS + 1):
        v = vals * float(2 ** s)  # exact: float32 values, power-of-two factor
        if np.abs(v).max(initial=0.0) >= MAX_SCALED:
            break
        if np.all(v == np.floor(v)):
            return s
    raise ValueError("coordinates have no exact int64 scale")


def _ints(a, s):
    # a float32 value has at most 24 significant bits, so times 2^s it is
    # exact in float64 at any magnitude, and below 2^60 exact in int64
    return (np.asarray(a, np.float32).astype(np.float64) * float(2 ** s)).astype(np.int64)


def _overlap_pairs(a, b, same=False):
    """Index pairs (i, j) with rectangle a_i overlapping b_j (interiors
    intersect), by a sweep over x; same=True counts each unordered pair of one
    set once."""
    out = []
    if len(a) == 0 or len(b) == 0:
        return out
    if not same and len(a) > len(b):  # sweep the smaller set
        return [(i, j) for j, i in _overlap_pairs(b, a)]
    order_b = np.argsort(b.x0, kind="stable")
    bx0 = b.x0[order_b]
    for i in range(len(a)):
        hi = np.searchsorted(bx0, a.x1[i], side="left")  # b.x0 < a.x1
        cand = order_b[:hi]
        m = (b.x1[cand] > a.x0[i]) & (b.y0[cand] < a.y1[i]) & (b.y1[cand] > a.y0[i])
        for j in cand[m]:
            if same and j <= i:
                continue
            out.append((i, int(j)))
    return out


def check(nl, cx, cy, fixed_macro=None, max_report=10, macros_only=False, macros_vs_fixed=True):
    """Legality of movable-node centres (cx, cy) on netlist nl.

    fixed_macro: optional bool array over nodes marking macros that count as
    fixed obstacles (they are checked for overlap with one another and with
    the cells but not for row alignment).  Movable nodes taller than one row
    are macros.  macros_only: only the macro tests (after macro legalization,
    before the cells are legalized).  macros_vs_fixed=False leaves out the
    overlap of movable macros with fixed objects (counted apart, as
    "macro_fixed_overlap"): the reference's SA macro legalizer does not see
    the fixed objects (Legalization/legalizer.h:305-307).  Returns a dict: counts
    per violation kind, the first few offending node indices per kind, and
    legal (no violation at all)."""
    n = nl.num_nodes
    cx = np.asarray(cx, np.float32)[:n]
    cy = np.asarray(cy, np.float32)[:n]
    w = np.asarray(nl.node_w, np.float32)
    h = np.asarray(nl.node_h, np.float32)
    llx = (cx.astype(np.float64) - w.astype(np.float64) / 2).astype(np.float32)
    lly = (cy.astype(np.float64) - h.astype(np.float64) / 2).astype(np.float32)
    # the lower-left corners as float32, as the reference keeps them; the
    # centre minus half the width is exact when both are (they are dyadic)
    if not (np.array_equal(llx.astype(np.float64) + w / 2.0, cx.astype(np.float64)) and
            np.array_equal(lly.astype(np.float64) + h / 2.0, cy.astype(np.float64))):
        raise ValueError("centres and sizes do not give exact float32 corners")
    rows = (np.asarray(nl.row_llx, np.float32), np.asarray(nl.row_lly, np.float32),
            np.asarray(nl.row_urx, np.float32), np.asarray(nl.row_h, np.float32),
            np.asarray(nl.row_site_w, np.float32))
    tw, th = np.asarray(nl.term_w, np.float32), np.asarray(nl.term_h, np.float32)
    tx, ty = np.asarray(nl.term_llx, np.float32), np.asarray(nl.term_lly, np.float32)
    s = _scale_bits(llx, lly, w, h, tx, ty, tw, th, *rows)
    X, Y, W, H = _ints(llx, s), _ints(lly, s), _ints(w, s), _ints(h, s)
    RX, RY, RU, RH, RS = (_ints(r, s) for r in rows)
    if np.any(RS <= 0) or np.any(RH <= 0):
        raise ValueError("rows need positive height and site width")
    macro = H > RH.min()
    if fixed_macro is not None:
        macro = macro | np.asarray(fixed_macro, bool)[:n]
    cell = ~macro & (not macros_only)
    bad = {k: [] for k in ("off_row", "row_height", "outside_row", "off_site", "width_sites",
                           "overlap", "fixed_overlap", "macro_overlap", "outside_core")}
    # row membership: the row whose bottom is the cell's bottom
    row_of_y = {int(y): r for r, y in enumerate(RY)}
    row = np.full(n, -1, np.int64)
    for i in np.flatnonzero(cell):
        r = row_of_y.get(int(Y[i]), -1)
        if r < 0:
            bad["off_row"].append(int(i))
            continue
        row[i] = r
        if H[i] != RH[r]:
            bad["row_height"].append(int(i))
        if X[i] < RX[r] or X[i] + W[i] > RU[r]:
            bad["outside_row"].append(int(i))
        if (X[i] - RX[r]) % RS[r] != 0:
            bad["off_site"].append(int(i))
        if W[i] % RS[r] != 0:
            bad["width_sites"].append(int(i))
    # overlap inside rows
    for r in np.unique(row[row >= 0]):
        idx = np.flatnonzero(row == r)
        idx = idx[np.argsort(X[idx], kind="stable")]
        ends = X[idx[:-1]] + W[idx[:-1]]
        for k in np.flatnonzero(ends > X[idx[1:]]):
            bad["overlap"].append(int(idx[k + 1]))
    cells = Rects(X[cell], Y[cell], X[cell] + W[cell], Y[cell] + H[cell])
    cell_idx = np.flatnonzero(cell)
    # fixed obstacles: terminals of non-zero area, and the macros
    TX, TY, TW, TH = _ints(tx, s), _ints(ty, s), _ints(tw, s), _ints(th, s)
    solid = (TW > 0) & (TH > 0)
    terms = Rects(TX[solid], TY[solid], TX[solid] + TW[solid], TY[solid] + TH[solid])
    for i, _ in _overlap_pairs(cells, terms):
        bad["fixed_overlap"].append(int(cell_idx[i]))
    mac_idx = np.flatnonzero(macro)
    macs = Rects(X[macro], Y[macro], X[macro] + W[macro], Y[macro] + H[macro])
    for i, _ in _overlap_pairs(cells, macs):
        bad["fixed_overlap"].append(int(cell_idx[i]))
    for i, j in _overlap_pairs(macs, macs, same=True):
        bad["macro_overlap"].append(int(mac_idx[j]))
    vs_fixed = [int(mac_idx[i]) for i, _ in _overlap_pairs(macs, terms)]
    if macros_vs_fixed:
        bad["macro_overlap"] += vs_fixed
    core_x0, core_y0 = RX.min(), RY.min()
    core_x1, core_y1 = RU.max(), (RY + RH).max()
    for i in mac_idx:
        if X[i] < core_x0 or Y[i] < core_y0 or X[i] + W[i] > core_x1 or Y[i] + H[i] > core_y1:
            bad["outside_core"].append(int(i))
    out = {"legal": not any(bad.values()), "scale_bits": s, "cells": int(cell.sum()), "macros": int(macro.sum()),
           "macro_fixed_overlap": len(set(vs_fixed))}
    for k, v in bad.items():
        out[k] = len(set(v))
        out[k + "_first"] = sorted(set(v))[:max_report]
    return out


def assert_legal(nl, cx, cy, **kw):
    r = check(nl, cx, cy, **kw)
    if not r["legal"]:
        raise AssertionError({k: v for k, v in r.items() if v and not k.endswith("_first") or k == "legal"} |
                             {k: v for k, v in r.items() if k.endswith("_first") and v})
    return r
