"""Seeded synthetic Bookshelf-style netlists for the ePlace global-placement path.

No public benchmark suite is shipped or used: these generators stand in for
the design shapes the engine is measured on.  Every array is produced from a
``numpy.random.Generator`` seeded by the caller, so a (generator, seed) pair
names a design exactly.

Conventions follow the reference data model (PlaceDB/placedb.h:52-185,
PlaceCommon/objects.h:32-229):
  * movable nodes (std cells, movable macros) come first; a node is a macro
    iff its height exceeds the common row height (PlaceDB/placedb.cpp:96-114);
  * terminals are fixed; ``term_is_ni`` marks "terminal_NI" pins, which are
    left out of the whitespace computation (EPlace/eplace.cpp:68-92);
  * pins are listed net by net (a CSR ``net_start``), each with an owner and
    an offset from the owner's centre (Pin::calculateAbsolutePos,
    PlaceCommon/objects.cpp:454-459);
  * rows are [row_llx, row_urx] x [row_lly, row_lly + row_h].
"""
from dataclasses import dataclass, field
import math

import numpy as np


@dataclass
class Netlist:
    name: str
    node_w: np.ndarray
    node_h: np.ndarray
    node_cx: np.ndarray
    node_cy: np.ndarray
    term_llx: np.ndarray
    term_lly: np.ndarray
    term_w: np.ndarray
    term_h: np.ndarray
    term_is_ni: np.ndarray
    net_start: np.ndarray
    pin_owner: np.ndarray
    pin_dx: np.ndarray
    pin_dy: np.ndarray
    row_llx: np.ndarray
    row_lly: np.ndarray
    row_urx: np.ndarray
    row_h: np.ndarray
    row_site_w: np.ndarray
    target_density: float = 1.0
    bins: int = 0  # 0 = the reference's automatic rule
    meta: dict = field(default_factory=dict)

    @property
    def num_nodes(self):
        return int(self.node_w.shape[0])

    @property
    def num_terminals(self):
        return int(self.term_w.shape[0])

    @property
    def num_nets(self):
        return int(self.net_start.shape[0] - 1)

    @property
    def num_pins(self):
        return int(self.pin_owner.shape[0])

    @property
    def num_rows(self):
        return int(self.row_h.shape[0])

    def core(self):
        return (float(self.row_llx.min()), float(self.row_lly.min()),
                float(self.row_urx.max()), float((self.row_lly + self.row_h).max()))

    def with_positions(self, cx, cy):
        import copy
        n = copy.copy(self)
        n.node_cx = np.ascontiguousarray(cx, dtype=np.float32)
        n.node_cy = np.ascontiguousarray(cy, dtype=np.float32)
        return n

    def validate(self):
        assert self.net_start[0] == 0 and self.net_start[-1] == self.num_pins
        assert np.all(np.diff(self.net_start) >= 1)
        assert self.pin_owner.min() >= 0
        assert self.pin_owner.max() < self.num_nodes + self.num_terminals
        assert np.all(self.node_w > 0) and np.all(self.node_h > 0)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _rows(side, row_h=1.0):
    n = int(round(side / row_h))
    return dict(
        row_llx=_f32(np.zeros(n)), row_lly=_f32(np.arange(n) * row_h),
        row_urx=_f32(np.full(n, side)), row_h=_f32(np.full(n, row_h)),
        row_site_w=_f32(np.ones(n)))


def fit_powerlaw_alpha(mean, dmin=2, dmax=500):
    """alpha such that P(d) ~ d^-alpha on [dmin, dmax] has the given mean."""
    d = np.arange(dmin, dmax + 1, dtype=np.float64)

    def m(a):
        w = d ** -a
        return float((d * w).sum() / w.sum())

    lo, hi = 1.01, 6.0
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        if m(mid) > mean:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def _powerlaw_degrees(rng, n, alpha, dmin=2, dmax=500):
    d = np.arange(dmin, dmax + 1)
    w = d.astype(np.float64) ** -alpha
    return rng.choice(d, size=n, p=w / w.sum()).astype(np.int64)


def _pad_ring(nt, side):
    """Lower-left corners of ``nt`` 1x1 pads evenly spaced on a ring just
    outside a square core [0, side]^2."""
    t = (np.arange(nt) + 0.5) / nt * 4.0
    edge = np.floor(t).astype(int)
    f = t - edge
    tx = np.select([edge == 0, edge == 1, edge == 2, edge == 3], [f * side, side + 1.0, (1 - f) * side, -2.0])
    ty = np.select([edge == 0, edge == 1, edge == 2, edge == 3], [-2.0, f * side, side + 1.0, (1 - f) * side])
    return tx, ty


def _offsets(rng, owner, w, h):
    dx = (rng.random(owner.shape[0]) - 0.5) * w[owner]
    dy = (rng.random(owner.shape[0]) - 0.5) * h[owner]
    return dx, dy


def smoke(seed=1):
    """Smoke-size design: 100 cells (h = 1 row, w ~ U{1..4} sites), 4 fixed
    I/O pins at the die-edge midpoints, 184 nets with degree 2 (60%),
    3 (25%), 4-6 (15%) whose pins are drawn uniformly from cells and I/O
    pins with uniform offsets inside the cell, a square die at 60%
    utilisation, targetDensity 0.8, 16x16 bins."""
    rng = np.random.default_rng(seed)
    nc, nt, nn = 100, 4, 184
    w = rng.integers(1, 5, nc).astype(np.float64)
    h = np.ones(nc)
    side = float(math.ceil(math.sqrt(w.sum() / 0.6)))
    rows = _rows(side)
    tx = np.array([side / 2, side, side / 2, 0.0])
    ty = np.array([0.0, side / 2, side, side / 2])
    u = rng.random(nn)
    deg = np.where(u < 0.6, 2, np.where(u < 0.85, 3, rng.integers(4, 7, nn)))
    owners = []
    for d in deg:
        owners.append(rng.choice(nc + nt, size=int(d), replace=False))
    owner = np.concatenate(owners)
    ww = np.concatenate([w, np.zeros(nt)])
    hh = np.concatenate([h, np.zeros(nt)])
    dx, dy = _offsets(rng, owner, ww, hh)
    return Netlist(
        name=f"smoke_s{seed}", node_w=_f32(w), node_h=_f32(h),
        node_cx=_f32(np.full(nc, side / 2)), node_cy=_f32(np.full(nc, side / 2)),
        term_llx=_f32(tx), term_lly=_f32(ty), term_w=_f32(np.zeros(nt)), term_h=_f32(np.zeros(nt)),
        term_is_ni=np.ones(nt, np.uint8), net_start=_i32(np.concatenate([[0], np.cumsum(deg)])),
        pin_owner=_i32(owner), pin_dx=_f32(dx), pin_dy=_f32(dy), target_density=0.8, bins=16,
        meta=dict(generator="smoke", seed=seed), **rows)


def _morton_home(idx, n):
    """Home of cell ``idx`` (of ``n``) in the unit square: the cell's place in
    the index order read as a Morton (Z-order) code, so that every aligned
    index range of the cluster hierarchy maps to one compact region (x from
    the even bits, y from the odd bits of a 20-bit code)."""
    code = ((np.asarray(idx, np.float64) + 0.5) / n * (1 << 20)).astype(np.int64)
    x = np.zeros(code.shape, np.float64)
    y = np.zeros(code.shape, np.float64)
    for b in range(10):
        x += ((code >> (2 * b + 1)) & 1) * 2.0 ** (b - 10)
        y += ((code >> (2 * b)) & 1) * 2.0 ** (b - 10)
    return x + 2.0 ** -11, y + 2.0 ** -11


def _nearest_pads(hx, hy, nt, rng, spread=2):
    """Pad index nearest to each home point (unit square), by the pad ring's
    parameter of the closest core edge (the ring order of ``_pad_ring``:
    bottom, right, top, left), plus a seeded offset of up to ``spread`` pads."""
    d = np.stack([hy, 1.0 - hx, 1.0 - hy, hx])  # distance to bottom, right, top, left
    edge = np.argmin(d, axis=0)
    f = np.select([edge == 0, edge == 1, edge == 2, edge == 3], [hx, hy, 1.0 - hx, 1.0 - hy])
    u = (edge + f) / 4.0
    k = np.floor(u * nt).astype(np.int64) + rng.integers(-spread, spread + 1, hx.shape[0])
    return np.mod(k, nt)


def standard_cell(num_cells=200_000, num_nets=None, num_terminals=None, seed=7,
                  utilisation=0.7, target_density=1.0, mean_degree=3.6, max_degree=500,
                  rent_p=0.6, leaf_cluster=8, terminal_net_fraction=0.05, bins=0,
                  every_cell_pinned=False, local_pads=False):
    """Standard-cell design: cells of height 1 row with widths log-normal
    (mean 3 sites) clipped to 1..20 sites; ``num_terminals`` fixed I/O pads in a
    ring just outside the core; nets with power-law degree (alpha fitted so the
    mean is ``mean_degree``; max ``max_degree``) and Rent-style locality: a net
    picks a random cell, climbs a binary cluster hierarchy over the cell index
    order one level at a time with probability ``rent_p`` (starting from
    clusters of ``leaf_cluster`` cells) and draws its other pins uniformly in
    that cluster; a ``terminal_net_fraction`` of nets also takes one pad.
    Defaults give the 200k-cell / 220k-net / 2k-pad / 512x512-bin workload.

    ``every_cell_pinned``: the first ``num_cells`` nets start at the cells in
    a seeded random order (so no cell is left without a pin; otherwise about
    e^-4 of the cells have none, and quadratic placement leaves all of those
    at one point).  ``local_pads``: a net's pad is one of the pads nearest to
    its first cell's home (the cell's index read as a Morton code over the
    core, so each cluster of the hierarchy has a region) instead of a pad
    drawn uniformly from the ring, as I/O-connected logic sits near its pads.
    Both change the random stream, so a seed names a different design when
    either is set."""
    rng = np.random.default_rng(seed)
    nc = int(num_cells)
    nn = int(num_nets if num_nets is not None else round(1.1 * nc))
    nt = int(num_terminals if num_terminals is not None else max(4, nc // 100))
    sigma = 0.6
    mu = math.log(3.0) - 0.5 * sigma * sigma
    w = np.clip(np.rint(rng.lognormal(mu, sigma, nc)), 1, 20)
    h = np.ones(nc)
    side = float(math.ceil(math.sqrt(w.sum() / utilisation)))
    rows = _rows(side)

    tx, ty = _pad_ring(nt, side)

    alpha = fit_powerlaw_alpha(mean_degree, 2, max_degree)
    deg = _powerlaw_degrees(rng, nn, alpha, 2, max_degree)
    deg = np.minimum(deg, nc)
    has_pad = rng.random(nn) < terminal_net_fraction
    n_cell_pins = deg - has_pad
    n_cell_pins = np.maximum(n_cell_pins, 1)
    deg = n_cell_pins + has_pad

    # Rent-style cluster level per net: leaf size * 2^level >= pins needed
    root = rng.integers(0, nc, nn)
    if every_cell_pinned:
        root[:min(nc, nn)] = rng.permutation(nc)[:min(nc, nn)]
    level = rng.geometric(1.0 - rent_p, nn) - 1
    need = np.ceil(np.log2(np.maximum(n_cell_pins, 1) * 2.0 / leaf_cluster)).clip(0, None)
    level = np.maximum(level, need.astype(np.int64))
    size = np.minimum(leaf_cluster * (2 ** np.minimum(level, 40)), nc).astype(np.int64)
    start = (root // size) * size
    start = np.minimum(start, nc - size)

    total = int(deg.sum())
    owner = np.empty(total, np.int64)
    net_start = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
    # draw distinct cells inside each cluster: sample with replacement, then
    # repair duplicates by re-drawing (cheap: clusters are >= 2x the pin count)
    for lo_deg in (True, False):
        sel = np.nonzero((n_cell_pins <= 8) == lo_deg)[0]
        if sel.size == 0:
            continue
        if lo_deg:
            k = n_cell_pins[sel]
            kmax = 8
            draw = rng.random((sel.size, kmax))
            cells = start[sel, None] + (draw * size[sel, None]).astype(np.int64)
            cells[:, 0] = root[sel]
            for _ in range(6):
                srt = np.sort(cells, axis=1)
                dup = np.zeros_like(cells, dtype=bool)
                # mark any duplicate within the first k entries
                for j in range(1, kmax):
                    dup[:, j] = np.any(cells[:, :j] == cells[:, j:j + 1], axis=1) & (j < k)
                if not dup.any():
                    break
                redraw = rng.random(dup.sum())
                rows_idx = np.nonzero(dup)[0]
                cells[dup] = start[sel][rows_idx] + (redraw * size[sel][rows_idx]).astype(np.int64)
            for r, n in enumerate(sel):
                kk = int(k[r])
                owner[net_start[n]:net_start[n] + kk] = cells[r, :kk]
        else:
            for n in sel:
                kk = int(n_cell_pins[n])
                c = rng.choice(int(size[n]), size=kk, replace=False) + start[n]
                c[0] = root[n] if root[n] not in c[1:] else c[0]
                owner[net_start[n]:net_start[n] + kk] = c
    pad_nets = np.nonzero(has_pad)[0]
    if local_pads:
        hx, hy = _morton_home(root[pad_nets], nc)
        owner[net_start[pad_nets + 1] - 1] = nc + _nearest_pads(hx, hy, nt, rng)
    else:
        owner[net_start[pad_nets + 1] - 1] = nc + rng.integers(0, nt, pad_nets.size)

    ww = np.concatenate([w, np.ones(nt)])
    hh = np.concatenate([h, np.ones(nt)])
    dx, dy = _offsets(rng, owner, ww, hh)
    is_pad = owner >= nc
    dx[is_pad] = 0.0
    dy[is_pad] = 0.0
    nl = Netlist(
        name=f"stdcell_{nc}_s{seed}", node_w=_f32(w), node_h=_f32(h),
        node_cx=_f32(np.full(nc, side / 2)), node_cy=_f32(np.full(nc, side / 2)),
        term_llx=_f32(tx), term_lly=_f32(ty), term_w=_f32(np.ones(nt)), term_h=_f32(np.ones(nt)),
        term_is_ni=np.zeros(nt, np.uint8), net_start=_i32(net_start), pin_owner=_i32(owner),
        pin_dx=_f32(dx), pin_dy=_f32(dy), target_density=target_density, bins=bins,
        meta=dict(generator="standard_cell", seed=seed, alpha=alpha, utilisation=utilisation,
                  rent_p=rent_p, mean_degree=float(deg.mean()), every_cell_pinned=every_cell_pinned,
                  local_pads=local_pads), **rows)
    return nl


def mixed_size(num_cells=20_000, num_movable_macros=12, num_fixed_macros=4, seed=11,
               utilisation=0.75, target_density=1.0, bins=0, macro_rows=None, **cell_options):
    """Mixed-size design (the ePlace-MS shape at reduced scale): standard cells as
    in ``standard_cell`` plus movable macros (square or 2:1, side log-uniform
    between 2% and 8% of the die, or between ``macro_rows`` = (lo, hi) rows)
    and fixed macros inside the core, which exercise the macro density
    scaling, terminal density and base density.  ``cell_options`` go to
    ``standard_cell``."""
    base = standard_cell(num_cells=num_cells, seed=seed, utilisation=utilisation,
                         target_density=target_density, bins=bins, **cell_options)
    rng = np.random.default_rng(seed + 1000)
    side = base.core()[2]
    nm, nf = num_movable_macros, num_fixed_macros
    lo, hi = (0.02 * side, 0.08 * side) if macro_rows is None else macro_rows
    ms = np.exp(rng.uniform(np.log(lo), np.log(hi), nm + nf))
    ms = np.maximum(np.rint(ms), 2.0)
    aspect = np.where(rng.random(nm + nf) < 0.5, 1.0, 2.0)
    mw, mh = ms * aspect, ms
    # grow the die so the macros fit at the requested utilisation
    area = float(base.node_w.sum() + (mw * mh).sum())
    side = float(math.ceil(math.sqrt(area / utilisation)))
    rows = _rows(side)
    nc = base.num_nodes
    w = np.concatenate([base.node_w, mw[:nm]])
    h = np.concatenate([base.node_h, mh[:nm]])
    # fixed macros inside the core at seeded spots; pads stay on the ring
    fx = rng.uniform(0.1 * side, 0.9 * side - mw[nm:])
    fy = rng.uniform(0.1 * side, 0.9 * side - mh[nm:])
    t_old = base.num_terminals
    px, py = _pad_ring(t_old, side)
    tx = np.concatenate([px, fx])
    ty = np.concatenate([py, fy])
    tw = np.concatenate([base.term_w, mw[nm:]])
    th = np.concatenate([base.term_h, mh[nm:]])
    # owner ids: terminals shift by nm; connect each macro to a few extra nets
    owner = base.pin_owner.astype(np.int64).copy()
    owner[owner >= nc] += nm
    extra_nets = []
    for m in range(nm):
        for _ in range(4):
            k = int(rng.integers(2, 6))
            cells = rng.choice(nc, size=k - 1, replace=False)
            extra_nets.append(np.concatenate([[nc + m], cells]))
    for f in range(nf):
        k = int(rng.integers(2, 6))
        cells = rng.choice(nc, size=k - 1, replace=False)
        extra_nets.append(np.concatenate([[nc + nm + t_old + f], cells]))
    deg = np.diff(base.net_start).tolist() + [len(e) for e in extra_nets]
    owner = np.concatenate([owner] + extra_nets)
    net_start = np.concatenate([[0], np.cumsum(deg)])
    ww = np.concatenate([w, tw])
    hh = np.concatenate([h, th])
    dx, dy = _offsets(rng, owner, ww, hh)
    old = base.num_pins
    dx[:old] = base.pin_dx
    dy[:old] = base.pin_dy
    return Netlist(
        name=f"mixed_{nc}_{nm}m_s{seed}", node_w=_f32(w), node_h=_f32(h),
        node_cx=_f32(np.full(nc + nm, side / 2)), node_cy=_f32(np.full(nc + nm, side / 2)),
        term_llx=_f32(tx), term_lly=_f32(ty), term_w=_f32(tw), term_h=_f32(th),
        term_is_ni=np.zeros(t_old + nf, np.uint8), net_start=_i32(net_start),
        pin_owner=_i32(owner), pin_dx=_f32(dx), pin_dy=_f32(dy), target_density=target_density,
        bins=bins, meta=dict(generator="mixed_size", seed=seed), **rows)


def config3(seed=31):
    """The ePlace-MS workload: 1M standard cells as ``standard_cell`` draws
    them, 300 movable macros (square or 2:1, side 50-400 rows, log-uniform)
    and 50 fixed macros inside the core, nets with the same degree law (1.1M
    with the macros' own), utilisation 0.75, 1024 x 1024 bins."""
    return mixed_size(1_000_000, 300, 50, seed=seed, utilisation=0.75, target_density=1.0, bins=1024,
                      macro_rows=(50.0, 400.0), num_nets=1_100_000, num_terminals=4_000,
                      every_cell_pinned=True, local_pads=True)


def blob_start(nl, seed=3, sigma_frac=0.05):
    """Initial placement used when no QP result is supplied: every movable
    node at the core centre plus seeded Gaussian jitter of ``sigma_frac`` of the
    core side (a compact blob, like the clustered output of quadratic
    placement).  Returns a copy of ``nl`` with the new node centres."""
    rng = np.random.default_rng(seed)
    llx, lly, urx, ury = nl.core()
    cx = 0.5 * (llx + urx) + rng.normal(0.0, sigma_frac * (urx - llx), nl.num_nodes)
    cy = 0.5 * (lly + ury) + rng.normal(0.0, sigma_frac * (ury - lly), nl.num_nodes)
    return nl.with_positions(cx, cy)


def write_bookshelf(nl, directory):
    """Write .aux/.nodes/.nets/.pl/.scl/.wts (positions at full precision)."""
    import os
    os.makedirs(directory, exist_ok=True)
    base = os.path.join(directory, nl.name)
    nn, nt = nl.num_nodes, nl.num_terminals
    names = [f"o{i}" for i in range(nn)] + [f"t{i}" for i in range(nt)]
    with open(base + ".aux", "w") as f:
        f.write(f"RowBasedPlacement : {nl.name}.nodes {nl.name}.nets {nl.name}.wts {nl.name}.pl {nl.name}.scl\n")
    with open(base + ".nodes", "w") as f:
        f.write(f"UCLA nodes 1.0\nNumNodes : {nn + nt}\nNumTerminals : {nt}\n")
        for i in range(nn):
            f.write(f"{names[i]} {nl.node_w[i]:.9g} {nl.node_h[i]:.9g}\n")
        for i in range(nt):
            kind = "terminal_NI" if nl.term_is_ni[i] else "terminal"
            f.write(f"{names[nn + i]} {nl.term_w[i]:.9g} {nl.term_h[i]:.9g} {kind}\n")
    with open(base + ".nets", "w") as f:
        f.write(f"UCLA nets 1.0\nNumNets : {nl.num_nets}\nNumPins : {nl.num_pins}\n")
        for n in range(nl.num_nets):
            a, b = nl.net_start[n], nl.net_start[n + 1]
            f.write(f"NetDegree : {b - a} n{n}\n")
            for p in range(a, b):
                f.write(f"{names[nl.pin_owner[p]]} B : {nl.pin_dx[p]:.9g} {nl.pin_dy[p]:.9g}\n")
    with open(base + ".wts", "w") as f:
        f.write("UCLA wts 1.0\n")
    with open(base + ".pl", "w") as f:
        f.write("UCLA pl 1.0\n\n")
        for i in range(nn):
            f.write(f"{names[i]} {nl.node_cx[i] - 0.5 * nl.node_w[i]:.9g} {nl.node_cy[i] - 0.5 * nl.node_h[i]:.9g} : N\n")
        for i in range(nt):
            fixed = "/FIXED_NI" if nl.term_is_ni[i] else "/FIXED"
            f.write(f"{names[nn + i]} {nl.term_llx[i]:.9g} {nl.term_lly[i]:.9g} : N {fixed}\n")
    with open(base + ".scl", "w") as f:
        f.write(f"UCLA scl 1.0\nNumRows : {nl.num_rows}\n")
        for r in range(nl.num_rows):
            f.write("CoreRow Horizontal\n")
            f.write(f" Coordinate : {nl.row_lly[r]:.9g}\n Height : {nl.row_h[r]:.9g}\n")
            f.write(f" Sitewidth : {nl.row_site_w[r]:.9g}\n Sitespacing : {nl.row_site_w[r]:.9g}\n")
            f.write(" Siteorient : N\n Sitesymmetry : Y\n")
            ns = (nl.row_urx[r] - nl.row_llx[r]) / nl.row_site_w[r]
            f.write(f" SubrowOrigin : {nl.row_llx[r]:.9g} Numsites : {ns:.9g}\nEnd\n")
    return base + ".aux"
