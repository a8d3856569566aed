"""Bookshelf reader producing the engine's array netlist.

Follows the reference parser (Parser/parser.cpp:44-819): .aux names the
.nodes/.nets/.wts/.pl/.scl files; "terminal" and "terminal_NI" lines are
fixed terminals (the latter flagged NI); a pin line "<owner> <dir> : dx dy"
gives an offset from the owner's centre; .pl gives lower-left corners; .scl
rows carry Coordinate / Height / Sitewidth / SubrowOrigin / Numsites.
"""
import os

import numpy as np

from .synth import Netlist


def _tokens(line):
    return line.replace(":", " : ").split()


def read_aux(aux_path, target_density=1.0, bins=0):
    d = os.path.dirname(os.path.abspath(aux_path))
    with open(aux_path) as f:
        toks = f.readline().split()
    files = {os.path.splitext(t)[1]: os.path.join(d, t) for t in toks[2:]}
    names, w, h, kinds = _read_nodes(files[".nodes"])
    index = {n: i for i, n in enumerate(names)}
    movable = [i for i, k in enumerate(kinds) if k == "node"]
    terms = [i for i, k in enumerate(kinds) if k != "node"]
    remap = np.empty(len(names), np.int64)
    remap[movable] = np.arange(len(movable))
    remap[terms] = len(movable) + np.arange(len(terms))
    net_start, owner, dx, dy = _read_nets(files[".nets"], index)
    llx, lly = _read_pl(files[".pl"], index, len(names))
    rows = _read_scl(files[".scl"])
    mv = np.array(movable, np.int64)
    tm = np.array(terms, np.int64)
    w = np.asarray(w, np.float32)
    h = np.asarray(h, np.float32)
    return Netlist(
        name=os.path.splitext(os.path.basename(aux_path))[0],
        node_w=w[mv], node_h=h[mv],
        node_cx=(llx[mv] + np.float32(0.5) * w[mv]).astype(np.float32),
        node_cy=(lly[mv] + np.float32(0.5) * h[mv]).astype(np.float32),
        term_llx=llx[tm], term_lly=lly[tm], term_w=w[tm], term_h=h[tm],
        term_is_ni=np.array([kinds[i] == "terminal_NI" for i in terms], np.uint8),
        net_start=np.asarray(net_start, np.int32),
        pin_owner=remap[np.asarray(owner, np.int64)].astype(np.int32),
        pin_dx=np.asarray(dx, np.float32), pin_dy=np.asarray(dy, np.float32),
        target_density=target_density, bins=bins, meta=dict(source=aux_path), **rows)


def _read_nodes(path):
    names, w, h, kinds = [], [], [], []
    with open(path) as f:
        f.readline()
        for line in f:
            t = line.split()
            if not t or t[0].startswith("#") or t[0] in ("NumNodes", "NumTerminals"):
                continue
            names.append(t[0])
            w.append(float(t[1]))
            h.append(float(t[2]))
            kinds.append(t[3] if len(t) > 3 and t[3].startswith("terminal") else "node")
    return names, w, h, kinds


def _read_nets(path, index):
    net_start, owner, dx, dy = [0], [], [], []
    with open(path) as f:
        f.readline()
        lines = iter(f)
        for line in lines:
            t = _tokens(line)
            if not t or t[0].startswith("#") or t[0] in ("NumNets", "NumPins"):
                continue
            if t[0] != "NetDegree":
                raise ValueError(f"unsupported line in {path}: {line!r}")
            deg = int(t[2])
            for _ in range(deg):
                p = _tokens(next(lines))
                owner.append(index[p[0]])
                rest = p[p.index(":") + 1:] if ":" in p else []
                dx.append(float(rest[0]) if len(rest) > 0 else 0.0)
                dy.append(float(rest[1]) if len(rest) > 1 else 0.0)
            net_start.append(len(owner))
    return net_start, owner, dx, dy


def _read_pl(path, index, n):
    llx = np.zeros(n, np.float32)
    lly = np.zeros(n, np.float32)
    with open(path) as f:
        f.readline()
        for line in f:
            for ch in "(),:=\r":
                line = line.replace(ch, " ")
            t = line.split()
            if len(t) < 3 or t[0].startswith("#") or t[0] not in index:
                continue
            i = index[t[0]]
            llx[i] = np.float32(float(t[1]))
            lly[i] = np.float32(float(t[2]))
    return llx, lly


def _read_scl(path):
    rows = []
    cur = None
    site = 1.0
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            if t[0] == "CoreRow":
                cur = dict(bottom=0.0, height=0.0, site=site, origin=0.0, sites=0.0)
                rows.append(cur)
            elif t[0] == "Coordinate":
                cur["bottom"] = float(t[2])
            elif t[0] == "Height":
                cur["height"] = float(t[2])
            elif t[0] == "Sitewidth":
                site = float(t[2])
                cur["site"] = site
            elif len(t) >= 6 and t[3] in ("Numsites", "NumSites"):
                cur["origin"] = float(t[2])
                cur["sites"] = float(t[5])
    f32 = lambda a: np.asarray(a, np.float32)
    return dict(
        row_llx=f32([r["origin"] for r in rows]), row_lly=f32([r["bottom"] for r in rows]),
        row_urx=f32([r["sites"] * r["site"] + r["origin"] for r in rows]),
        row_h=f32([r["height"] for r in rows]), row_site_w=f32([r["site"] for r in rows]))
