"""ctypes wrapper of oracle/liboracle.so -- TEST INFRASTRUCTURE ONLY.

The C restatement of the ePlace hot path (eplace_oracle.c) that tests/ use as
the FP64 checker of the CUDA engine.  Never imported by the product package.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")

MACRO = 1
FILLER = 2

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)


class Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("core_llx", ctypes.c_float), ("core_lly", ctypes.c_float),
                ("core_urx", ctypes.c_float), ("core_ury", ctypes.c_float),
                ("step_x", ctypes.c_float), ("step_y", ctypes.c_float),
                ("target_density", ctypes.c_float)]


class Design(ctypes.Structure):
    _fields_ = [("grid", Grid), ("num_nodes", ctypes.c_int), ("num_fillers", ctypes.c_int),
                ("num_terms", ctypes.c_int), ("num_nets", ctypes.c_int),
                ("w", _f32p), ("h", _f32p), ("flags", _u8p), ("pins_per_object", _i32p),
                ("net_start", _i32p), ("pin_owner", _i32p), ("pin_dx", _f32p), ("pin_dy", _f32p),
                ("term_cx", _f32p), ("term_cy", _f32p), ("terminal", _f32p), ("base", _f32p),
                ("std_area", ctypes.c_double), ("macro_area", ctypes.c_double),
                ("target_overflow", ctypes.c_float), ("max_iterations", ctypes.c_int),
                ("exp_mode", ctypes.c_int)]


class RunStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("overflow", ctypes.c_double),
                ("hpwl", ctypes.c_double), ("lambda_", ctypes.c_double)]


_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE, "oracle"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.or_bin_dimension.restype = ctypes.c_int
        L.or_bin_dimension.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                       ctypes.c_float, ctypes.c_float, ctypes.c_float]
        L.or_filler_sizing.restype = ctypes.c_int
        L.or_filler_sizing.argtypes = ([ctypes.c_int, _f32p, _f32p, _u8p, ctypes.c_int] + [_f32p] * 4 +
                                       [_u8p, ctypes.c_int] + [_f32p] * 4 +
                                       [ctypes.c_float, ctypes.c_float, ctypes.c_float] + [_f32p] * 4)
        L.or_terminal_base_density.argtypes = ([ctypes.POINTER(Grid), ctypes.c_int] + [_f32p] * 4 +
                                               [ctypes.c_int] + [_f32p] * 4 + [_f32p, _f32p])
        L.or_scatter.argtypes = ([ctypes.POINTER(Grid), ctypes.c_int] + [_f32p] * 4 +
                                 [_u8p, ctypes.c_double, _f64p, _f64p, _i64p, _i64p])
        L.or_poisson.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                 _f64p, _f64p, _f64p, _f64p]
        L.or_gather.argtypes = [ctypes.POINTER(Grid), ctypes.c_int] + [_f32p] * 4 + [_f64p] * 3
        L.or_overflow.restype = ctypes.c_double
        L.or_overflow.argtypes = [ctypes.POINTER(Grid), _f64p, _f64p, _f64p, ctypes.c_double,
                                  ctypes.c_double]
        L.or_inv_gamma.argtypes = [ctypes.c_double, ctypes.c_float, ctypes.c_float, _f64p, _f64p]
        L.or_hpwl.restype = ctypes.c_double
        L.or_hpwl.argtypes = [ctypes.c_int, _i32p, _i32p, _f32p, _f32p, ctypes.c_int] + [_f32p] * 4
        L.or_wirelength_grad.restype = ctypes.c_double
        L.or_wirelength_grad.argtypes = ([ctypes.c_int, _i32p, _i32p, _f32p, _f32p, ctypes.c_int] +
                                         [_f32p] * 4 + [ctypes.c_double, ctypes.c_double,
                                                        ctypes.c_int, ctypes.c_int, _f64p, _f64p])
        L.or_combine.argtypes = [ctypes.c_int, _i32p, _f32p, _u8p, ctypes.c_double, _f64p, _f64p, _f64p]
        L.or_lambda0.restype = ctypes.c_double
        L.or_lambda0.argtypes = [ctypes.c_int, ctypes.c_int, _f64p, _f64p]
        L.or_lambda_multiplier.restype = ctypes.c_double
        L.or_lambda_multiplier.argtypes = [ctypes.c_double, ctypes.c_double]
        L.or_clamp.argtypes = [_f32p, _f32p] + [ctypes.c_float] * 6
        L.or_mgp_run.argtypes = [ctypes.POINTER(Design), _f32p, _f32p, ctypes.POINTER(RunStats)]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def u8(a):
    return np.ascontiguousarray(a, dtype=np.uint8)


def make_grid(nx, ny, core, step_x, step_y, target_density):
    return Grid(int(nx), int(ny), float(core[0]), float(core[1]), float(core[2]), float(core[3]),
                float(step_x), float(step_y), float(target_density))


def bin_dimension(std_area, macro_area, num_nodes, core_w, core_h, target_density):
    return lib().or_bin_dimension(std_area, macro_area, num_nodes, core_w, core_h, target_density)


def filler_sizing(nl, node_is_macro):
    fw = ctypes.c_float()
    fh = ctypes.c_float()
    sa = ctypes.c_float()
    ma = ctypes.c_float()
    row_area = np.float32(0)
    for r in range(nl.num_rows):
        row_area = np.float32(row_area + np.float32((nl.row_urx[r] - nl.row_llx[r]) * nl.row_h[r]))
    k = [f32(nl.node_w), f32(nl.node_h), u8(node_is_macro), f32(nl.term_llx), f32(nl.term_lly),
         f32(nl.term_w), f32(nl.term_h), u8(nl.term_is_ni), f32(nl.row_llx), f32(nl.row_lly),
         f32(nl.row_urx), f32(nl.row_h)]
    n = lib().or_filler_sizing(
        nl.num_nodes, _p(k[0], _f32p), _p(k[1], _f32p), _p(k[2], _u8p), nl.num_terminals,
        _p(k[3], _f32p), _p(k[4], _f32p), _p(k[5], _f32p), _p(k[6], _f32p), _p(k[7], _u8p),
        nl.num_rows, _p(k[8], _f32p), _p(k[9], _f32p), _p(k[10], _f32p), _p(k[11], _f32p),
        float(row_area), float(nl.target_density), float(nl.row_h[-1]),
        ctypes.byref(fw), ctypes.byref(fh), ctypes.byref(sa), ctypes.byref(ma))
    return dict(num_fillers=n, filler_w=fw.value, filler_h=fh.value, std_area=sa.value,
                macro_area=ma.value, total_row_area=float(row_area))


def terminal_base_density(grid, nl):
    nb = grid.nx * grid.ny
    term = np.zeros(nb, np.float32)
    base = np.zeros(nb, np.float32)
    k = [f32(nl.term_llx), f32(nl.term_lly), f32(nl.term_w), f32(nl.term_h), f32(nl.row_llx),
         f32(nl.row_lly), f32(nl.row_urx), f32(nl.row_h)]
    lib().or_terminal_base_density(ctypes.byref(grid), nl.num_terminals, *[_p(a, _f32p) for a in k[:4]],
                                   nl.num_rows, *[_p(a, _f32p) for a in k[4:]],
                                   _p(term, _f32p), _p(base, _f32p))
    return term.reshape(grid.nx, grid.ny), base.reshape(grid.nx, grid.ny)


def scatter(grid, cx, cy, w, h, flags, qscale=0.0):
    nb = grid.nx * grid.ny
    nd = np.zeros(nb)
    fd = np.zeros(nb)
    nq = np.zeros(nb, np.int64)
    fq = np.zeros(nb, np.int64)
    a = [f32(cx), f32(cy), f32(w), f32(h)]
    fl = u8(flags)
    lib().or_scatter(ctypes.byref(grid), len(a[0]), *[_p(x, _f32p) for x in a], _p(fl, _u8p),
                     float(qscale), _p(nd, _f64p), _p(fd, _f64p), _p(nq, _i64p), _p(fq, _i64p))
    s = (grid.nx, grid.ny)
    return nd.reshape(s), fd.reshape(s), nq.reshape(s), fq.reshape(s)


def poisson(rho, step_x, step_y):
    rho = f64(rho)
    nx, ny = rho.shape
    ex = np.zeros_like(rho)
    ey = np.zeros_like(rho)
    phi = np.zeros_like(rho)
    lib().or_poisson(nx, ny, float(step_x), float(step_y), _p(rho, _f64p), _p(ex, _f64p),
                     _p(ey, _f64p), _p(phi, _f64p))
    return ex, ey, phi


def gather(grid, cx, cy, w, h, ex, ey):
    a = [f32(cx), f32(cy), f32(w), f32(h)]
    ex = f64(ex)
    ey = f64(ey)
    g = np.zeros((len(a[0]), 2))
    lib().or_gather(ctypes.byref(grid), len(a[0]), *[_p(x, _f32p) for x in a], _p(ex, _f64p),
                    _p(ey, _f64p), _p(g, _f64p))
    return g


def overflow(grid, node, terminal, base, std_area, macro_area):
    return lib().or_overflow(ctypes.byref(grid), _p(f64(node), _f64p), _p(f64(terminal), _f64p),
                             _p(f64(base), _f64p), float(std_area), float(macro_area))


def inv_gamma(tau, step_x, step_y):
    gx = ctypes.c_double()
    gy = ctypes.c_double()
    lib().or_inv_gamma(float(tau), float(step_x), float(step_y), ctypes.byref(gx), ctypes.byref(gy))
    return gx.value, gy.value


def _net_args(nl):
    return [i32(nl.net_start), i32(nl.pin_owner), f32(nl.pin_dx), f32(nl.pin_dy)]


def hpwl(nl, cx, cy, term_cx, term_cy):
    k = _net_args(nl)
    a = [f32(cx), f32(cy), f32(term_cx), f32(term_cy)]
    return lib().or_hpwl(nl.num_nets, _p(k[0], _i32p), _p(k[1], _i32p), _p(k[2], _f32p),
                         _p(k[3], _f32p), len(a[0]), *[_p(x, _f32p) for x in a])


def wirelength_grad(nl, cx, cy, term_cx, term_cy, igx, igy, exp_mode=0, lse=False):
    """Returns (smooth wirelength, hpwl, grad[num_objects, 2])."""
    k = _net_args(nl)
    a = [f32(cx), f32(cy), f32(term_cx), f32(term_cy)]
    g = np.zeros((len(a[0]), 2))
    hp = ctypes.c_double()
    wl = lib().or_wirelength_grad(nl.num_nets, _p(k[0], _i32p), _p(k[1], _i32p), _p(k[2], _f32p),
                                  _p(k[3], _f32p), len(a[0]), *[_p(x, _f32p) for x in a],
                                  float(igx), float(igy), int(exp_mode), int(bool(lse)),
                                  _p(g, _f64p), ctypes.byref(hp))
    return wl, hp.value, g


def combine(pins_per_object, area, flags, lam, gd, gwl):
    gd = f64(gd)
    gwl = f64(gwl)
    g = np.zeros_like(gd)
    ppo = i32(pins_per_object)
    ar = f32(area)
    fl = u8(flags)
    lib().or_combine(len(ppo), _p(ppo, _i32p), _p(ar, _f32p), _p(fl, _u8p), float(lam),
                     _p(gd, _f64p), _p(gwl, _f64p), _p(g, _f64p))
    return g


def lambda0(num_nodes, gwl, gd):
    gwl = f64(gwl)
    gd = f64(gd)
    return lib().or_lambda0(int(num_nodes), gd.shape[0], _p(gwl, _f64p), _p(gd, _f64p))


def lambda_multiplier(cur, last):
    return lib().or_lambda_multiplier(float(cur), float(last))


def clamp(x, y, w, h, core):
    xs = ctypes.c_float(x)
    ys = ctypes.c_float(y)
    lib().or_clamp(ctypes.byref(xs), ctypes.byref(ys), float(w), float(h), *map(float, core))
    return xs.value, ys.value


def mgp_run(grid, nl, w, h, flags, pins_per_object, num_fillers, term_cx, term_cy, terminal, base,
            std_area, macro_area, cx, cy, target_overflow=0.1, max_iterations=1000, exp_mode=0):
    keep = dict(w=f32(w), h=f32(h), flags=u8(flags), ppo=i32(pins_per_object),
                ns=i32(nl.net_start), po=i32(nl.pin_owner), dx=f32(nl.pin_dx), dy=f32(nl.pin_dy),
                tcx=f32(term_cx), tcy=f32(term_cy), term=f32(terminal).ravel(), base=f32(base).ravel())
    d = Design(grid, nl.num_nodes, int(num_fillers), nl.num_terminals, nl.num_nets,
               _p(keep["w"], _f32p), _p(keep["h"], _f32p), _p(keep["flags"], _u8p),
               _p(keep["ppo"], _i32p), _p(keep["ns"], _i32p), _p(keep["po"], _i32p),
               _p(keep["dx"], _f32p), _p(keep["dy"], _f32p), _p(keep["tcx"], _f32p),
               _p(keep["tcy"], _f32p), _p(keep["term"], _f32p), _p(keep["base"], _f32p),
               float(std_area), float(macro_area), float(target_overflow), int(max_iterations),
               int(exp_mode))
    x = f32(cx).copy()
    y = f32(cy).copy()
    st = RunStats()
    lib().or_mgp_run(ctypes.byref(d), _p(x, _f32p), _p(y, _f32p), ctypes.byref(st))
    return x, y, dict(iterations=st.iterations, overflow=st.overflow, hpwl=st.hpwl, lambda_=st.lambda_)
