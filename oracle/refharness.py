"""ctypes wrapper of oracle/_ref/libeplace_ref.so -- TEST INFRASTRUCTURE ONLY.

The library is the unmodified reference (Xinyu-lumos/ePlace) hot path compiled
from its own sources plus the driver in ``ref_harness.cpp``.  Only tests/,
``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` may use it, and
only as the checker / the timed reference arm -- never as the product path.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libeplace_ref.so")

_f32p = ctypes.POINTER(ctypes.c_float)
_i32p = ctypes.POINTER(ctypes.c_int)
_u8p = ctypes.POINTER(ctypes.c_ubyte)
_f64p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

_lib = None

INFO_FIELDS = (
    "num_nodes", "num_fillers", "bins_x", "bins_y", "bin_step_x", "bin_step_y",
    "core_llx", "core_lly", "core_urx", "core_ury", "filler_w", "filler_h",
    "std_area", "macro_area", "target_density", "overflow", "lambda",
    "inv_gamma_x", "inv_gamma_y", "last_hpwl", "stage", "mgp_iterations",
    "total_row_area", "num_cells_and_fillers", "iter_count", "ns_param",
)


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("reference harness not built: run `make -C oracle ref`")
        L = ctypes.CDLL(LIB_PATH)
        L.ref_create_bookshelf.restype = _vp
        L.ref_create_bookshelf.argtypes = [ctypes.c_char_p]
        L.ref_create_arrays.restype = _vp
        L.ref_create_arrays.argtypes = [ctypes.c_int] * 4 + [_f32p] * 8 + [_u8p, _i32p, _i32p] + [_f32p] * 7
        for name in ("ref_destroy", "ref_penalty_init", "ref_penalty_update", "ref_opt_begin",
                     "ref_opt_end", "ref_switch_filler_only", "ref_switch_cgp"):
            getattr(L, name).argtypes = [_vp]
            getattr(L, name).restype = None
        for name in ("ref_qp", "ref_eval", "ref_opt_run", "ref_calc_hpwl", "ref_abacus", "ref_detailed"):
            getattr(L, name).argtypes = [_vp]
            getattr(L, name).restype = ctypes.c_double
        L.ref_init.argtypes = [_vp, ctypes.c_float]
        L.ref_init.restype = ctypes.c_double
        L.ref_macro_legalize.argtypes = [_vp, ctypes.c_float]
        L.ref_macro_legalize.restype = ctypes.c_double
        L.ref_netlist_counts.argtypes = [_vp, _i32p]
        L.ref_get_info.argtypes = [_vp, _f64p]
        L.ref_get_positions.argtypes = [_vp, _f32p, _f32p]
        L.ref_set_positions.argtypes = [_vp, _f32p, _f32p]
        L.ref_get_node_centers.argtypes = [_vp, _f32p, _f32p]
        L.ref_set_node_centers.argtypes = [_vp, _f32p, _f32p]
        L.ref_set_lambda.argtypes = [_vp, ctypes.c_float]
        L.ref_set_last_hpwl.argtypes = [_vp, ctypes.c_double]
        L.ref_get_bins.argtypes = [_vp] + [_f32p] * 7
        L.ref_get_gradients.argtypes = [_vp, _f32p, _f32p, _f32p]
        L.ref_get_stage_gradient.argtypes = [_vp, _f32p]
        L.ref_get_stage_gradient.restype = ctypes.c_int
        L.ref_opt_step.argtypes = [_vp, _f64p]
        L.ref_opt_step.restype = ctypes.c_int
        L.ref_opt_state.argtypes = [_vp] + [_f32p] * 5
        L.ref_opt_state.restype = ctypes.c_int
        L.ref_get_node_flags.argtypes = [_vp, _u8p]
        L.ref_ooura_2d.argtypes = [ctypes.c_int] * 4 + [_f32p]
        L.ref_set_flag.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        L.ref_clear_flag.argtypes = [ctypes.c_char_p]
        L.ref_set_quiet.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def ooura_2d(kind, data, isgn):
    """Run the reference's ddct2d (0) / ddsct2d (1) / ddcst2d (2) in place on a copy."""
    a = np.ascontiguousarray(data, dtype=np.float32).copy()
    lib().ref_ooura_2d(kind, a.shape[0], a.shape[1], isgn, _p(a, _f32p))
    return a


def set_flag(name, value="1"):
    lib().ref_set_flag(name.encode(), value.encode())


def clear_flag(name):
    lib().ref_clear_flag(name.encode())


class RefPlacer:
    """One reference PlaceDB + EPlacer_2D + EplaceNesterovOpt instance."""

    def __init__(self, netlist=None, aux=None):
        L = lib()
        if aux is not None:
            self.h = L.ref_create_bookshelf(aux.encode())
        else:
            nl = netlist
            f = lambda a: np.ascontiguousarray(a, dtype=np.float32)
            self._keep = dict(
                node_w=f(nl.node_w), node_h=f(nl.node_h), node_cx=f(nl.node_cx), node_cy=f(nl.node_cy),
                term_llx=f(nl.term_llx), term_lly=f(nl.term_lly), term_w=f(nl.term_w), term_h=f(nl.term_h),
                term_ni=np.ascontiguousarray(nl.term_is_ni, dtype=np.uint8),
                net_start=np.ascontiguousarray(nl.net_start, dtype=np.int32),
                pin_owner=np.ascontiguousarray(nl.pin_owner, dtype=np.int32),
                pin_dx=f(nl.pin_dx), pin_dy=f(nl.pin_dy),
                row_llx=f(nl.row_llx), row_lly=f(nl.row_lly), row_urx=f(nl.row_urx), row_h=f(nl.row_h),
                row_site=f(nl.row_site_w),
            )
            k = self._keep
            self.h = L.ref_create_arrays(
                nl.num_nodes, nl.num_terminals, nl.num_nets, nl.num_rows,
                _p(k["node_w"], _f32p), _p(k["node_h"], _f32p), _p(k["node_cx"], _f32p), _p(k["node_cy"], _f32p),
                _p(k["term_llx"], _f32p), _p(k["term_lly"], _f32p), _p(k["term_w"], _f32p), _p(k["term_h"], _f32p),
                _p(k["term_ni"], _u8p), _p(k["net_start"], _i32p), _p(k["pin_owner"], _i32p),
                _p(k["pin_dx"], _f32p), _p(k["pin_dy"], _f32p),
                _p(k["row_llx"], _f32p), _p(k["row_lly"], _f32p), _p(k["row_urx"], _f32p), _p(k["row_h"], _f32p),
                _p(k["row_site"], _f32p))
        c = np.zeros(6, np.int32)
        L.ref_netlist_counts(self.h, _p(c, _i32p))
        self.num_nodes, self.num_terminals, self.num_nets, self.num_pins, self.num_rows, self.num_macros = map(int, c)

    # --- netlist-stage helpers -------------------------------------------------
    def qp(self):
        return lib().ref_qp(self.h)

    # --- the CPU stages around global placement (main/ePlace_main.cpp:174-279)
    def macro_legalize(self, target_density):
        """SAMacroLegalizer::legalization on the current positions; seconds."""
        return lib().ref_macro_legalize(self.h, float(target_density))

    def abacus(self):
        """AbacusLegalizer::legalization on the current positions; seconds."""
        return lib().ref_abacus(self.h)

    def detailed(self):
        """DetailedPlacer::detailedPlacement after the legalizer; seconds."""
        return lib().ref_detailed(self.h)

    def node_centers(self):
        cx = np.zeros(self.num_nodes, np.float32)
        cy = np.zeros(self.num_nodes, np.float32)
        lib().ref_get_node_centers(self.h, _p(cx, _f32p), _p(cy, _f32p))
        return cx, cy

    def set_node_centers(self, cx, cy):
        cx = np.ascontiguousarray(cx, np.float32)
        cy = np.ascontiguousarray(cy, np.float32)
        lib().ref_set_node_centers(self.h, _p(cx, _f32p), _p(cy, _f32p))

    def node_is_macro(self):
        m = np.zeros(self.num_nodes, np.uint8)
        lib().ref_get_node_flags(self.h, _p(m, _u8p))
        return m

    # --- EPlacer_2D ------------------------------------------------------------
    def initialization(self, target_density):
        return lib().ref_init(self.h, float(target_density))

    def info(self):
        out = np.zeros(len(INFO_FIELDS), np.float64)
        lib().ref_get_info(self.h, _p(out, _f64p))
        return dict(zip(INFO_FIELDS, out.tolist()))

    @property
    def num_objects(self):
        i = self.info()
        return int(i["num_nodes"] + i["num_fillers"])

    def positions(self):
        n = self.num_objects
        cx = np.zeros(n, np.float32)
        cy = np.zeros(n, np.float32)
        lib().ref_get_positions(self.h, _p(cx, _f32p), _p(cy, _f32p))
        return cx, cy

    def set_positions(self, cx, cy):
        cx = np.ascontiguousarray(cx, np.float32)
        cy = np.ascontiguousarray(cy, np.float32)
        lib().ref_set_positions(self.h, _p(cx, _f32p), _p(cy, _f32p))

    def total_gradient_update(self):
        return lib().ref_eval(self.h)

    def set_lambda(self, lam):
        lib().ref_set_lambda(self.h, float(lam))

    def set_last_hpwl(self, v):
        lib().ref_set_last_hpwl(self.h, float(v))

    def penalty_init(self):
        lib().ref_penalty_init(self.h)

    def penalty_update(self):
        lib().ref_penalty_update(self.h)

    def hpwl(self):
        return lib().ref_calc_hpwl(self.h)

    def bins(self):
        i = self.info()
        nx, ny = int(i["bins_x"]), int(i["bins_y"])
        maps = {k: np.zeros((nx, ny), np.float32) for k in ("node", "filler", "terminal", "base", "ex", "ey", "phi")}
        lib().ref_get_bins(self.h, *[_p(maps[k], _f32p) for k in ("node", "filler", "terminal", "base", "ex", "ey", "phi")])
        return maps

    def gradients(self):
        n = self.num_objects
        wl = np.zeros((self.num_nodes, 2), np.float32)
        dens = np.zeros((n, 2), np.float32)
        tot = np.zeros((n, 2), np.float32)
        lib().ref_get_gradients(self.h, _p(wl, _f32p), _p(dens, _f32p), _p(tot, _f32p))
        return wl, dens, tot

    def stage_gradient(self):
        g = np.zeros((self.num_objects, 2), np.float32)
        m = lib().ref_get_stage_gradient(self.h, _p(g, _f32p))
        return g[:m]

    def switch_filler_only(self):
        lib().ref_switch_filler_only(self.h)

    def switch_cgp(self):
        lib().ref_switch_cgp(self.h)

    # --- EplaceNesterovOpt -----------------------------------------------------
    def opt_run(self):
        return lib().ref_opt_run(self.h)

    def opt_begin(self):
        lib().ref_opt_begin(self.h)

    def opt_step(self):
        """Returns (stopped, seconds)."""
        t = ctypes.c_double(0.0)
        stopped = lib().ref_opt_step(self.h, ctypes.byref(t))
        return bool(stopped), t.value

    def opt_end(self):
        lib().ref_opt_end(self.h)

    def opt_state(self):
        n = self.num_objects
        arrs = [np.zeros((n, 2), np.float32) for _ in range(5)]
        m = lib().ref_opt_state(self.h, *[_p(a, _f32p) for a in arrs])
        return [a[:m] for a in arrs]

    def close(self):
        if self.h:
            lib().ref_destroy(self.h)
            self.h = None
