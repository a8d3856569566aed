"""Host-side mirror of the reference's global-placement call surface.

``EPlacer2D`` keeps the method names of EPlacer_2D (EPlace/eplace.h:95-200) and
``EplaceNesterovOpt`` those of the optimizer (Optimization/nesterov.hpp:59-77,
Optimization/opt.hpp:19-36), so a driver written against the reference
(main/ePlace_main.cpp:141-211) reads the same.  Every call goes through the
C-ABI of include/eplace_gpu.h into ``libeplace_b200.so``; there is no CPU
fallback: without the CUDA library or a GPU the calls raise.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libeplace_b200.so")

EP_OK, EP_ERR_ARG, EP_ERR_CUDA, EP_ERR_NAN, EP_ERR_TIMEOUT, EP_ERR_STATE, EP_ERR_NOMEM, EP_ERR_UNSUPPORTED = range(8)
STATUS_NAMES = ["EP_OK", "EP_ERR_ARG", "EP_ERR_CUDA", "EP_ERR_NAN", "EP_ERR_TIMEOUT", "EP_ERR_STATE",
                "EP_ERR_NOMEM", "EP_ERR_UNSUPPORTED"]
MGP, FILLERONLY, CGP = 0, 1, 2
WL_WA, WL_LSE = 0, 1
EXP_FAST, EXP_EXACT = 0, 1
STEP_LIPSCHITZ, STEP_BB, STEP_BKTRK = 0, 1, 2
DCT_FP32, DCT_BF16X3, DCT_AUTO, DCT_FFT = 0, 1, 2, 3
PREC_MIXED, PREC_FP64 = 0, 1
ABI_VERSION = 3

_f32p = ctypes.POINTER(ctypes.c_float)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_f64p = ctypes.POINTER(ctypes.c_double)


class EPError(RuntimeError):
    def __init__(self, status, msg):
        self.status = status
        super().__init__(f"{STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else status}: {msg}")


class Netlist(ctypes.Structure):
    _fields_ = [("num_nodes", ctypes.c_int32), ("num_terminals", ctypes.c_int32),
                ("num_nets", ctypes.c_int32), ("num_rows", ctypes.c_int32),
                ("node_w", _f32p), ("node_h", _f32p), ("node_cx", _f32p), ("node_cy", _f32p),
                ("term_llx", _f32p), ("term_lly", _f32p), ("term_w", _f32p), ("term_h", _f32p),
                ("term_is_ni", _u8p), ("net_start", _i32p), ("pin_owner", _i32p),
                ("pin_dx", _f32p), ("pin_dy", _f32p), ("row_llx", _f32p), ("row_lly", _f32p),
                ("row_urx", _f32p), ("row_h", _f32p), ("common_row_height", ctypes.c_float)]


class Params(ctypes.Structure):
    _fields_ = [("target_density", ctypes.c_float), ("target_overflow", ctypes.c_float),
                ("bins_x", ctypes.c_int32), ("bins_y", ctypes.c_int32),
                ("max_iterations", ctypes.c_int32), ("wl_model", ctypes.c_int32),
                ("exp_mode", ctypes.c_int32), ("step_rule", ctypes.c_int32),
                ("dct_mode", ctypes.c_int32), ("filler_seed", ctypes.c_uint64),
                ("device", ctypes.c_int32), ("keep_maps", ctypes.c_int32),
                ("precision", ctypes.c_int32)]


class Limits(ctypes.Structure):
    _fields_ = [("wait_polls", ctypes.c_uint32), ("bktrk_trials", ctypes.c_int32),
                ("bktrk_accept", ctypes.c_double)]


class Scalars(ctypes.Structure):
    _fields_ = [("overflow", ctypes.c_double), ("lambda_", ctypes.c_double), ("hpwl", ctypes.c_double),
                ("last_hpwl", ctypes.c_double), ("inv_gamma_x", ctypes.c_double),
                ("inv_gamma_y", ctypes.c_double), ("wirelength", ctypes.c_double),
                ("step", ctypes.c_double), ("ns_param", ctypes.c_double),
                ("iteration", ctypes.c_int32), ("stage", ctypes.c_int32),
                ("mgp_iterations", ctypes.c_int32), ("done", ctypes.c_int32)]


class Info(ctypes.Structure):
    _fields_ = [("num_nodes", ctypes.c_int32), ("num_fillers", ctypes.c_int32),
                ("num_objects", ctypes.c_int32), ("num_terminals", ctypes.c_int32),
                ("num_nets", ctypes.c_int32), ("num_pins", ctypes.c_int32),
                ("num_macros", ctypes.c_int32), ("num_cells_and_fillers", ctypes.c_int32),
                ("bins_x", ctypes.c_int32), ("bins_y", ctypes.c_int32),
                ("bin_step_x", ctypes.c_float), ("bin_step_y", ctypes.c_float),
                ("core_llx", ctypes.c_float), ("core_lly", ctypes.c_float),
                ("core_urx", ctypes.c_float), ("core_ury", ctypes.c_float),
                ("filler_w", ctypes.c_float), ("filler_h", ctypes.c_float),
                ("std_area", ctypes.c_double), ("macro_area", ctypes.c_double),
                ("total_row_area", ctypes.c_double), ("density_scale", ctypes.c_double),
                ("dct_mode", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("create_seconds", ctypes.c_double * 5)]


class RunStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("overflow", ctypes.c_double),
                ("hpwl", ctypes.c_double), ("lambda_", ctypes.c_double), ("seconds", ctypes.c_double),
                ("kernel_launches", ctypes.c_int64)]


class QpStats(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_int32), ("solver_iterations", ctypes.c_int32), ("hpwl", ctypes.c_double),
                ("error_x", ctypes.c_double), ("error_y", ctypes.c_double), ("seconds", ctypes.c_double),
                ("kernel_launches", ctypes.c_int64)]


MAX_TIMED = 12


class KernelTimes(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int32), ("names", (ctypes.c_char * 24) * MAX_TIMED),
                ("ms", ctypes.c_double * MAX_TIMED), ("bytes", ctypes.c_double * MAX_TIMED),
                ("flops", ctypes.c_double * MAX_TIMED), ("launches", ctypes.c_int32 * MAX_TIMED)]


# every symbol include/eplace_gpu.h declares
EXPORTS = (
    "ep_default_params", "ep_abi_version", "ep_create", "ep_destroy", "ep_last_error", "ep_get_info",
    "ep_set_stream", "ep_synchronize", "ep_get_positions", "ep_set_positions", "ep_initialize",
    "ep_eval_gradient", "ep_get_gradient", "ep_get_component_gradients", "ep_get_bin_maps",
    "ep_get_positions_f64", "ep_get_field_f64", "ep_get_component_gradients_f64",
    "ep_get_limits", "ep_set_limits", "ep_quadratic_refine", "ep_state_size", "ep_save_state", "ep_load_state",
    "ep_gnn_num_weights", "ep_gnn_create", "ep_gnn_destroy", "ep_gnn_last_error", "ep_gnn_get_weights",
    "ep_gnn_set_weights", "ep_gnn_release", "ep_gnn_features", "ep_gnn_forward", "ep_gnn_loss_grad",
    "ep_gnn_train_step", "ep_gnn_propose", "ep_gnn_set_wait_limit",
    "ep_get_density_fixed", "ep_query", "ep_set_lambda", "ep_penalty_init", "ep_penalty_update",
    "ep_hpwl", "ep_switch_stage", "ep_nesterov_run", "ep_nesterov_begin", "ep_nesterov_step",
    "ep_nesterov_end", "ep_save_positions", "ep_load_positions", "ep_time_kernels", "ep_quadratic_placement", "ep_run_batch",
    "ep_netbin_write", "ep_netbin_open", "ep_netbin_close",
    "ep_bookshelf_read", "ep_bookshelf_write_pl", "ep_bookshelf_write", "ep_bookshelf_row_site_widths",
    "ep_bookshelf_close",
    "ep_density_scatter_noalloc",
)


class ScatterGrid(ctypes.Structure):
    _fields_ = [("bins_x", ctypes.c_int32), ("bins_y", ctypes.c_int32),
                ("core_llx", ctypes.c_float), ("core_lly", ctypes.c_float),
                ("bin_step_x", ctypes.c_float), ("bin_step_y", ctypes.c_float),
                ("target_density", ctypes.c_float)]


def density_scatter_noalloc(grid, num_objects, cx, cy, w, h, flags, node_out, filler_out, stream=0):
    """ep_density_scatter_noalloc on raw DEVICE pointers (ints); returns (status, message)."""
    L = load()
    buf = ctypes.create_string_buffer(256)
    vp = lambda p: ctypes.c_void_p(int(p)) if p else None
    rc = L.ep_density_scatter_noalloc(ctypes.byref(grid), int(num_objects), vp(cx), vp(cy), vp(w), vp(h),
                                      vp(flags), vp(node_out), vp(filler_out), vp(stream), buf, 256)
    return rc, buf.value.decode()

_lib = None


def load():
    """Load the engine library; raises if it was not built (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m eplace_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    L.ep_default_params.argtypes = [ctypes.POINTER(Params)]
    L.ep_default_params.restype = None
    L.ep_abi_version.restype = ctypes.c_int32
    if L.ep_abi_version() != ABI_VERSION:
        raise RuntimeError(f"{LIB_PATH} has ABI {L.ep_abi_version()}, this binding {ABI_VERSION}: rebuild it")
    L.ep_create.argtypes = [ctypes.POINTER(Netlist), ctypes.POINTER(Params), ctypes.POINTER(vp)]
    L.ep_destroy.argtypes = [vp]
    L.ep_destroy.restype = None
    L.ep_last_error.argtypes = [vp]
    L.ep_last_error.restype = ctypes.c_char_p
    L.ep_get_info.argtypes = [vp, ctypes.POINTER(Info)]
    L.ep_set_stream.argtypes = [vp, vp]
    L.ep_synchronize.argtypes = [vp]
    for n in ("ep_get_positions", "ep_set_positions", "ep_get_gradient"):
        getattr(L, n).argtypes = [vp, ctypes.c_int32, _f32p, ctypes.c_int32]
    for n in ("ep_initialize", "ep_eval_gradient", "ep_penalty_init", "ep_penalty_update",
              "ep_nesterov_begin", "ep_nesterov_end", "ep_save_positions", "ep_load_positions"):
        getattr(L, n).argtypes = [vp]
    L.ep_time_kernels.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(KernelTimes)]
    L.ep_quadratic_placement.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(QpStats)]
    L.ep_quadratic_refine.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(QpStats)]
    L.ep_state_size.argtypes = [vp]
    L.ep_state_size.restype = ctypes.c_uint64
    L.ep_save_state.argtypes = [vp, vp, ctypes.c_uint64]
    L.ep_load_state.argtypes = [vp, vp, ctypes.c_uint64]
    L.ep_run_batch.argtypes = [ctypes.POINTER(vp), ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(RunStats)]
    L.ep_netbin_write.argtypes = [ctypes.c_char_p, ctypes.POINTER(Netlist), ctypes.c_float, ctypes.c_int32]
    L.ep_netbin_open.argtypes = [ctypes.c_char_p, ctypes.POINTER(Netlist), ctypes.POINTER(ctypes.c_float),
                                 ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(vp)]
    L.ep_netbin_close.argtypes = [vp]
    L.ep_netbin_close.restype = None
    L.ep_bookshelf_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(Netlist), ctypes.POINTER(ctypes.c_void_p),
                                    ctypes.c_char_p, ctypes.c_int32]
    L.ep_bookshelf_write_pl.argtypes = [vp, ctypes.c_char_p, _f32p, _f32p]
    L.ep_bookshelf_write.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(Netlist), vp]
    L.ep_bookshelf_row_site_widths.argtypes = [vp, _f32p, ctypes.c_int32]
    L.ep_bookshelf_close.argtypes = [vp]
    L.ep_bookshelf_close.restype = None
    L.ep_density_scatter_noalloc.argtypes = [ctypes.POINTER(ScatterGrid), ctypes.c_int32] + [vp] * 8 + \
        [ctypes.c_char_p, ctypes.c_int32]
    L.ep_get_component_gradients.argtypes = [vp, _f32p, _f32p]
    L.ep_get_component_gradients_f64.argtypes = [vp, _f64p, _f64p]
    L.ep_get_limits.argtypes = [vp, ctypes.POINTER(Limits)]
    L.ep_gnn_num_weights.restype = ctypes.c_int32
    L.ep_gnn_create.argtypes = [ctypes.c_int32, ctypes.c_uint64, ctypes.POINTER(vp)]
    L.ep_gnn_destroy.argtypes = [vp]
    L.ep_gnn_destroy.restype = None
    L.ep_gnn_last_error.argtypes = [vp]
    L.ep_gnn_last_error.restype = ctypes.c_char_p
    L.ep_gnn_get_weights.argtypes = [vp, _f32p]
    L.ep_gnn_set_weights.argtypes = [vp, _f32p]
    L.ep_gnn_release.argtypes = [vp, vp]
    L.ep_gnn_features.argtypes = [vp, vp, _f32p]
    L.ep_gnn_forward.argtypes = [vp, vp, _f32p]
    L.ep_gnn_loss_grad.argtypes = [vp, vp, _f32p, ctypes.POINTER(ctypes.c_double), _f32p]
    L.ep_gnn_train_step.argtypes = [vp, vp, _f32p, ctypes.c_float, ctypes.POINTER(ctypes.c_double)]
    L.ep_gnn_propose.argtypes = [vp, vp, ctypes.c_float]
    L.ep_gnn_set_wait_limit.argtypes = [vp, ctypes.c_int32]
    L.ep_set_limits.argtypes = [vp, ctypes.POINTER(Limits)]
    L.ep_get_positions_f64.argtypes = [vp, ctypes.c_int32, _f64p, ctypes.c_int32]
    L.ep_get_field_f64.argtypes = [vp, _f64p, _f64p, _f64p]
    L.ep_get_bin_maps.argtypes = [vp] + [_f32p] * 7
    L.ep_get_density_fixed.argtypes = [vp, _i64p, _i64p]
    L.ep_query.argtypes = [vp, ctypes.POINTER(Scalars)]
    L.ep_set_lambda.argtypes = [vp, ctypes.c_double]
    L.ep_hpwl.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    L.ep_switch_stage.argtypes = [vp, ctypes.c_int32, _f32p]
    L.ep_nesterov_run.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(RunStats)]
    L.ep_nesterov_step.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
    _lib = L
    return L


def netlist_struct(nl):
    """ep_netlist view of a synth.Netlist; returns (struct, arrays it points
    into), the arrays kept alive by the caller."""
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    k = dict(
        node_w=f(nl.node_w), node_h=f(nl.node_h), node_cx=f(nl.node_cx), node_cy=f(nl.node_cy),
        term_llx=f(nl.term_llx), term_lly=f(nl.term_lly), term_w=f(nl.term_w), term_h=f(nl.term_h),
        term_ni=np.ascontiguousarray(nl.term_is_ni, dtype=np.uint8),
        net_start=np.ascontiguousarray(nl.net_start, dtype=np.int32),
        pin_owner=np.ascontiguousarray(nl.pin_owner, dtype=np.int32),
        pin_dx=f(nl.pin_dx), pin_dy=f(nl.pin_dy), row_llx=f(nl.row_llx), row_lly=f(nl.row_lly),
        row_urx=f(nl.row_urx), row_h=f(nl.row_h))
    c = Netlist(nl.num_nodes, nl.num_terminals, nl.num_nets, nl.num_rows,
                _p(k["node_w"], _f32p), _p(k["node_h"], _f32p), _p(k["node_cx"], _f32p),
                _p(k["node_cy"], _f32p), _p(k["term_llx"], _f32p), _p(k["term_lly"], _f32p),
                _p(k["term_w"], _f32p), _p(k["term_h"], _f32p), _p(k["term_ni"], _u8p),
                _p(k["net_start"], _i32p), _p(k["pin_owner"], _i32p), _p(k["pin_dx"], _f32p),
                _p(k["pin_dy"], _f32p), _p(k["row_llx"], _f32p), _p(k["row_lly"], _f32p),
                _p(k["row_urx"], _f32p), _p(k["row_h"], _f32p), 0.0)
    return c, k


def netbin_write(nl, path):
    """ep_netbin_write: the netlist as the engine's binary netlist file."""
    c, keep = netlist_struct(nl)
    rc = load().ep_netbin_write(str(path).encode(), ctypes.byref(c), float(nl.target_density), int(nl.bins))
    if rc:
        raise EPError(rc, f"ep_netbin_write({path}): {STATUS_NAMES[rc]}")
    return path


def _netlist_copy(c, name, target_density, bins):
    """A synth.Netlist holding copies of the arrays an ep_netlist points at
    (row site widths are not part of ep_netlist and come back as 1)."""
    from .synth import Netlist as SynthNetlist
    nn, nt, nnet, nr = c.num_nodes, c.num_terminals, c.num_nets, c.num_rows
    a = lambda ptr, n: np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0, np.float32)
    np_ = int(np.ctypeslib.as_array(c.net_start, shape=(nnet + 1,))[nnet])
    return SynthNetlist(
        name=name,
        node_w=a(c.node_w, nn), node_h=a(c.node_h, nn), node_cx=a(c.node_cx, nn), node_cy=a(c.node_cy, nn),
        term_llx=a(c.term_llx, nt), term_lly=a(c.term_lly, nt), term_w=a(c.term_w, nt),
        term_h=a(c.term_h, nt), term_is_ni=a(c.term_is_ni, nt).astype(np.uint8),
        net_start=a(c.net_start, nnet + 1).astype(np.int32), pin_owner=a(c.pin_owner, np_).astype(np.int32),
        pin_dx=a(c.pin_dx, np_), pin_dy=a(c.pin_dy, np_), row_llx=a(c.row_llx, nr), row_lly=a(c.row_lly, nr),
        row_urx=a(c.row_urx, nr), row_h=a(c.row_h, nr), row_site_w=np.ones(nr, np.float32),
        target_density=target_density, bins=bins)


def netbin_read(path):
    """ep_netbin_open: map a binary netlist file; returns a synth.Netlist
    holding copies of its arrays (row site widths are not part of
    ep_netlist and come back as 1)."""
    L = load()
    c, td, bins, h = Netlist(), ctypes.c_float(), ctypes.c_int32(), ctypes.c_void_p()
    rc = L.ep_netbin_open(str(path).encode(), ctypes.byref(c), ctypes.byref(td), ctypes.byref(bins),
                          ctypes.byref(h))
    if rc:
        raise EPError(rc, f"ep_netbin_open({path}): {STATUS_NAMES[rc]}")
    try:
        return _netlist_copy(c, str(path).rsplit("/", 1)[-1].split(".")[0], td.value, bins.value)
    finally:
        L.ep_netbin_close(h)


def bookshelf_write(nl, directory, name=None, design=None):
    """ep_bookshelf_write: the netlist as Bookshelf files in `directory`
    (names o<i> / t<i> unless `design`, a BookshelfDesign of the same
    design, gives the original ones); returns the .aux path."""
    import os
    os.makedirs(directory, exist_ok=True)
    name = name or nl.name
    c, keep = netlist_struct(nl)
    h = design._h if design is not None else None
    rc = load().ep_bookshelf_write(str(directory).encode(), name.encode(), ctypes.byref(c), h)
    if rc:
        raise EPError(rc, f"ep_bookshelf_write({directory}, {name}): {STATUS_NAMES[rc]}")
    return os.path.join(str(directory), name + ".aux")


class BookshelfDesign:
    """A Bookshelf design parsed by the library (ep_bookshelf_read).
    `netlist` is a synth.Netlist with copies of the parsed arrays;
    write_pl(path, cx, cy) writes movable-node centres back as a .pl file
    under the design's own names (ep_bookshelf_write_pl)."""

    def __init__(self, aux_path, target_density=1.0, bins=0):
        self._L = load()
        c, self._h = Netlist(), ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        rc = self._L.ep_bookshelf_read(str(aux_path).encode(), ctypes.byref(c), ctypes.byref(self._h), err, 512)
        if rc:
            raise EPError(rc, f"ep_bookshelf_read({aux_path}): {err.value.decode()}")
        name = str(aux_path).rsplit("/", 1)[-1].rsplit(".", 1)[0]
        self.netlist = _netlist_copy(c, name, target_density, bins)
        site = np.zeros(c.num_rows, np.float32)
        rc = self._L.ep_bookshelf_row_site_widths(self._h, _p(site, _f32p), int(c.num_rows))
        if rc:
            self.close()
            raise EPError(rc, f"ep_bookshelf_row_site_widths({aux_path}): {STATUS_NAMES[rc]}")
        self.netlist.row_site_w = site

    def write_pl(self, path, node_cx, node_cy):
        cx = np.ascontiguousarray(node_cx, np.float32)
        cy = np.ascontiguousarray(node_cy, np.float32)
        if len(cx) != self.netlist.num_nodes or len(cy) != self.netlist.num_nodes:
            raise ValueError("one centre per movable node")
        rc = self._L.ep_bookshelf_write_pl(self._h, str(path).encode(), _p(cx, _f32p), _p(cy, _f32p))
        if rc:
            raise EPError(rc, f"ep_bookshelf_write_pl({path}): {STATUS_NAMES[rc]}")
        return path

    def write(self, directory, name=None, netlist=None):
        """All files of the design (ep_bookshelf_write) under its own names;
        `netlist` (default: the one read) may carry moved centres."""
        return bookshelf_write(netlist if netlist is not None else self.netlist, directory, name, design=self)

    def close(self):
        if self._h:
            self._L.ep_bookshelf_close(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def create_engines(netlists, params, threads=0):
    """One Engine per netlist (params: one Params, or one per netlist), built
    on a pool of host threads: ep_create's host set-up of one design runs
    beside another's (ctypes releases the interpreter lock for the call).
    threads 0: up to 8, at most one per design.  Each engine is what
    Engine(nl, p) gives alone (its fillers come from its own seed)."""
    import concurrent.futures as cf
    plist = params if isinstance(params, (list, tuple)) else [params] * len(netlists)
    n = threads if threads > 0 else min(8, os.cpu_count() or 1, max(1, len(netlists)))
    if n <= 1:
        return [Engine(nl, p) for nl, p in zip(netlists, plist)]
    with cf.ThreadPoolExecutor(max_workers=n) as ex:
        futs = [ex.submit(Engine, nl, p) for nl, p in zip(netlists, plist)]
        engines, err = [], None
        for f in futs:
            try:
                engines.append(f.result())
            except Exception as x:  # close the others, then raise the first error
                err = err or x
        if err is not None:
            for e in engines:
                e.close()
            raise err
    return engines


def run_batch(engines, max_steps=0):
    """ep_run_batch: the optimizer loops of several engines at once (each
    engine initialized first); returns one run-stats dict per engine."""
    L = load()
    n = len(engines)
    arr = (ctypes.c_void_p * n)(*[e.h.value for e in engines])
    st = (RunStats * n)()
    rc = L.ep_run_batch(arr, n, int(max_steps), st)
    if rc:
        raise EPError(rc, f"ep_run_batch: {STATUS_NAMES[rc]}")
    return [{k: getattr(s, k) for k, _ in RunStats._fields_} for s in st]


def default_params(**kw):
    p = Params()
    load().ep_default_params(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


class Engine:
    """One ep_engine handle (device-resident netlist and placer state)."""

    def __init__(self, nl, params=None, **kw):
        L = load()
        self._L = L
        if params is None:
            params = default_params(target_density=float(nl.target_density),
                                    bins_x=int(nl.bins), bins_y=int(nl.bins))
        for k, v in kw.items():
            setattr(params, k, v)
        self.params = params
        c, self._keep = netlist_struct(nl)
        h = ctypes.c_void_p()
        rc = L.ep_create(ctypes.byref(c), ctypes.byref(params), ctypes.byref(h))
        self.h = h
        if rc != EP_OK:
            msg = L.ep_last_error(h).decode() if h.value else "ep_create failed"
            self.close()
            raise EPError(rc, msg)
        self.info = Info()
        self._check(L.ep_get_info(self.h, ctypes.byref(self.info)))

    def _check(self, rc):
        if rc != EP_OK:
            raise EPError(rc, self._L.ep_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self._L.ep_destroy(self.h)
        self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- sizes ----
    def view_size(self, view):
        i = self.info
        return [i.num_objects, i.num_fillers, i.num_cells_and_fillers][view]

    # ---- wrappers ----
    def get_positions(self, view=MGP):
        n = self.view_size(view)
        xy = np.zeros((n, 2), np.float32)
        self._check(self._L.ep_get_positions(self.h, view, _p(xy, _f32p), n))
        return xy

    def limits(self):
        lim = Limits()
        self._check(self._L.ep_get_limits(self.h, ctypes.byref(lim)))
        return {k: getattr(lim, k) for k, _ in Limits._fields_}

    def set_limits(self, **kw):
        lim = Limits()
        self._check(self._L.ep_get_limits(self.h, ctypes.byref(lim)))
        for k, v in kw.items():
            setattr(lim, k, v)
        self._check(self._L.ep_set_limits(self.h, ctypes.byref(lim)))

    def get_positions_f64(self, view=MGP):
        n = self.view_size(view)
        xy = np.zeros((n, 2), np.float64)
        self._check(self._L.ep_get_positions_f64(self.h, view, _p(xy, _f64p), n))
        return xy

    def set_positions(self, xy, view=MGP):
        xy = np.ascontiguousarray(xy, np.float32).reshape(-1, 2)
        self._check(self._L.ep_set_positions(self.h, view, _p(xy, _f32p), xy.shape[0]))

    def set_positions_ptr(self, host_ptr, count, view=MGP):
        """ep_set_positions from a raw host pointer (e.g. pinned memory)."""
        self._check(self._L.ep_set_positions(self.h, view, ctypes.cast(host_ptr, _f32p), int(count)))

    def get_positions_ptr(self, host_ptr, count, view=MGP):
        self._check(self._L.ep_get_positions(self.h, view, ctypes.cast(host_ptr, _f32p), int(count)))

    def get_gradient(self, view=MGP):
        n = self.view_size(view)
        g = np.zeros((n, 2), np.float32)
        self._check(self._L.ep_get_gradient(self.h, view, _p(g, _f32p), n))
        return g

    def component_gradients(self):
        n = self.info.num_objects
        gd = np.zeros((n, 2), np.float32)
        gw = np.zeros((n, 2), np.float32)
        self._check(self._L.ep_get_component_gradients(self.h, _p(gd, _f32p), _p(gw, _f32p)))
        return gd, gw

    def component_gradients_f64(self):
        n = self.info.num_objects
        gd = np.zeros((n, 2), np.float64)
        gw = np.zeros((n, 2), np.float64)
        self._check(self._L.ep_get_component_gradients_f64(self.h, _p(gd, _f64p), _p(gw, _f64p)))
        return gd, gw

    def field_f64(self):
        nx, ny = self.info.bins_x, self.info.bins_y
        out = {k: np.zeros((nx, ny), np.float64) for k in ("ex", "ey", "phi")}
        self._check(self._L.ep_get_field_f64(self.h, *[_p(out[k], _f64p) for k in ("ex", "ey", "phi")]))
        return out

    def bin_maps(self, which=("node", "filler", "terminal", "base", "ex", "ey", "phi")):
        nx, ny = self.info.bins_x, self.info.bins_y
        out = {k: np.zeros((nx, ny), np.float32) for k in which}
        args = [_p(out[k], _f32p) if k in out else None
                for k in ("node", "filler", "terminal", "base", "ex", "ey", "phi")]
        self._check(self._L.ep_get_bin_maps(self.h, *args))
        return out

    def density_fixed(self):
        nx, ny = self.info.bins_x, self.info.bins_y
        a = np.zeros((nx, ny), np.int64)
        b = np.zeros((nx, ny), np.int64)
        self._check(self._L.ep_get_density_fixed(self.h, _p(a, _i64p), _p(b, _i64p)))
        return a, b

    def query(self):
        s = Scalars()
        self._check(self._L.ep_query(self.h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in Scalars._fields_}

    def initialize(self):
        self._check(self._L.ep_initialize(self.h))

    def eval_gradient(self):
        self._check(self._L.ep_eval_gradient(self.h))

    def set_lambda(self, v):
        self._check(self._L.ep_set_lambda(self.h, float(v)))

    def penalty_init(self):
        self._check(self._L.ep_penalty_init(self.h))

    def penalty_update(self):
        self._check(self._L.ep_penalty_update(self.h))

    def hpwl(self):
        v = ctypes.c_double()
        self._check(self._L.ep_hpwl(self.h, ctypes.byref(v)))
        return v.value

    def quadratic_placement(self, max_iterations=0):
        """QPPlacer::quadraticPlacement on the device; returns its stats."""
        st = QpStats()
        self._check(self._L.ep_quadratic_placement(self.h, int(max_iterations), ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in QpStats._fields_}

    def quadratic_refine(self, rounds, solver_iterations=0, jacobi=False):
        """ep_quadratic_refine: rounds of the quadratic model from the current
        centres (jacobi 1: diagonally preconditioned solves, 0: none)."""
        st = QpStats()
        self._check(self._L.ep_quadratic_refine(self.h, int(rounds), int(solver_iterations), int(jacobi),
                                                ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in QpStats._fields_}

    def switch_stage(self, stage, filler_ll=None):
        a = None if filler_ll is None else np.ascontiguousarray(filler_ll, np.float32)
        self._check(self._L.ep_switch_stage(self.h, stage, _p(a, _f32p)))

    def nesterov_run(self, max_steps=0):
        st = RunStats()
        self._check(self._L.ep_nesterov_run(self.h, int(max_steps), ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in RunStats._fields_}

    def nesterov_begin(self):
        self._check(self._L.ep_nesterov_begin(self.h))

    def nesterov_step(self):
        stopped = ctypes.c_int32(0)
        self._check(self._L.ep_nesterov_step(self.h, ctypes.byref(stopped)))
        return bool(stopped.value)

    def nesterov_end(self):
        self._check(self._L.ep_nesterov_end(self.h))

    def synchronize(self):
        self._check(self._L.ep_synchronize(self.h))

    def save_positions(self):
        self._check(self._L.ep_save_positions(self.h))

    def load_positions(self):
        self._check(self._L.ep_load_positions(self.h))

    def save_state(self):
        """ep_save_state: the optimizer's whole state as bytes (checkpoint)."""
        n = int(self._L.ep_state_size(self.h))
        buf = ctypes.create_string_buffer(n)
        self._check(self._L.ep_save_state(self.h, buf, n))
        return buf.raw

    def load_state(self, blob):
        """ep_load_state: resume from save_state's bytes (same design and
        parameters, after initialize, in the saved stage)."""
        blob = bytes(blob)
        buf = ctypes.create_string_buffer(blob, len(blob))
        self._check(self._L.ep_load_state(self.h, buf, len(blob)))

    def set_stream(self, stream_ptr):
        self._check(self._L.ep_set_stream(self.h, ctypes.c_void_p(stream_ptr)))

    def time_kernels(self, reps=20):
        t = KernelTimes()
        self._check(self._L.ep_time_kernels(self.h, int(reps), ctypes.byref(t)))
        return [dict(name=t.names[i].value.decode(), ms=t.ms[i], bytes=t.bytes[i], flops=t.flops[i],
                     launches=t.launches[i]) for i in range(t.count)]


class EPlacer2D:
    """EPlacer_2D's call surface (EPlace/eplace.h:164-194) over one Engine."""

    def __init__(self, netlist, **params):
        self.netlist = netlist
        self._params = params
        self.targetDensity = float(params.pop("target_density", netlist.target_density))
        self.engine = None

    def setTargetDensity(self, v):
        self.targetDensity = float(v)

    # initialization(): fillers + bins (ep_create), first gradient, lambda_0
    def initialization(self):
        nl = self.netlist
        p = default_params(target_density=self.targetDensity, bins_x=int(nl.bins), bins_y=int(nl.bins))
        for k, v in self._params.items():
            setattr(p, k, v)
        self.engine = Engine(nl, p)
        self.engine.initialize()

    def totalGradientUpdate(self):
        self.engine.eval_gradient()

    def getGradient(self):
        return self.engine.get_gradient(self.placementStage)

    def getPosition(self):
        return self.engine.get_positions(self.placementStage)

    def setPosition(self, xy):
        self.engine.set_positions(xy, self.placementStage)

    def penaltyFactorInitilization(self):
        self.engine.penalty_init()

    def updatePenaltyFactor(self):
        self.engine.penalty_update()

    def switch2FillerOnly(self, filler_ll=None):
        self.engine.switch_stage(FILLERONLY, filler_ll)

    def switch2cGP(self):
        self.engine.switch_stage(CGP)

    def showInfo(self):
        s = self.engine.query()
        print(f"Overflow: {s['overflow']}\npenalty factor: {s['lambda_']:.6f}\nHPWL: {s['last_hpwl']}\n")

    # public fields read by callers (EPlace/eplace.h:108-136)
    @property
    def globalDensityOverflow(self):
        return self.engine.query()["overflow"]

    @property
    def lambda_(self):
        return self.engine.query()["lambda_"]

    @property
    def placementStage(self):
        return self.engine.query()["stage"]

    @property
    def mGPIterationCount(self):
        return self.engine.query()["mgp_iterations"]

    @property
    def binDimension(self):
        return (self.engine.info.bins_x, self.engine.info.bins_y)

    @property
    def binStep(self):
        return (self.engine.info.bin_step_x, self.engine.info.bin_step_y)


class EplaceNesterovOpt:
    """FirstOrderOptimizer<T>::opt with EplaceNesterovOpt's steps
    (Optimization/opt.hpp:30-36, Optimization/nesterov.hpp:86-415); the loop
    itself runs on the device."""

    def __init__(self, placer):
        self.placer = placer
        self.last_run = None

    def opt(self, max_steps=0):
        self.last_run = self.placer.engine.nesterov_run(max_steps)
        return self.last_run


class Gnn:
    """The learned warm start (ep_gnn_*): a message-passing network that
    proposes an initial placement for an Engine."""

    FEATURES = 9

    def __init__(self, device=0, seed=1, weights=None):
        self._L = load()
        self.h = ctypes.c_void_p()
        rc = self._L.ep_gnn_create(int(device), int(seed), ctypes.byref(self.h))
        if rc != EP_OK:
            msg = self._L.ep_gnn_last_error(self.h).decode() if self.h.value else ""
            self.close()
            raise EPError(rc, f"ep_gnn_create: {msg}")
        if weights is not None:
            self.set_weights(weights)

    def _check(self, rc):
        if rc != EP_OK:
            raise EPError(rc, self._L.ep_gnn_last_error(self.h).decode())

    @property
    def num_weights(self):
        return int(self._L.ep_gnn_num_weights())

    def get_weights(self):
        w = np.zeros(self.num_weights, np.float32)
        self._check(self._L.ep_gnn_get_weights(self.h, _p(w, _f32p)))
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        if w.shape != (self.num_weights,):
            raise ValueError(f"expected {self.num_weights} weights")
        self._check(self._L.ep_gnn_set_weights(self.h, _p(w, _f32p)))

    def release(self, engine):
        self._check(self._L.ep_gnn_release(self.h, engine.h))

    def features(self, engine):
        i = engine.info
        x = np.zeros((i.num_nodes + i.num_terminals, self.FEATURES), np.float32)
        self._check(self._L.ep_gnn_features(self.h, engine.h, _p(x, _f32p)))
        return x

    def forward(self, engine):
        """[num_nodes, 4]: the predicted quadratic-placement centre (x, y)
        and final centre (x, y) of each movable node."""
        xy = np.zeros((engine.info.num_nodes, 4), np.float32)
        self._check(self._L.ep_gnn_forward(self.h, engine.h, _p(xy, _f32p)))
        return xy

    def loss_grad(self, engine, target4):
        t = np.ascontiguousarray(target4, np.float32)
        if t.shape != (engine.info.num_nodes, 4):
            raise ValueError("targets: [num_nodes, 4] (QP x, y, final x, y)")
        loss = ctypes.c_double()
        g = np.zeros(self.num_weights, np.float32)
        self._check(self._L.ep_gnn_loss_grad(self.h, engine.h, _p(t, _f32p), ctypes.byref(loss), _p(g, _f32p)))
        return loss.value, g

    def train_step(self, engine, target4, lr):
        t = np.ascontiguousarray(target4, np.float32)
        if t.shape != (engine.info.num_nodes, 4):
            raise ValueError("targets: [num_nodes, 4] (QP x, y, final x, y)")
        loss = ctypes.c_double()
        self._check(self._L.ep_gnn_train_step(self.h, engine.h, _p(t, _f32p), float(lr), ctypes.byref(loss)))
        return loss.value

    def propose(self, engine, alpha=1.0):
        self._check(self._L.ep_gnn_propose(self.h, engine.h, float(alpha)))

    def set_wait_limit(self, polls=None):
        """ep_gnn_set_wait_limit: polls of the tensor-core layers' bounded
        wait before it gives up (None: the default)."""
        self._check(self._L.ep_gnn_set_wait_limit(self.h, -1 if polls is None else int(polls)))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self._L.ep_gnn_destroy(self.h)
        self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
