"""The engine's binary netlist file in numpy (the C side is
ep_netbin_write / ep_netbin_open in csrc/netbin.cu, with the layout written
out there): a header, then the netlist arrays as raw little-endian data,
each on a 64-byte boundary, so loading is a memory map instead of a parse.

    write(nl, path)      -> path
    read(path, mmap=True) -> synth.Netlist
"""
import numpy as np

from .synth import Netlist

MAGIC = b"EPNETBN1"
VERSION = 1
# (field, dtype, count key) in file order
ARRAYS = (
    ("node_w", np.float32, "nn"), ("node_h", np.float32, "nn"), ("node_cx", np.float32, "nn"),
    ("node_cy", np.float32, "nn"), ("term_llx", np.float32, "nt"), ("term_lly", np.float32, "nt"),
    ("term_w", np.float32, "nt"), ("term_h", np.float32, "nt"), ("term_is_ni", np.uint8, "nt"),
    ("net_start", np.int32, "nnet1"), ("pin_owner", np.int32, "np"), ("pin_dx", np.float32, "np"),
    ("pin_dy", np.float32, "np"), ("row_llx", np.float32, "nr"), ("row_lly", np.float32, "nr"),
    ("row_urx", np.float32, "nr"), ("row_h", np.float32, "nr"), ("row_site_w", np.float32, "nr"),
)
HEADER = 48 + 8 * len(ARRAYS)


def _align(x):
    return (x + 63) & ~63


def _counts(nn, nt, nnet, nr, np_):
    return dict(nn=nn, nt=nt, nnet1=nnet + 1, nr=nr, np=np_)


def write(nl, path, common_row_height=0.0):
    nn, nt, nnet, nr, np_ = nl.num_nodes, nl.num_terminals, nl.num_nets, nl.num_rows, nl.num_pins
    cnt = _counts(nn, nt, nnet, nr, np_)
    offs, pos = [], _align(HEADER)
    for name, dt, key in ARRAYS:
        offs.append(pos)
        pos = _align(pos + np.dtype(dt).itemsize * cnt[key])
    head = bytearray(_align(HEADER))
    head[0:8] = MAGIC
    head[8:16] = np.array([VERSION, len(ARRAYS)], "<u4").tobytes()
    head[16:36] = np.array([nn, nt, nnet, nr, np_], "<i4").tobytes()
    head[36:44] = np.array([common_row_height, nl.target_density], "<f4").tobytes()
    head[44:48] = np.array([nl.bins], "<i4").tobytes()
    head[48:HEADER] = np.array(offs, "<u8").tobytes()
    with open(path, "wb") as f:
        f.write(head)
        at = len(head)
        for (name, dt, key), off in zip(ARRAYS, offs):
            f.write(b"\0" * (off - at))
            a = np.ascontiguousarray(getattr(nl, name), dtype=np.dtype(dt).newbyteorder("<"))
            assert a.size == cnt[key], name
            f.write(a.tobytes())
            at = off + a.nbytes
    return path


def read(path, mmap=True):
    raw = np.memmap(path, np.uint8, "r") if mmap else np.fromfile(path, np.uint8)
    if bytes(raw[:8]) != MAGIC:
        raise ValueError(f"{path}: not an engine netlist file")
    ver, narr = np.frombuffer(raw[8:16], "<u4")
    if ver != VERSION or narr != len(ARRAYS):
        raise ValueError(f"{path}: version {ver} with {narr} arrays is not supported")
    nn, nt, nnet, nr, np_ = (int(v) for v in np.frombuffer(raw[16:36], "<i4"))
    crh, td = (float(v) for v in np.frombuffer(raw[36:44], "<f4"))
    bins = int(np.frombuffer(raw[44:48], "<i4")[0])
    offs = np.frombuffer(raw[48:HEADER], "<u8")
    cnt = _counts(nn, nt, nnet, nr, np_)
    fields = {}
    for (name, dt, key), off in zip(ARRAYS, offs):
        n = cnt[key]
        fields[name] = np.frombuffer(raw, np.dtype(dt).newbyteorder("<"), count=n, offset=int(off))
    return Netlist(name=path.rsplit("/", 1)[-1].split(".")[0], target_density=td, bins=bins,
                   meta=dict(common_row_height=crh), **fields)
