"""ctypes binding of the C oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py``; never by the product package.  See ``prism_oracle.h``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


def build(force=False):
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE, "ORACLE_CC=gcc"], check=True)
    return LIB_PATH


class Geom(C.Structure):
    _fields_ = [
        ("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32),
        ("n", C.c_uint64),
        ("ax", C.c_uint32), ("ay", C.c_uint32), ("az", C.c_uint32),
        ("anchors", C.c_uint64),
        ("leaps", (C.c_uint64 * 2) * 5),
        ("lm_prefix", C.c_uint64 * 5),
        ("dprefix", C.c_int64 * 5),
        ("align_dev", C.c_int64),
        ("dstride", C.c_int64 * 4),
        ("daprefix", C.c_int64 * 4),
        ("hprefix", C.c_int64 * 5),
        ("align_host", C.c_int64),
        ("hstride", C.c_int64 * 4),
        ("hastride", C.c_int64 * 4),
        ("aligned_size", C.c_uint64),
        ("aligned_len", C.c_uint64),
        ("sh_grid", C.c_int64),
        ("sh_res", C.c_int64),
        ("chunks_level", C.c_int64 * 4),
        ("chunks", C.c_int64),
        ("header_size", C.c_uint64),
    ]


class Intp(C.Structure):
    _fields_ = [("alpha", C.c_double), ("beta", C.c_double),
                ("use_md", C.c_uint8 * 4), ("use_natural", C.c_uint8 * 4),
                ("reverse", C.c_uint8 * 4)]


class Policy(C.Structure):
    _fields_ = [(k, C.c_int) for k in ("quant", "recon", "cubic_md", "cubic_axis", "quad_l",
                                        "quad_r", "att", "line_cubic", "line_quad_l", "line_quad_r",
                                        "face_cubic", "face_quad_l", "face_quad_r", "cube_cubic",
                                        "cube_quad_l", "cube_quad_r")]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB_PATH)
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def geometry(nx, ny, nz, tsize=4):
    g = Geom()
    lib().or_geometry(C.c_uint32(nx), C.c_uint32(ny), C.c_uint32(nz), C.c_int(tsize), C.byref(g))
    return g


def get_policy():
    p = Policy()
    lib().or_get_policy(C.byref(p))
    return {k: getattr(p, k) for k, _ in Policy._fields_}


def set_policy(**kw):
    cur = get_policy()
    cur.update(kw)
    p = Policy(**cur)
    lib().or_set_policy(C.byref(p))


def _suffix(dtype):
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


def intp(use_md, reverse):
    p = Intp()
    p.alpha, p.beta = 1.75, 4.0
    for i in range(4):
        p.use_md[i] = int(use_md[i])
        p.reverse[i] = int(reverse[i])
        p.use_natural[i] = 0
    return p


def compress(data, mode, bound, bt, force=None):
    """data: ndarray [nz][ny][nx]; mode 0 ABS / 1 REL; bt 0 NB / 1 SM.
    Returns (container bytes, (use_md, reverse), errors)."""
    data = np.ascontiguousarray(data)
    nz, ny, nx = data.shape
    g = geometry(nx, ny, nz, data.itemsize)
    cap = data.nbytes + int(g.header_size) + 8 + 2 * int(g.chunks) + (1 << 16)
    out = np.zeros(cap + int(g.aligned_size), dtype=np.uint8)
    used = Intp()
    errs = np.zeros(18, dtype=data.dtype)
    fn = getattr(lib(), "or_compress_" + _suffix(data.dtype))
    fn.restype = C.c_uint64
    size = fn(_p(data), C.c_uint32(nx), C.c_uint32(ny), C.c_uint32(nz), C.c_int(mode),
              C.c_double(bound), C.c_int(bt), C.byref(force) if force is not None else None,
              _p(out), C.byref(used), _p(errs))
    flags = (tuple(used.use_md), tuple(used.reverse))
    return out[:size].tobytes(), flags, errs


def decompress(cont, shape, dtype, mode, bound):
    nz, ny, nx = shape
    buf = np.frombuffer(cont, dtype=np.uint8).copy()
    out = np.zeros(shape, dtype=dtype)
    rc = getattr(lib(), "or_decompress_" + _suffix(dtype))(
        _p(buf), C.c_uint64(len(cont)), C.c_uint32(nx), C.c_uint32(ny), C.c_uint32(nz),
        C.c_int(mode), C.c_double(bound), _p(out))
    if rc:
        raise RuntimeError(f"oracle decompress failed: {rc}")
    return out


class ProgressiveState:
    def __init__(self):
        self.begin = (C.c_int * 4)(0, 0, 0, 0)
        self.end = (C.c_int * 4)(0, 0, 0, 0)
        self.maxlevel = C.c_int(4)
        self.last = 0.0
        self.prev = None


def progressive_step(cont, shape, dtype, mode, bound, target, state, exact=False):
    """One step of the reference's progressive retrieval; exact=True is this
    library's exact refinement (or_progressive_step_exact)."""
    nz, ny, nx = shape
    buf = np.frombuffer(cont, dtype=np.uint8).copy()
    out = np.zeros(shape, dtype=dtype)
    old = state.prev if state.prev is not None else np.zeros(shape, dtype=dtype)
    rc = getattr(lib(), ("or_progressive_step_exact_" if exact else "or_progressive_step_") + _suffix(dtype))(
        _p(buf), C.c_uint64(len(cont)), C.c_uint32(nx), C.c_uint32(ny), C.c_uint32(nz),
        C.c_int(mode), C.c_double(bound), C.c_double(target), C.c_double(state.last),
        state.begin, state.end, C.byref(state.maxlevel), _p(old), _p(out))
    if rc:
        raise RuntimeError(f"oracle progressive step failed: {rc}")
    state.last = target
    state.prev = out
    return out, (list(state.begin), list(state.end), state.maxlevel.value)


# ---- stage-level hooks (for stage-by-stage parity) ----

def predict(data, eb, use_md, reverse, rel_eb):
    data = np.ascontiguousarray(data)
    nz, ny, nx = data.shape
    g = geometry(nx, ny, nz, data.itemsize)
    p = intp(use_md, reverse)
    p.alpha = lib_alpha(rel_eb)
    anchors = np.zeros(int(g.anchors), dtype=data.dtype)
    qc = np.zeros(int(g.n + g.anchors) + 2 * 16384 + 64, dtype=np.int32)
    scratch = np.zeros(int(g.aligned_size) + (1 << 20), dtype=np.uint8)
    getattr(lib(), "or_predict_" + _suffix(data.dtype))(
        _p(data), C.byref(g), C.c_double(eb), C.byref(p), _p(anchors), _p(qc), _p(scratch))
    return anchors, qc, scratch


def reconstruct(qc, anchors, shape, dtype, eb, use_md, reverse, rel_eb, maxlevel=4, old=None):
    """Reconstruction from level-major codes and anchors (or_reconstruct, the
    reference's interpolation_reverse / interpolation_progressive_reverse);
    `old` selects the progressive form."""
    nz, ny, nx = shape
    dtype = np.dtype(dtype)
    g = geometry(nx, ny, nz, dtype.itemsize)
    p = intp(use_md, reverse)
    p.alpha = lib_alpha(rel_eb)
    qc = np.ascontiguousarray(qc, dtype=np.int32)
    anchors = np.ascontiguousarray(anchors, dtype=dtype)
    o = None if old is None else np.ascontiguousarray(old, dtype=dtype)
    out = np.zeros(shape, dtype=dtype)
    getattr(lib(), "or_reconstruct_" + _suffix(dtype))(
        _p(qc), _p(anchors), C.byref(g), C.c_double(eb), C.byref(p), C.c_int(maxlevel),
        _p(o) if o is not None else None, _p(out))
    return out


def lib_alpha(rel_eb):
    f = lib().or_alpha
    f.restype = C.c_double
    return f(C.c_double(rel_eb))


def autotune(data, eb, rel_eb):
    data = np.ascontiguousarray(data)
    nz, ny, nx = data.shape
    g = geometry(nx, ny, nz, data.itemsize)
    errs = np.zeros(18, dtype=data.dtype)
    p = intp([1] * 4, [0] * 4)
    getattr(lib(), "or_autotune_" + _suffix(data.dtype))(
        _p(data), C.byref(g), C.c_double(eb), C.c_double(rel_eb), C.byref(p), _p(errs))
    d = intp([1] * 4, [0] * 4)
    getattr(lib(), "or_decide_" + _suffix(data.dtype))(_p(errs), C.byref(d))
    return errs, (tuple(d.use_md), tuple(d.reverse))


def bitshuffle(qc, g, bt, scratch):
    planes = scratch.copy()
    lib().or_bitshuffle(_p(qc), C.byref(g), C.c_int(bt), _p(planes))
    return planes


def inverse_bitshuffle(planes, g, bt):
    qc = np.zeros(int(g.n + g.anchors) + 2 * 16384 + 64, dtype=np.int32)
    lib().or_inverse_bitshuffle(_p(planes), C.byref(g), C.c_int(bt), _p(qc))
    return qc


def inverse_bitshuffle_progressive(planes, g, begin, end):
    qc = np.zeros(int(g.n + g.anchors) + 2 * 16384 + 64, dtype=np.int32)
    b = (C.c_int * 4)(*begin)
    e = (C.c_int * 4)(*end)
    lib().or_inverse_bitshuffle_progressive(_p(planes), C.byref(g), b, e, _p(qc))
    return qc


def shuffle_network(words):
    w = np.ascontiguousarray(words, dtype=np.uint32)
    o = np.zeros(8, dtype=np.uint32)
    lib().or_shuffle_network(_p(w), _p(o))
    return o


def zbpc_encode(planes, g):
    out = np.zeros(int(g.aligned_size) + 8 + 2 * int(g.chunks) + 64, dtype=np.uint8)
    cs = np.zeros(128, dtype=np.uint64)
    f = lib().or_zbpc_encode
    f.restype = C.c_uint64
    n = f(_p(planes), C.byref(g), _p(out), _p(cs))
    return out[:n].tobytes(), cs


def zbpc_encode_chunk(chunk):
    c = np.ascontiguousarray(chunk, dtype=np.uint8)
    out = np.zeros(max(len(c), 16), dtype=np.uint8)
    n = lib().or_zbpc_encode_chunk(_p(c), C.c_int(len(c)), _p(out))
    return out[:n].tobytes()


def zbpc_decode_chunk(data, osize):
    d = np.frombuffer(bytes(data) + b"\0" * 8, dtype=np.uint8).copy()
    out = np.zeros(osize, dtype=np.uint8)
    rc = lib().or_zbpc_decode_chunk(_p(d), C.c_int(len(data)), C.c_int(osize), _p(out))
    if rc:
        raise ValueError(f"bad chunk ({rc})")
    return out.tobytes()


def find_strategy(cs, eb, target, begin, end):
    c = np.ascontiguousarray(cs, dtype=np.uint64)
    b = (C.c_int * 4)(*begin)
    e = (C.c_int * 4)(*end)
    ml = C.c_int(4)
    lib().or_find_strategy(_p(c), C.c_double(eb), C.c_double(target), b, e, C.byref(ml))
    return list(b), list(e), ml.value


def strategy_costs():
    cost = np.zeros((4, 33), dtype=np.uint64)
    lib().or_strategy_costs(_p(cost))
    return cost
