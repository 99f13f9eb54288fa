"""prism_b200 -- B200-native PRISM compression hot path.

Python side of the C ABI in ``include/prism_b200.h``.  Device memory is held in
torch CUDA tensors (plumbing only); every computation runs in the sm_100a
kernels of ``libprism_b200.so``.  There is no CPU fallback: importing works on
any machine, but every call needs the library and a CUDA device and raises
``PrismError`` otherwise.

The names mirror the reference's ``prism::Compressor`` pipeline
(include/compressor.hpp:35-83) and ``prism_context`` (include/utils/
parameters.hpp:27-56): ``Context`` carries dims, dtype, error mode, bound and
the SM/NB plane coding; ``Compressor`` offers ``compress_pipeline``,
``decompress_pipeline`` and ``decompress_progressive_pipeline``.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import _build

LIB_PATH = _build.LIB
ABS, REL = 0, 1
SM, NB = 0, 1  # progressive=0 -> sign-magnitude planes, 1 -> negabinary

_STATUS = {0: "ok", -1: "bad argument", -2: "CUDA error", -3: "corrupt container",
           -4: "device wait timed out", -5: "out of device memory",
           -6: "input larger than the entry point's fixed limit"}


class PrismError(RuntimeError):
    pass


_lib = None


def lib():
    """Load libprism_b200.so (fails loudly if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PrismError(f"{LIB_PATH} is missing: run prism_b200._build.build_lib()")
        l = C.CDLL(LIB_PATH)
        vp, u32, u64, i32, dbl = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_double
        l.prism_create.argtypes = [C.POINTER(vp)]
        l.prism_destroy.argtypes = [vp]
        l.prism_last_error.argtypes = [vp]
        l.prism_last_error.restype = C.c_char_p
        for fn in ("prism_max_container_size", "prism_trailer_size"):
            getattr(l, fn).argtypes = [u32, u32, u32, i32]
            getattr(l, fn).restype = u64
        for fn in ("prism_plane_buffer_size", "prism_code_buffer_len"):
            getattr(l, fn).argtypes = [u32, u32, u32]
            getattr(l, fn).restype = u64
        l.prism_compress.argtypes = [vp, vp, i32, u32, u32, u32, i32, dbl, i32, vp, u64, C.POINTER(u64), vp, vp]
        l.prism_compress_host.argtypes = [vp, vp, i32, u32, u32, u32, i32, dbl, i32, vp, u64, C.POINTER(u64), vp]
        l.prism_decompress.argtypes = [vp, vp, u64, i32, u32, u32, u32, i32, dbl, vp, vp]
        l.prism_decompress_host.argtypes = [vp, vp, u64, i32, u32, u32, u32, i32, dbl, vp, vp]
        l.prism_progressive_open.argtypes = [vp, vp, u64, i32, u32, u32, u32, i32, dbl, C.POINTER(vp)]
        l.prism_progressive_step.argtypes = [vp, dbl, vp, vp]
        l.prism_progressive_step_into.argtypes = [vp, dbl, vp, vp, vp]
        l.prism_progressive_state.argtypes = [vp, vp, vp, vp, vp]
        l.prism_progressive_close.argtypes = [vp]
        l.prism_extrema.argtypes = [vp, vp, i32, u64, C.POINTER(dbl), vp]
        l.prism_autotune.argtypes = [vp, vp, i32, u32, u32, u32, vp, vp, vp]
        l.prism_predict.argtypes = [vp, vp, i32, u32, u32, u32, dbl, dbl, vp, vp, vp, vp]
        l.prism_reconstruct.argtypes = [vp, vp, vp, i32, u32, u32, u32, dbl, dbl, vp, i32, vp, vp, vp]
        l.prism_bitshuffle.argtypes = [vp, vp, u32, u32, u32, i32, vp, vp]
        l.prism_inverse_bitshuffle.argtypes = [vp, vp, u32, u32, u32, i32, vp, vp, vp, vp]
        l.prism_lossless_encode.argtypes = [vp, vp, u32, u32, u32, vp, u64, C.POINTER(u64), vp, vp]
        l.prism_lossless_decode.argtypes = [vp, vp, u32, u32, u32, vp, vp, vp, vp]
        l.prism_find_strategy.argtypes = [vp, vp, dbl, dbl, vp, vp, vp, vp]
        l.prism_find_strategy_batch.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp, vp]
        l.prism_lossless_encode_static.argtypes = [vp, u32, u32, u32, vp, u64, C.POINTER(u64), vp, vp]
        l.prism_lossless_wait_selftest.argtypes = [vp, vp, u32, u32, u32, vp, u64, C.c_longlong, vp]
        l.prism_extrema_minmax.argtypes = [vp, vp, i32, u64, vp, vp]
        l.prism_progressive_resume.argtypes = [vp, vp, vp]
        l.prism_progressive_exact.argtypes = [vp, C.c_int]
        l.prism_server_set_refine.argtypes = [vp, i32]
        l.prism_lost_codes.argtypes = [u32, u32, u32]
        l.prism_lost_codes.restype = u64
        l.prism_batch_create.argtypes = [vp, i32, i32, C.POINTER(vp)]
        l.prism_batch_compress.argtypes = [vp, vp, vp, vp]
        l.prism_batch_schedule.argtypes = [vp, vp, vp, vp, vp]
        l.prism_batch_last_error.argtypes = [vp]
        l.prism_batch_last_error.restype = C.c_char_p
        l.prism_batch_destroy.argtypes = [vp]
        l.prism_statistics.argtypes = [vp, vp, vp, i32, u64, vp, C.POINTER(u64), vp]
        l.prism_file_save.argtypes = [C.c_char_p, vp, u64, vp]
        l.prism_file_open.argtypes = [vp, C.c_char_p, i32, u32, u32, u32, i32, dbl, C.POINTER(vp)]
        l.prism_file_step.argtypes = [vp, dbl, vp, vp]
        l.prism_file_info.argtypes = [vp, C.POINTER(u64), C.POINTER(u64), vp]
        l.prism_file_close.argtypes = [vp]
        l.prism_server_create.argtypes = [u64, i32, C.POINTER(vp)]
        l.prism_server_add_field.argtypes = [vp, vp, u64, i32, i32, u32, u32, u32, i32, dbl, C.POINTER(i32)]
        l.prism_server_submit.argtypes = [vp, i32, dbl, vp, i32, C.POINTER(u64)]
        l.prism_server_wait.argtypes = [vp, u64, C.POINTER(dbl), vp, C.POINTER(i32), C.POINTER(i32)]
        l.prism_server_stats_get.argtypes = [vp, vp, i32]
        l.prism_server_poll.argtypes = [vp, u64, C.POINTER(i32)]
        l.prism_server_destroy.argtypes = [vp]
        l.prism_profile.argtypes = [vp, i32]
        l.prism_profile_stages.argtypes = [vp, u32]
        l.prism_stage_times.argtypes = [vp, vp, vp, i32, i32]
        l.prism_launch_count.argtypes = [vp]
        l.prism_launch_count.restype = u64
        _lib = l
    return _lib


EXPORTED = [
    "prism_create", "prism_destroy", "prism_last_error", "prism_max_container_size",
    "prism_plane_buffer_size", "prism_trailer_size", "prism_compress", "prism_compress_host",
    "prism_decompress", "prism_decompress_host", "prism_progressive_open", "prism_progressive_step",
    "prism_progressive_state", "prism_progressive_close", "prism_extrema", "prism_autotune",
    "prism_code_buffer_len", "prism_predict", "prism_reconstruct", "prism_bitshuffle",
    "prism_inverse_bitshuffle", "prism_lossless_encode", "prism_lossless_decode", "prism_find_strategy",
    "prism_find_strategy_batch",
    "prism_profile", "prism_stage_times", "prism_launch_count", "prism_lossless_encode_static",
    "prism_batch_create", "prism_batch_compress", "prism_batch_schedule", "prism_batch_last_error",
    "prism_batch_destroy", "prism_server_create", "prism_server_add_field", "prism_server_submit",
    "prism_server_wait", "prism_server_stats_get", "prism_server_destroy", "prism_statistics", "prism_server_poll",
    "prism_file_save", "prism_file_open", "prism_file_step", "prism_file_info", "prism_file_close",
    "prism_progressive_step_into", "prism_profile_stages", "prism_lossless_wait_selftest", "prism_lost_codes",
    "prism_extrema_minmax", "prism_progressive_resume", "prism_progressive_exact", "prism_server_set_refine",
]


def lost_codes(nx, ny, nz):
    """Level-0 codes whose bits the reference's last shuffle block does not
    carry for these dimensions (the container keeps the reference's bytes, so
    their points may miss the bound); 0 for shapes without the effect.
    Geometry only."""
    return int(lib().prism_lost_codes(nx, ny, nz))

STAGES = ["extrema", "autotune", "predict", "shuffle", "encode", "trailer", "strategy", "decode",
          "inverse_shuffle", "reconstruct"]


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise PrismError("prism_b200 needs a CUDA device")
    return torch


class Handle:
    """Owns a prism_handle (device workspace cache)."""

    def __init__(self):
        self.ptr = C.c_void_p()
        rc = lib().prism_create(C.byref(self.ptr))
        if rc:
            raise PrismError(f"prism_create failed ({_STATUS.get(rc, rc)})")

    def check(self, rc, what):
        if rc:
            msg = lib().prism_last_error(self.ptr)
            raise PrismError(f"{what}: {_STATUS.get(rc, rc)}: {msg.decode() if msg else ''}")

    def profile(self, enable=True, stages=None):
        """Stage timing on/off; `stages` (names from STAGES) limits it to those."""
        if stages is None:
            self.check(lib().prism_profile(self.ptr, int(enable)), "prism_profile")
        else:
            mask = sum(1 << STAGES.index(s) for s in stages) if enable else 0
            self.check(lib().prism_profile_stages(self.ptr, mask), "prism_profile_stages")

    def stage_times(self, reset=True):
        ms = (C.c_double * 16)()
        cnt = (C.c_int * 16)()
        n = lib().prism_stage_times(self.ptr, ms, cnt, 16, int(reset))
        return {STAGES[i]: (ms[i], cnt[i]) for i in range(min(n, len(STAGES)))}

    def statistics(self, d_original, d_data):
        """Error statistics of d_data against d_original (CUDA tensors)."""
        torch = _torch()
        out = (C.c_double * 7)()
        idx = C.c_uint64()
        self.check(lib().prism_statistics(self.ptr, C.c_void_p(d_original.data_ptr()), C.c_void_p(d_data.data_ptr()),
                                          d_original.element_size(), d_original.numel(), out, C.byref(idx),
                                          _stream(torch)), "prism_statistics")
        keys = ["max_err", "max_rel_err", "psnr", "nrmse", "min", "max", "l2"]
        r = dict(zip(keys, list(out)))
        r["max_err_index"] = idx.value
        return r

    def launches(self):
        return int(lib().prism_launch_count(self.ptr))

    def close(self):
        if self.ptr:
            lib().prism_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _stream(torch):
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


@dataclass
class Context:
    """The fields of the reference's prism_context that the path uses."""
    nx: int
    ny: int = 1
    nz: int = 1
    dtype: np.dtype = np.dtype(np.float32)
    error_mode: int = REL
    bound: float = 1e-4          # -R rel_eb or -A eb
    progressive: bool = False    # -prog (negabinary planes)
    targets: list = field(default_factory=list)  # -errors

    @property
    def tsize(self):
        return np.dtype(self.dtype).itemsize

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)


class Compressor:
    """Device-side compress / decompress / progressive retrieval of one field."""

    def __init__(self, ctx: Context, handle: Handle | None = None):
        self.ctx = ctx
        self.h = handle or Handle()
        self.flags = None

    def max_container_size(self):
        c = self.ctx
        return int(lib().prism_max_container_size(c.nx, c.ny, c.nz, c.tsize))

    def compress_pipeline(self, d_in, d_out=None):
        """d_in: CUDA tensor of the field; returns a uint8 CUDA tensor (container)."""
        torch = _torch()
        c = self.ctx
        cap = self.max_container_size()
        if d_out is None:
            d_out = torch.empty(cap, dtype=torch.uint8, device=d_in.device)
        size = C.c_uint64(0)
        flags = (C.c_uint8 * 8)()
        rc = lib().prism_compress(self.h.ptr, C.c_void_p(d_in.data_ptr()), c.tsize, c.nx, c.ny, c.nz,
                                  c.error_mode, c.bound, int(c.progressive), C.c_void_p(d_out.data_ptr()),
                                  d_out.numel(), C.byref(size), flags, _stream(torch))
        self.h.check(rc, "prism_compress")
        self.flags = (tuple(flags[:4]), tuple(flags[4:]))
        return d_out[: size.value]

    def decompress_pipeline(self, d_cont, d_out=None):
        torch = _torch()
        c = self.ctx
        if d_out is None:
            d_out = torch.empty(c.shape, dtype=_torch_dtype(torch, c.dtype), device=d_cont.device)
        rc = lib().prism_decompress(self.h.ptr, C.c_void_p(d_cont.data_ptr()), d_cont.numel(), c.tsize, c.nx,
                                    c.ny, c.nz, c.error_mode, c.bound, C.c_void_p(d_out.data_ptr()),
                                    _stream(torch))
        self.h.check(rc, "prism_decompress")
        return d_out

    def progressive(self, d_cont):
        return Progressive(self, d_cont)


class Progressive:
    """decompress_progressive_pipeline as a resident object: each step refines
    the reconstruction in place (compressor.cu:166-190).  Steps are enqueued
    on the current stream without waiting; state() waits and reports errors."""

    def __init__(self, comp: Compressor, d_cont):
        torch = _torch()
        self.comp = comp
        self.cont = d_cont
        c = comp.ctx
        self.ptr = C.c_void_p()
        rc = lib().prism_progressive_open(comp.h.ptr, C.c_void_p(d_cont.data_ptr()), d_cont.numel(), c.tsize, c.nx,
                                          c.ny, c.nz, c.error_mode, c.bound, C.byref(self.ptr))
        comp.h.check(rc, "prism_progressive_open")
        self.values = torch.zeros(c.shape, dtype=_torch_dtype(torch, c.dtype), device=d_cont.device)

    def step(self, target):
        torch = _torch()
        rc = lib().prism_progressive_step(self.ptr, target, C.c_void_p(self.values.data_ptr()), _stream(torch))
        self.comp.h.check(rc, "prism_progressive_step")
        return self.values

    def step_into(self, target, prev, out):
        """The step out of place (output_old -> output_new, compressor.hpp:80):
        reads the previous step's values from `prev` (None on the first step)
        and writes the refined values to `out`."""
        torch = _torch()
        rc = lib().prism_progressive_step_into(self.ptr, target, C.c_void_p(prev.data_ptr()) if prev is not None
                                               else None, C.c_void_p(out.data_ptr()), _stream(torch))
        self.comp.h.check(rc, "prism_progressive_step_into")
        return out

    def resume(self, end):
        """Start from values that hold planes [0, end[l]) of every level (before
        the first step); the next step_into refines them."""
        torch = _torch()
        e = (C.c_int * 4)(*end)
        self.comp.h.check(lib().prism_progressive_resume(self.ptr, e, _stream(torch)), "prism_progressive_resume")

    def exact(self, enable=True):
        """Exact refinement (prism_progressive_exact): later steps also decode
        the chunks of the plane below their range, so every step's values
        equal the one-step retrieval to its planes up to rounding."""
        self.comp.h.check(lib().prism_progressive_exact(self.ptr, int(bool(enable))), "prism_progressive_exact")

    def state(self):
        """Plane state after the last step (waits for it; raises on a corrupt chunk)."""
        b = (C.c_int * 4)()
        e = (C.c_int * 4)()
        ml = C.c_int()
        self.comp.h.check(lib().prism_progressive_state(self.ptr, b, e, C.byref(ml), None), "prism_progressive_state")
        return list(b), list(e), ml.value

    def close(self):
        if self.ptr:
            lib().prism_progressive_close(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def save_container(path, d_cont):
    """Write a device container (uint8 CUDA tensor) to a file."""
    torch = _torch()
    rc = lib().prism_file_save(str(path).encode(), C.c_void_p(d_cont.data_ptr()), d_cont.numel(), _stream(torch))
    if rc:
        raise PrismError(f"prism_file_save: {_STATUS.get(rc, rc)}")


class FileProgressive:
    """Progressive retrieval straight from a container file: each step reads
    only the chunks of the planes it adds."""

    def __init__(self, comp: Compressor, path):
        torch = _torch()
        c = comp.ctx
        self.comp = comp
        self.ptr = C.c_void_p()
        comp.h.check(lib().prism_file_open(comp.h.ptr, str(path).encode(), c.tsize, c.nx, c.ny, c.nz, c.error_mode,
                                           c.bound, C.byref(self.ptr)), "prism_file_open")
        self.values = torch.zeros(c.shape, dtype=_torch_dtype(torch, c.dtype), device="cuda")

    def step(self, target):
        torch = _torch()
        self.comp.h.check(lib().prism_file_step(self.ptr, target, C.c_void_p(self.values.data_ptr()), _stream(torch)),
                          "prism_file_step")
        return self.values

    def info(self):
        fb, br = C.c_uint64(), C.c_uint64()
        end = (C.c_int * 4)()
        lib().prism_file_info(self.ptr, C.byref(fb), C.byref(br), end)
        return {"file_bytes": fb.value, "bytes_read": br.value, "end": list(end)}

    def close(self):
        if self.ptr:
            lib().prism_file_close(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FieldDesc(C.Structure):
    """prism_field_desc: one field of a batch (device buffers)."""
    _fields_ = [("d_in", C.c_void_p), ("d_out", C.c_void_p), ("out_capacity", C.c_uint64), ("nx", C.c_uint32),
                ("ny", C.c_uint32), ("nz", C.c_uint32), ("dtype_size", C.c_int), ("mode", C.c_int),
                ("bound", C.c_double), ("progressive", C.c_int)]


class Batch:
    """Batched compression of many fields (prism_batch_*): one launch per stage
    over all fields, a schedule tuned on the batch, the pipeline captured in a
    CUDA graph.  `items` is a list of (Context, device input tensor); output
    buffers are allocated here and stay bound to the batch."""

    def __init__(self, items, use_graph=True):
        torch = _torch()
        self.items = items
        self.outs = []
        descs = (FieldDesc * len(items))()
        for i, (ctx, d_in) in enumerate(items):
            cap = int(lib().prism_max_container_size(ctx.nx, ctx.ny, ctx.nz, ctx.tsize))
            out = torch.empty(cap, dtype=torch.uint8, device=d_in.device)
            self.outs.append(out)
            descs[i] = FieldDesc(d_in.data_ptr(), out.data_ptr(), cap, ctx.nx, ctx.ny, ctx.nz, ctx.tsize,
                                 ctx.error_mode, ctx.bound, int(ctx.progressive))
        self.ptr = C.c_void_p()
        rc = lib().prism_batch_create(descs, len(items), int(use_graph), C.byref(self.ptr))
        if rc:
            raise PrismError(f"prism_batch_create: {_STATUS.get(rc, rc)}")

    def compress(self):
        """Returns the list of containers (views into the bound outputs) and flags."""
        torch = _torch()
        n = len(self.items)
        sizes = (C.c_uint64 * n)()
        flags = (C.c_uint8 * (8 * n))()
        rc = lib().prism_batch_compress(self.ptr, _stream(torch), sizes, flags)
        if rc:
            raise PrismError(f"prism_batch_compress: {_STATUS.get(rc, rc)}: "
                             f"{lib().prism_batch_last_error(self.ptr).decode()}")
        conts = [self.outs[i][: sizes[i]] for i in range(n)]
        fl = [(tuple(flags[8 * i:8 * i + 4]), tuple(flags[8 * i + 4:8 * i + 8])) for i in range(n)]
        return conts, fl

    def schedule(self):
        pred = (C.c_int * 2)()
        enc = C.c_int()
        ms = (C.c_double * 2)()
        launches = C.c_uint64()
        lib().prism_batch_schedule(self.ptr, pred, C.byref(enc), ms, C.byref(launches))
        return {"predict_ctas_per_sm": list(pred), "encode_ctas_per_sm": enc.value,
                "tuned_ms": list(ms), "launches_per_run": launches.value}

    def close(self):
        if self.ptr:
            lib().prism_batch_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("completed", "cache_hits", "shared", "evictions", "failed", "bytes_out",
                                          "bytes_resident", "bytes_reserved", "bytes_peak")] + \
               [(k, C.c_double) for k in ("p50_ms", "p99_ms", "mean_ms", "max_ms", "elapsed_s", "queue_p50_ms",
                                          "queue_p99_ms", "service_p50_ms", "service_p99_ms")] + \
               [("refined", C.c_uint64), ("plan_calls", C.c_uint64)]


class Server:
    """Progressive-retrieval server (prism_server_*): -prog containers and
    reconstructions resident on the device, requests served by `slots`
    worker threads under an HBM budget (bytes)."""

    def __init__(self, hbm_budget, slots=4):
        self.ptr = C.c_void_p()
        rc = lib().prism_server_create(int(hbm_budget), int(slots), C.byref(self.ptr))
        if rc:
            raise PrismError(f"prism_server_create: {_STATUS.get(rc, rc)}")
        self.fields = []

    def add_field(self, ctx: Context, container):
        """container: uint8 CUDA tensor or numpy array of a -prog container."""
        fid = C.c_int()
        on_dev = hasattr(container, "is_cuda") and container.is_cuda
        ptr = container.data_ptr() if on_dev else container.ctypes.data
        n = container.numel() if on_dev else container.size
        rc = lib().prism_server_add_field(self.ptr, C.c_void_p(ptr), n, int(on_dev), ctx.tsize, ctx.nx, ctx.ny,
                                          ctx.nz, ctx.error_mode, ctx.bound, C.byref(fid))
        if rc:
            raise PrismError(f"prism_server_add_field: {_STATUS.get(rc, rc)}")
        self.fields.append(ctx)
        return fid.value

    def refine(self, enable=True):
        """Refine misses from resident coarser reconstructions (default on)."""
        rc = lib().prism_server_set_refine(self.ptr, int(enable))
        if rc:
            raise PrismError(f"prism_server_set_refine: {_STATUS.get(rc, rc)}")

    def submit(self, field_id, target, out):
        """out: CUDA tensor (or numpy array) of the field's shape and dtype."""
        rid = C.c_uint64()
        on_dev = hasattr(out, "is_cuda") and out.is_cuda
        ptr = out.data_ptr() if on_dev else out.ctypes.data
        rc = lib().prism_server_submit(self.ptr, int(field_id), float(target), C.c_void_p(ptr), int(on_dev),
                                       C.byref(rid))
        if rc:
            raise PrismError(f"prism_server_submit: {_STATUS.get(rc, rc)}")
        return rid.value

    def wait(self, request_id):
        lat = C.c_double()
        end = (C.c_int * 4)()
        ml = C.c_int()
        hit = C.c_int()
        rc = lib().prism_server_wait(self.ptr, C.c_uint64(request_id), C.byref(lat), end, C.byref(ml), C.byref(hit))
        if rc:
            raise PrismError(f"prism_server_wait: {_STATUS.get(rc, rc)}")
        return {"latency_ms": lat.value, "end": list(end), "maxlevel": ml.value, "from_cache": hit.value == 1,
                "refined": hit.value == 2}

    def done(self, request_id):
        d = C.c_int()
        rc = lib().prism_server_poll(self.ptr, C.c_uint64(request_id), C.byref(d))
        if rc:
            raise PrismError(f"prism_server_poll: {_STATUS.get(rc, rc)}")
        return bool(d.value)

    def stats(self, reset=False):
        st = ServerStats()
        lib().prism_server_stats_get(self.ptr, C.byref(st), int(reset))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def close(self):
        if self.ptr:
            lib().prism_server_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _torch_dtype(torch, dt):
    return torch.float32 if np.dtype(dt) == np.float32 else torch.float64
