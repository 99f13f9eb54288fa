"""Failure detection on the GPU without a fault: the lossless encoder's
look-back wait gives up after a bounded number of polls.

prism_lossless_wait_selftest runs the encoder with its chunk tickets starting
at 1, so chunk 0 never publishes its size and the waits that reach it run
out.  The call must come back with PRISM_ERR_TIMEOUT within milliseconds (the
kernel sets an error flag and returns; nothing hangs), and the next normal
encode on the same handle must give the same stream as before."""
import ctypes as C
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_lookback_wait_runs_out_and_handle_recovers():
    import torch
    import prism_b200 as P
    assert torch.cuda.is_available()
    l = P.lib()
    h = P.Handle()
    nx, ny, nz = 96, 80, 64
    pbytes = int(l.prism_plane_buffer_size(nx, ny, nz))
    rng = np.random.default_rng(5)
    planes = rng.integers(0, 256, pbytes, dtype=np.uint8)
    planes[rng.random(pbytes) < 0.7] = 0  # mixed raw and eliminated chunks
    d_planes = torch.from_numpy(planes).cuda()
    cap = pbytes + 2 * (pbytes // 16384 + 256) + 64
    d_stream = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    size = C.c_uint64()

    def encode():
        rc = l.prism_lossless_encode(h.ptr, C.c_void_p(d_planes.data_ptr()), nx, ny, nz,
                                     C.c_void_p(d_stream.data_ptr()), cap, C.byref(size), None, st)
        assert rc == 0, P.lib().prism_last_error(h.ptr)
        return bytes(d_stream[: size.value].cpu().numpy())

    before = encode()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = l.prism_lossless_wait_selftest(h.ptr, C.c_void_p(d_planes.data_ptr()), nx, ny, nz,
                                        C.c_void_p(d_stream.data_ptr()), cap, 2000, st)
    dt = time.perf_counter() - t0
    assert rc == -4  # PRISM_ERR_TIMEOUT
    assert dt < 2.0, dt
    assert b"look-back" in l.prism_last_error(h.ptr)
    after = encode()
    assert after == before
    # bad arguments are refused before any device work
    assert l.prism_lossless_wait_selftest(h.ptr, C.c_void_p(d_planes.data_ptr()), nx, ny, nz,
                                          C.c_void_p(d_stream.data_ptr()), cap, 0, st) == -1
    h.close()
