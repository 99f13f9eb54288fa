"""prism_lossless_encode_static: the lossless encoder that allocates nothing.

Runs through the C ABI and compares with prism_lossless_encode (handle-based)
on the same plane buffers: stream bytes, size and the 128 cumulative plane
sizes must be identical, on two calls in a row and on two different inputs.
Named to run last so it also runs after the other GPU tests in one process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRISM_ERR_LIMIT = -6


@pytest.fixture(scope="module")
def env():
    import torch
    import prism_b200 as P
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch, P


def planes_of_field(torch, P, h, dims, seed):
    """Real plane buffer: predictor + bit-plane shuffle of a sinusoid field."""
    from prism_b200 import fields
    nx, ny, nz = dims
    data = fields.make("sinusoid", (nz, ny, nx), np.float32, seed)
    l = P.lib()
    d_in = torch.from_numpy(data).cuda()
    ncodes = int(l.prism_code_buffer_len(nx, ny, nz))
    codes = torch.zeros(ncodes + 4096, dtype=torch.int32, device="cuda")
    anchors = torch.zeros(ncodes, dtype=torch.float32, device="cuda")
    flags = (C.c_uint8 * 8)(1, 1, 1, 1, 0, 0, 0, 0)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    h.check(l.prism_predict(h.ptr, C.c_void_p(d_in.data_ptr()), 4, nx, ny, nz, C.c_double(1e-4), C.c_double(0.0),
                            flags, C.c_void_p(codes.data_ptr()), C.c_void_p(anchors.data_ptr()), st), "predict")
    planes = torch.zeros(int(l.prism_plane_buffer_size(nx, ny, nz)) + 64, dtype=torch.uint8, device="cuda")
    h.check(l.prism_bitshuffle(h.ptr, C.c_void_p(codes.data_ptr()), nx, ny, nz, 0, C.c_void_p(planes.data_ptr()),
                               st), "bitshuffle")
    torch.cuda.synchronize()
    return planes


def planes_sparse(torch, P, dims, seed):
    """Synthetic plane buffer: zero runs, repeated words and random bytes."""
    nx, ny, nz = dims
    size = int(P.lib().prism_plane_buffer_size(nx, ny, nz))
    rng = np.random.default_rng(seed)
    b = np.zeros(size + 64, dtype=np.uint8)
    dense = rng.random(size) < 0.05
    b[:size][dense] = rng.integers(1, 256, int(dense.sum()), dtype=np.uint8)
    b[size // 3: size // 3 + 40000] = 0xA5          # a long repeated run
    b[size // 2: size // 2 + 20000] = rng.integers(0, 256, 20000, dtype=np.uint8)  # incompressible
    return torch.from_numpy(b).cuda()


def encode_handle(torch, P, h, planes, dims):
    nx, ny, nz = dims
    l = P.lib()
    cap = int(l.prism_max_container_size(nx, ny, nz, 4))
    out = torch.full((cap,), 0x5C, dtype=torch.uint8, device="cuda")
    size = C.c_uint64()
    csbp = (C.c_uint64 * 128)()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    h.check(l.prism_lossless_encode(h.ptr, C.c_void_p(planes.data_ptr()), nx, ny, nz, C.c_void_p(out.data_ptr()),
                                    cap, C.byref(size), csbp, st), "prism_lossless_encode")
    return out[: size.value].cpu().numpy(), size.value, list(csbp)


def encode_static(torch, P, planes, dims, fill):
    nx, ny, nz = dims
    l = P.lib()
    cap = int(l.prism_max_container_size(nx, ny, nz, 4))
    out = torch.full((cap,), fill, dtype=torch.uint8, device="cuda")
    size = C.c_uint64()
    csbp = (C.c_uint64 * 128)()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = l.prism_lossless_encode_static(C.c_void_p(planes.data_ptr()), nx, ny, nz, C.c_void_p(out.data_ptr()), cap,
                                        C.byref(size), csbp, st)
    assert rc == 0, f"prism_lossless_encode_static returned {rc}"
    return out[: size.value].cpu().numpy(), size.value, list(csbp)


@pytest.mark.parametrize("dims", [(64, 48, 40), (200, 130, 97)])
def test_static_encode_matches_handle_encode(env, dims):
    torch, P = env
    h = P.Handle()
    inputs = [planes_of_field(torch, P, h, dims, 3), planes_sparse(torch, P, dims, 7)]
    expected = [encode_handle(torch, P, h, x, dims) for x in inputs]
    # two calls in a row on each input, alternating inputs, different output fill
    for rep in range(2):
        for x, (ref_bytes, ref_size, ref_csbp) in zip(inputs, expected):
            got_bytes, got_size, got_csbp = encode_static(torch, P, x, dims, 0x11 * (rep + 1))
            assert got_size == ref_size
            assert got_csbp == ref_csbp
            assert np.array_equal(got_bytes, ref_bytes)
    h.close()


def test_static_encode_rejects_fields_beyond_its_limit(env):
    """More than 16384 chunks (a 256 MiB plane buffer) is refused before any
    device work, so small dummy buffers are safe here."""
    torch, P = env
    l = P.lib()
    dims = (512, 512, 512)  # 128M values, plane buffer ~512 MiB
    assert l.prism_plane_buffer_size(*dims) > 256 * 2 ** 20
    dummy = torch.zeros(64, dtype=torch.uint8, device="cuda")
    size = C.c_uint64(12345)
    rc = l.prism_lossless_encode_static(C.c_void_p(dummy.data_ptr()), *dims, C.c_void_p(dummy.data_ptr()), 64,
                                        C.byref(size), None, None)
    assert rc == PRISM_ERR_LIMIT
    assert size.value == 12345
