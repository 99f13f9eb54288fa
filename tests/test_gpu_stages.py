"""Stage-level GPU parity of the tile kernels under every level-0 mode.

prism_predict with forced per-level flags against the oracle's predictor
(codes and anchors, bit for bit), and prism_reconstruct against the oracle's
full decompression of a container compressed with the same forced flags.
The shapes have interior tiles (the whole 17^3 window inside the field, not
the last tile along any axis) as well as edge tiles, so both kernel parts
run; the flag patterns cover md, per-axis forward and per-axis reverse at
every level, and mixtures."""
import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

# last-slab extents 6/13/1, 2, 2/8; all multiples of 16 (full-size edge
# tiles, as in 384x384x256); 1 and 16 (no interior tile along z)
SHAPES = [(70, 45, 33), (50, 50, 50), (33, 66, 40), (48, 32, 64), (17, 33, 16)]
FLAGS = {
    "md": ([1, 1, 1, 1], [0, 0, 0, 0]),
    "axis": ([0, 0, 0, 0], [0, 0, 0, 0]),
    "axis_rev": ([0, 0, 0, 0], [1, 1, 1, 1]),
    "mixed": ([1, 0, 1, 0], [0, 1, 1, 0]),
    "mixed2": ([0, 1, 0, 1], [1, 0, 0, 1]),
}


@pytest.fixture(scope="module")
def env():
    import torch
    import prism_b200 as P
    assert torch.cuda.is_available()
    return torch, P, P.Handle()


def field(dims, dtype, seed):
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    smooth = np.sin(0.11 * x + 0.05 * y) * np.cos(0.07 * z) + 0.3 * np.sin(0.013 * x * y / 7 + 0.2 * z)
    return (smooth + 0.02 * rng.standard_normal((nz, ny, nx))).astype(dtype)


def gpu_predict(torch, P, h, data, eb, flags8):
    nz, ny, nx = data.shape
    l = P.lib()
    n = int(l.prism_code_buffer_len(nx, ny, nz))
    codes = torch.zeros(n + 4096, dtype=torch.int32, device="cuda")
    anchors = torch.zeros(n, dtype=torch.from_numpy(data[:0]).dtype, device="cuda")
    d_in = torch.from_numpy(data).cuda()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    h.check(l.prism_predict(h.ptr, C.c_void_p(d_in.data_ptr()), data.itemsize, nx, ny, nz, C.c_double(eb),
                            C.c_double(0.0), flags8, C.c_void_p(codes.data_ptr()), C.c_void_p(anchors.data_ptr()),
                            st), "prism_predict")
    return codes, anchors


@pytest.mark.parametrize("flag_name", list(FLAGS))
@pytest.mark.parametrize("dims", SHAPES)
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_predict_and_reconstruct_forced_flags(env, dims, dtype, flag_name):
    torch, P, h = env
    md, rv = FLAGS[flag_name]
    nx, ny, nz = dims
    data = field(dims, dtype, sum(dims) + 7 * list(FLAGS).index(flag_name))
    eb = 1e-3
    flags8 = (C.c_uint8 * 8)(*md, *rv)
    codes, anchors = gpu_predict(torch, P, h, data, eb, flags8)
    o_anchors, o_qc, _ = O.predict(data, eb, md, rv, 0.0)
    n = nx * ny * nz
    g = O.geometry(nx, ny, nz, data.itemsize)
    na = int(g.anchors)
    assert np.array_equal(anchors[:na].cpu().numpy().view(np.uint8), o_anchors.view(np.uint8))
    assert np.array_equal(codes[:n].cpu().numpy(), o_qc[:n]), "codes differ from the oracle"

    # reconstruction from the same codes against the oracle's (the full
    # pipeline also passes the codes through the bit planes, whose last-block
    # quirk alters some codes on some shapes; that path has its own tests)
    l = P.lib()
    out = torch.empty((nz, ny, nx), dtype=torch.from_numpy(data[:0]).dtype, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    h.check(l.prism_reconstruct(h.ptr, C.c_void_p(codes.data_ptr()), C.c_void_p(anchors.data_ptr()), data.itemsize,
                                nx, ny, nz, C.c_double(eb), C.c_double(0.0), flags8, 4, None,
                                C.c_void_p(out.data_ptr()), st), "prism_reconstruct")
    ref = O.reconstruct(o_qc, o_anchors, (nz, ny, nx), dtype, eb, md, rv, 0.0)
    rec = out.cpu().numpy()
    assert np.array_equal(rec.view(np.uint8), ref.view(np.uint8)), "reconstruction differs from the oracle"

    # the progressive form (previous values added), also at a lower maxlevel
    old_np = field(dims, dtype, 5)
    old = torch.from_numpy(old_np).cuda()
    out2 = torch.empty_like(out)
    for maxlevel in (4, 2):
        h.check(l.prism_reconstruct(h.ptr, C.c_void_p(codes.data_ptr()), C.c_void_p(anchors.data_ptr()),
                                    data.itemsize, nx, ny, nz, C.c_double(eb), C.c_double(0.0), flags8, maxlevel,
                                    C.c_void_p(old.data_ptr()), C.c_void_p(out2.data_ptr()), st),
                "prism_reconstruct progressive")
        ref2 = O.reconstruct(o_qc, o_anchors, (nz, ny, nx), dtype, eb, md, rv, 0.0, maxlevel, old_np)
        assert np.array_equal(out2.cpu().numpy().view(np.uint8), ref2.view(np.uint8)), f"maxlevel {maxlevel}"


@pytest.mark.parametrize("dims", [(70, 45, 33), (48, 32, 64)])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_reconstruct_from_unaligned_code_buffer(env, dims, dtype):
    """Interior tiles load their level-0 codes in 16-byte pieces when the code
    buffer is 16-byte aligned and by 4-byte copies otherwise: a buffer one
    code off alignment gives the same bytes, fresh and progressive."""
    torch, P, h = env
    md, rv = FLAGS["md"]
    nx, ny, nz = dims
    data = field(dims, dtype, 11)
    eb = 1e-3
    flags8 = (C.c_uint8 * 8)(*md, *rv)
    codes, anchors = gpu_predict(torch, P, h, data, eb, flags8)
    shifted = torch.zeros(codes.numel() + 4, dtype=torch.int32, device="cuda")
    shifted[1:1 + codes.numel()] = codes
    assert (codes.data_ptr() % 16, shifted[1:].data_ptr() % 16) == (0, 4)
    l = P.lib()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    old = torch.from_numpy(field(dims, dtype, 5)).cuda()
    for prev in (None, old):
        outs = []
        for buf in (codes, shifted[1:]):
            out = torch.empty((nz, ny, nx), dtype=old.dtype, device="cuda")
            h.check(l.prism_reconstruct(h.ptr, C.c_void_p(buf.data_ptr()), C.c_void_p(anchors.data_ptr()),
                                        data.itemsize, nx, ny, nz, C.c_double(eb), C.c_double(0.0), flags8, 4,
                                        None if prev is None else C.c_void_p(prev.data_ptr()),
                                        C.c_void_p(out.data_ptr()), st), "prism_reconstruct")
            outs.append(out.cpu().numpy())
        assert np.array_equal(outs[0].view(np.uint8), outs[1].view(np.uint8))
