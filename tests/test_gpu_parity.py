"""GPU parity tests: the sm_100a path through the C ABI against the reference's
golden vectors and the CPU oracle, bit for bit."""
import ctypes as C

import numpy as np
import pytest

import golden_util as gu
import oracle as O

pytestmark = pytest.mark.gpu

SMALL = ["clean_f32", "clean_f64", "short_f32", "sparse_f32", "line1d_f32", "plane2d_f32", "spill_a"]
SMALL_PROG = ["clean_f32_prog", "clean_f64_prog", "sparse_f32_prog"]


@pytest.fixture(scope="module")
def env():
    import torch
    import prism_b200 as P
    assert torch.cuda.is_available()
    return torch, P, P.Handle()


def mode_of(c):
    return 1 if c["mode"] == "R" else 0


def ctx_of(P, name):
    c = gu.CASES[name]
    nx, ny, nz = c["dims"]
    return P.Context(nx, ny, nz, np.dtype(gu.dtype_of(c)), mode_of(c), c["bound"], c["bt"] == "NB",
                     c.get("targets", []))


def to_dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host_bytes(t):
    return t.cpu().numpy().tobytes()


@pytest.mark.parametrize("name", SMALL + SMALL_PROG)
def test_compress_matches_reference_container(env, name):
    torch, P, h = env
    comp = P.Compressor(ctx_of(P, name), h)
    cont = host_bytes(comp.compress_pipeline(to_dev(torch, gu.field(name))))
    md, rv = gu.flags(name)
    assert comp.flags == (tuple(md), tuple(rv)), "auto-tune decisions differ from the reference"
    size, digest = gu.digests(name)["cmp.bin"]
    assert len(cont) == size
    assert gu.sha(np.frombuffer(cont, np.uint8)) == digest


@pytest.mark.parametrize("name", [n for n in SMALL if gu.CASES[n]["bt"] == "SM"])
def test_decompress_reference_container(env, name):
    torch, P, h = env
    comp = P.Compressor(ctx_of(P, name), h)
    cont = to_dev(torch, np.frombuffer(gu.raw(name, "cmp.bin"), np.uint8))
    out = comp.decompress_pipeline(cont).cpu().numpy()
    assert gu.sha(out) == gu.digests(name)["dec.bin"][1]


@pytest.mark.parametrize("name", SMALL_PROG)
def test_progressive_reference_container(env, name):
    torch, P, h = env
    comp = P.Compressor(ctx_of(P, name), h)
    cont = to_dev(torch, np.frombuffer(gu.raw(name, "cmp.bin"), np.uint8))
    prog = comp.progressive(cont)
    ref = gu.steps(name)
    dg = gu.digests(name)
    for i, t in enumerate(gu.CASES[name]["targets"]):
        out = prog.step(t).cpu().numpy()
        b, e, ml = prog.state()
        assert (b, e, ml) == (ref[i][1], ref[i][2], ref[i][3])
        assert gu.sha(out) == dg[f"prog{i}.bin"][1], f"step {i}"
    prog.close()


@pytest.mark.parametrize("name", SMALL_PROG)
def test_progressive_out_of_place_reference_container(env, name):
    """Steps through two alternating buffers (output_old -> output_new, as the
    reference's CLI runs them) give the reference's bytes and leave the
    previous step's buffer untouched."""
    torch, P, h = env
    comp = P.Compressor(ctx_of(P, name), h)
    cont = to_dev(torch, np.frombuffer(gu.raw(name, "cmp.bin"), np.uint8))
    prog = comp.progressive(cont)
    dg = gu.digests(name)
    bufs = [torch.full_like(prog.values, 7.0), torch.full_like(prog.values, 7.0)]
    prev = None
    for i, t in enumerate(gu.CASES[name]["targets"]):
        out = bufs[i % 2]
        before = prev.clone() if prev is not None else None
        prog.step_into(t, prev, out)
        prog.state()
        assert gu.sha(out.cpu().numpy()) == dg[f"prog{i}.bin"][1], f"step {i}"
        if prev is not None:
            assert torch.equal(prev, before)
        prev = out
    prog.close()


def test_progressive_step_into_arguments(env):
    """The out-of-place step accepts no previous buffer on the first step only,
    and rejects a non-positive target."""
    torch, P, h = env
    name = SMALL_PROG[0]
    comp = P.Compressor(ctx_of(P, name), h)
    cont = to_dev(torch, np.frombuffer(gu.raw(name, "cmp.bin"), np.uint8))
    prog = comp.progressive(cont)
    l, st = P.lib(), C.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = torch.empty_like(prog.values)
    t0 = gu.CASES[name]["targets"][0]
    assert l.prism_progressive_step_into(prog.ptr, 0.0, None, C.c_void_p(out.data_ptr()), st) == -1
    assert l.prism_progressive_step_into(prog.ptr, t0, None, C.c_void_p(out.data_ptr()), st) == 0
    prog.state()
    assert gu.sha(out.cpu().numpy()) == gu.digests(name)["prog0.bin"][1]
    assert l.prism_progressive_step_into(prog.ptr, t0, None, C.c_void_p(out.data_ptr()), st) == -1
    prog.close()


RANDOM_SHAPES = [(40, 23, 17), (70, 45, 33), (129, 3, 5), (300, 41, 1), (2000, 1, 1), (16, 16, 16), (17, 17, 17),
                 (48, 48, 48)]


@pytest.mark.parametrize("dims", RANDOM_SHAPES)
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_compress_matches_oracle_random_shapes(env, dims, dtype):
    """Full pipeline vs the oracle, with the GPU's own flags forced on the
    oracle so that auto-tune near-ties cannot mask a difference."""
    torch, P, h = env
    nx, ny, nz = dims
    rng = np.random.default_rng(hash(dims) % 1000)
    data = (rng.standard_normal((nz, ny, nx)).cumsum(axis=2) * 0.1).astype(dtype)
    for mode, bound, prog in [(1, 1e-3, False), (0, 1e-2, True)]:
        ctx = P.Context(nx, ny, nz, np.dtype(dtype), mode, bound, prog)
        comp = P.Compressor(ctx, h)
        cont = host_bytes(comp.compress_pipeline(to_dev(torch, data)))
        md, rv = comp.flags
        ocont, oflags, _ = O.compress(data, mode, bound, 0 if prog else 1, force=O.intp(md, rv))
        assert cont == ocont
        out = comp.decompress_pipeline(to_dev(torch, np.frombuffer(cont, np.uint8))).cpu().numpy() if not prog else None
        if out is not None:
            oout = O.decompress(ocont, (nz, ny, nx), dtype, mode, bound)
            assert np.array_equal(out.view(np.uint8), oout.view(np.uint8))


def test_compress_is_deterministic(env):
    torch, P, h = env
    name = "clean_f32"
    comp = P.Compressor(ctx_of(P, name), h)
    d = to_dev(torch, gu.field(name))
    a = host_bytes(comp.compress_pipeline(d))
    b = host_bytes(comp.compress_pipeline(d))
    assert a == b


def test_sinusoids_128_matches_reference(env):
    """128^3 float sinusoids at REL 1e-4: container and round trip
    equal the reference build's."""
    torch, P, h = env
    name = "c0"
    comp = P.Compressor(ctx_of(P, name), h)
    cont = comp.compress_pipeline(to_dev(torch, gu.field(name)))
    dg = gu.digests(name)
    assert gu.sha(cont.cpu().numpy()) == dg["cmp.bin"][1]
    out = comp.decompress_pipeline(cont).cpu().numpy()
    assert gu.sha(out) == dg["dec.bin"][1]
