"""GPU error statistics (prism_statistics, the reference's --report cr
numbers), progressive loaded bytes, and the CLI's compress/decompress flow
with --report."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def env():
    import torch
    import prism_b200 as P
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch, P


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_statistics_match_numpy(env, dt):
    torch, P = env
    rng = np.random.default_rng(3)
    ori = rng.normal(0, 1, 1_000_003).astype(dt)
    dat = (ori + rng.normal(0, 1e-3, ori.size)).astype(dt)
    for i in (777, 900_001):  # the max error 0.5 (exact), reached twice
        ori[i], dat[i] = dt(0.25), dt(0.75)
    h = P.Handle()
    s = h.statistics(torch.from_numpy(ori).cuda(), torch.from_numpy(dat).cuda())
    err = np.abs((dat - ori).astype(np.float64))
    assert s["max_err"] == err.max()
    assert s["max_err_index"] == 777 == int(np.argmax(err))  # first index reaching the max
    assert s["min"] == float(ori.min()) and s["max"] == float(ori.max())
    l2 = float(np.sum(err * err))
    assert s["l2"] == pytest.approx(l2, rel=1e-12)
    rng_ = float(ori.max()) - float(ori.min())
    mse = l2 / ori.size
    assert s["psnr"] == pytest.approx(20 * np.log10(rng_) - 10 * np.log10(mse), abs=1e-9)
    assert s["nrmse"] == pytest.approx(np.sqrt(mse) / rng_, rel=1e-12)


def test_progressive_loaded_bytes(env):
    torch, P = env
    from prism_b200 import fields
    import ctypes as C
    nx, ny, nz = 64, 48, 40
    data = fields.make("grf", (nz, ny, nx), np.float64, 4)
    ctx = P.Context(nx, ny, nz, np.dtype(np.float64), P.REL, 1e-6, True)
    comp = P.Compressor(ctx)
    cont = comp.compress_pipeline(torch.from_numpy(data).cuda())
    host = cont.cpu().numpy()
    tr = len(host) - int(P.lib().prism_trailer_size(nx, ny, nz, 8))
    cum = np.frombuffer(host[tr + 16: tr + 1040].tobytes(), np.uint64)
    sizes = np.diff(np.concatenate([[0], cum.astype(np.int64)]))
    pg = comp.progressive(cont)
    prev = 0
    for t in [1e-2, 1e-4, 1e-6]:
        pg.step(t)
        b, e = (C.c_int * 4)(), (C.c_int * 4)()
        ml, loaded = C.c_int(), C.c_uint64()
        P.lib().prism_progressive_state(pg.ptr, b, e, C.byref(ml), C.byref(loaded))
        expect = sum(int(sizes[i * 32 + j]) for i in range(4) for j in range(e[i]))
        assert loaded.value == expect and loaded.value >= prev
        prev = loaded.value
    pg.close()


def test_cli_roundtrip_with_report(env, tmp_path):
    torch, P = env
    from prism_b200 import fields
    nx, ny, nz = 48, 40, 33
    data = fields.make("sinusoid", (nz, ny, nx), np.float32, 8)
    src = tmp_path / "field.f32"
    data.tofile(src)
    cli = os.path.join(ROOT, "prism_b200", "bin", "prism")
    p = subprocess.run([cli, "-i", str(src), "-f", "-3", str(nx), str(ny), str(nz), "-R", "1e-3", "-z", "-x",
                        "--report", "time,cr"], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert "PSNR" in p.stdout and "compression ratio" in p.stdout
    cont = np.fromfile(str(src) + ".prisma", dtype=np.uint8)
    ctx = P.Context(nx, ny, nz, np.dtype(np.float32), P.REL, 1e-3, False)
    ref = P.Compressor(ctx).compress_pipeline(torch.from_numpy(data).cuda()).cpu().numpy()
    assert np.array_equal(cont, ref)
    dec = np.fromfile(str(src) + ".prisma.out", dtype=np.float32).reshape(data.shape)
    got = P.Compressor(ctx).decompress_pipeline(torch.from_numpy(cont).cuda()).cpu().numpy()
    assert np.array_equal(dec, got)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_extrema_on_unaligned_slices(env, dtype):
    """prism_extrema on slices that start off a 16-byte boundary, with lengths
    of 1 to the whole buffer: the range is max - min in double, with the
    extreme values placed near the start and near the end."""
    import ctypes as C
    torch, P = env
    h = P.Handle()
    rng = np.random.default_rng(5)
    base = rng.standard_normal((1 << 20) + 7).astype(dtype)
    base[1] = 50.0     # in the head of an offset-1 slice
    base[-2] = -70.0   # in the tail
    d = torch.from_numpy(base).cuda()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for off in (0, 1, 2, 3):
        for length in (1, 3, 17, base.size - off - 1, base.size - off):
            sl = d[off:off + length]
            rng_out = C.c_double()
            h.check(P.lib().prism_extrema(h.ptr, C.c_void_p(sl.data_ptr()), base.itemsize, length,
                                          C.byref(rng_out), st), "prism_extrema")
            host = base[off:off + length]
            want = float(host.max()) - float(host.min())
            assert rng_out.value == want, (off, length, rng_out.value, want)
