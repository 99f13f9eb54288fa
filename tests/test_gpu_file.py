"""Container files: prism_file_save writes the container bytes; progressive
retrieval from the file gives the same values as from the in-memory
container at every step and reads only the chunks of the planes it adds."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    import prism_b200 as P
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch, P


@pytest.mark.parametrize("dt,mode,bound", [(np.float64, 1, 1e-6), (np.float32, 0, 1e-4)])
def test_file_progressive_equals_memory(env, tmp_path, dt, mode, bound):
    torch, P = env
    from prism_b200 import fields
    nx, ny, nz = 96, 80, 64
    data = fields.make("grf", (nz, ny, nx), dt, 21)
    ctx = P.Context(nx, ny, nz, np.dtype(dt), mode, bound, True)
    comp = P.Compressor(ctx)
    cont = comp.compress_pipeline(torch.from_numpy(data).cuda()).clone()
    path = tmp_path / "field.prisma"
    P.save_container(path, cont)
    assert np.array_equal(np.fromfile(path, dtype=np.uint8), cont.cpu().numpy())
    mem = comp.progressive(cont)
    fil = P.FileProgressive(P.Compressor(ctx), path)
    scale = 1.0 if mode == 1 else 1e-1
    reads = []
    ost = O.ProgressiveState()
    host = cont.cpu().numpy().tobytes()
    for t in [1e-1, 1e-3, 1e-5, 1e-6]:
        t = max(t * scale, bound)
        a = mem.step(t).clone()
        b = fil.step(t)
        assert torch.equal(a, b), t
        # and the oracle's progressive chain, bit for bit
        o, _ = O.progressive_step(host, (nz, ny, nx), dt, mode, bound, t, ost)
        assert np.array_equal(b.cpu().numpy().view(np.uint8), o.view(np.uint8)), t
        reads.append(fil.info()["bytes_read"])
        assert fil.info()["end"] == mem.state()[1]
    info = fil.info()
    assert reads == sorted(reads)
    assert reads[0] < info["file_bytes"]        # the coarse step read a part of the file
    assert info["bytes_read"] <= info["file_bytes"] + 2 * 8 * 2 ** 20
    fil.close()
    mem.close()
