"""Damaged containers come back as status codes, never as out-of-range
accesses: a truncated container, a size table entry larger than its chunk,
a size table that runs past the stream, and payload bytes flipped (decoded
to some values or reported corrupt).  The decoder checks every offset and
rank against the chunk and the stream before it reads."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    import prism_b200 as P
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from prism_b200 import fields
    nx, ny, nz = 64, 48, 40
    data = fields.make("grf", (nz, ny, nx), np.float32, 6)
    ctx = P.Context(nx, ny, nz, np.dtype(np.float32), P.REL, 1e-4, False)
    comp = P.Compressor(ctx)
    cont = comp.compress_pipeline(torch.from_numpy(data).cuda()).cpu().numpy().copy()
    return torch, P, ctx, cont


def decode(torch, P, ctx, blob):
    comp = P.Compressor(ctx)
    return comp.decompress_pipeline(torch.from_numpy(blob).cuda())


def test_truncated_container(env):
    torch, P, ctx, cont = env
    with pytest.raises(P.PrismError, match="corrupt"):
        decode(torch, P, ctx, cont[:100].copy())


def test_chunk_size_larger_than_chunk(env):
    torch, P, ctx, cont = env
    bad = cont.copy()
    sizes = bad[8:8 + 2 * 16].view(np.uint16)
    sizes[3] = 0xFFFF  # > 16384
    with pytest.raises(P.PrismError, match="corrupt"):
        decode(torch, P, ctx, bad)


def test_size_table_past_the_stream(env):
    torch, P, ctx, cont = env
    bad = cont.copy()
    nchunks = (int(P.lib().prism_plane_buffer_size(ctx.nx, ctx.ny, ctx.nz)) + 16383) // 16384
    sizes = bad[8:8 + 2 * nchunks].view(np.uint16)
    sizes[:] = 16384  # every chunk claims to be raw: the offsets overrun the stream
    with pytest.raises(P.PrismError, match="corrupt"):
        decode(torch, P, ctx, bad)


def test_flipped_payload_bytes_do_not_crash(env):
    torch, P, ctx, cont = env
    rng = np.random.default_rng(1)
    tr = int(P.lib().prism_trailer_size(ctx.nx, ctx.ny, ctx.nz, 4))
    for trial in range(5):
        bad = cont.copy()
        lo = 8 + 2 * 40
        idx = rng.integers(lo, len(bad) - tr, 64)
        bad[idx] ^= rng.integers(1, 256, 64).astype(np.uint8)
        try:
            out = decode(torch, P, ctx, bad)
            torch.cuda.synchronize()
            assert out.shape == ctx.shape
        except P.PrismError as e:
            assert "corrupt" in str(e)
    # the handle and the device stay usable afterwards
    out = decode(torch, P, ctx, cont)
    assert torch.isfinite(out).all()
