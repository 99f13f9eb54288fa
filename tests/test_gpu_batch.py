"""Batched compression (prism_batch_*): every field's container equals the
per-field prism_compress container byte for byte, with and without the CUDA
graph, on replays, for a mix of 1-D/2-D/3-D, float/double, ABS/REL and
sign-magnitude/negabinary fields of uneven shapes."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

# (kind, (nx, ny, nz), dtype, mode, bound, progressive)
MIX = [
    ("sinusoid", (5000, 1, 1), np.float32, 1, 1e-3, False),
    ("grf", (100, 37, 1), np.float32, 0, 1e-3, False),
    ("grf", (33, 56, 64), np.float32, 1, 1e-4, False),
    ("sinusoid", (79, 44, 33), np.float64, 0, 1e-4, True),
    ("voronoi", (64, 48, 40), np.float32, 0, 1e-3, False),
    ("grf", (17, 47, 64), np.float32, 1, 1e-3, True),
    ("sinusoid", (96, 80, 72), np.float64, 1, 1e-6, False),
    ("grf", (300, 200, 1), np.float32, 1, 1e-3, False),
    ("sinusoid", (129, 65, 33), np.float32, 1, 1e-3, False),
]


@pytest.fixture(scope="module")
def env():
    import torch
    import prism_b200 as P
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from prism_b200 import fields
    items, refs, datas = [], [], []
    h = P.Handle()
    for i, (kind, (nx, ny, nz), dt, mode, bound, prog) in enumerate(MIX):
        data = fields.make(kind, (nz, ny, nx), dt, 10 + i)
        d_in = torch.from_numpy(data).cuda()
        ctx = P.Context(nx, ny, nz, np.dtype(dt), mode, bound, prog)
        comp = P.Compressor(ctx, h)
        cont = comp.compress_pipeline(d_in).cpu().numpy().copy()
        items.append((ctx, d_in))
        refs.append((cont, comp.flags))
        datas.append(data)
    torch.cuda.synchronize()
    return torch, P, items, refs, datas


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_matches_per_field_containers(env, use_graph):
    torch, P, items, refs, _ = env
    b = P.Batch(items, use_graph=use_graph)
    for rep in range(2):
        conts, flags = b.compress()
        for i, (c, fl) in enumerate(zip(conts, flags)):
            ref, ref_flags = refs[i]
            got = c.cpu().numpy()
            assert got.size == ref.size, (i, MIX[i], got.size, ref.size)
            assert np.array_equal(got, ref), (i, MIX[i], rep)
            assert fl == ref_flags, (i, fl, ref_flags)
    sch = b.schedule()
    # 0 = one CTA per tile, else persistent CTAs per SM
    assert sch["predict_ctas_per_sm"][0] >= 0 and sch["encode_ctas_per_sm"] >= 1
    assert sch["launches_per_run"] > 0
    b.close()


def test_batch_recompresses_new_contents(env):
    """The graph is bound to the buffers: new data in the same input buffers
    gives the per-field containers of the new data."""
    torch, P, items, refs, _ = env
    b = P.Batch(items[:3], use_graph=True)
    b.compress()
    from prism_b200 import fields
    h = P.Handle()
    for i, (ctx, d_in) in enumerate(items[:3]):
        kind = MIX[i][0]
        new = fields.make(kind, ctx.shape, ctx.dtype, 99 + i)
        d_in.copy_(torch.from_numpy(new))
    conts, _ = b.compress()
    for i, (ctx, d_in) in enumerate(items[:3]):
        ref = P.Compressor(ctx, h).compress_pipeline(d_in).cpu().numpy()
        assert np.array_equal(conts[i].cpu().numpy(), ref)
    b.close()
    # restore the module's inputs
    for i, (ctx, d_in) in enumerate(items[:3]):
        kind, dims, dt = MIX[i][0], MIX[i][1], MIX[i][2]
        d_in.copy_(torch.from_numpy(fields.make(kind, (dims[2], dims[1], dims[0]), dt, 10 + i)))


def test_batch_containers_match_oracle(env):
    """Every batched container equals the oracle's container of that field
    (with the batch's auto-tune decisions forced on the oracle), byte for
    byte: the batched path against the reference's arithmetic directly."""
    torch, P, items, refs, datas = env
    b = P.Batch(items, use_graph=True)
    conts, flags = b.compress()
    for i, (kind, dims, dt, mode, bound, prog) in enumerate(MIX):
        md, rv = flags[i]
        ocont, _, _ = O.compress(datas[i], mode, bound, 0 if prog else 1, force=O.intp(md, rv))
        assert conts[i].cpu().numpy().tobytes() == ocont, (i, MIX[i])
    b.close()
