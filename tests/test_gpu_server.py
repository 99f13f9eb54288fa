"""Progressive-retrieval server (prism_server_*): each request's values equal
the standalone one-step retrieval of its field at its bound, bit for bit
(tolerance 0), whether it ran alone or in a mix of concurrent requests with
cache hits, shared computations and evictions under a tight HBM budget."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = [
    ("grf", (64, 48, 40), np.float64, 1, 1e-6),
    ("sinusoid", (96, 40, 33), np.float32, 1, 1e-5),
    ("voronoi", (50, 60, 30), np.float32, 0, 1e-4),
]
TARGETS = [1e-1, 1e-2, 1e-3, 1e-4, 1e-5, 1e-6]


@pytest.fixture(scope="module")
def env():
    import torch
    import prism_b200 as P
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from prism_b200 import fields
    out = []
    h = P.Handle()
    for i, (kind, (nx, ny, nz), dt, mode, bound) in enumerate(FIELDS):
        data = fields.make(kind, (nz, ny, nx), dt, 30 + i)
        ctx = P.Context(nx, ny, nz, np.dtype(dt), mode, bound, True)
        comp = P.Compressor(ctx, h)
        cont = comp.compress_pipeline(torch.from_numpy(data).cuda()).clone()
        out.append((ctx, cont, comp))
    return torch, P, out


def standalone(P, comp, cont, target):
    """One-step progressive retrieval of `cont` at `target`, alone."""
    pg = comp.progressive(cont)
    v = pg.step(target).clone()
    pg.close()
    return v


def requests():
    rng = np.random.default_rng(5)
    reqs = []
    for k in range(30):
        f = int(rng.integers(0, len(FIELDS)))
        scale = 1.0 if FIELDS[f][3] == 1 else 1e-2  # ABS fields: bounds in data units
        t = TARGETS[int(rng.integers(0, len(TARGETS)))] * scale
        reqs.append((f, max(t, FIELDS[f][4])))
    return reqs


def test_server_results_equal_standalone_in_a_mix(env):
    torch, P, flds = env
    reqs = requests()
    expect = {}
    for f, t in set(reqs):
        ctx, cont, comp = flds[f]
        expect[(f, t)] = standalone(P, comp, cont, t)
    # budget: containers + workspaces + room for about two reconstructions
    probe = P.Server(1 << 40, slots=3)
    for ctx, cont, _ in flds:
        probe.add_field(ctx, cont)
    st0 = probe.stats()
    probe.close()
    vbytes = max(np.prod(c.shape) * c.tsize for c, _, _ in flds)
    budget = int(st0["bytes_resident"] + st0["bytes_reserved"] + 2.2 * vbytes)
    srv = P.Server(budget, slots=3)
    ids = [srv.add_field(ctx, cont) for ctx, cont, _ in flds]
    outs, rids = [], []
    for f, t in reqs:
        ctx = flds[f][0]
        o = torch.full(ctx.shape, float("nan"), dtype=torch.float32 if ctx.tsize == 4 else torch.float64,
                       device="cuda")
        outs.append(o)
        rids.append(srv.submit(ids[f], t, o))
    infos = [srv.wait(r) for r in rids]
    for (f, t), o, info in zip(reqs, outs, infos):
        assert torch.equal(o, expect[(f, t)]), (f, t, info)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["cache_hits"] + st["shared"] > 0
    assert st["evictions"] > 0
    assert st["bytes_peak"] <= budget
    assert 0 < st["p50_ms"] <= st["p99_ms"]
    srv.close()


def test_server_host_output_and_alone(env):
    torch, P, flds = env
    srv = P.Server(1 << 34, slots=1)
    ctx, cont, comp = flds[0]
    fid = srv.add_field(ctx, cont.cpu().numpy())
    h_out = np.empty(ctx.shape, dtype=np.float64)
    info = srv.wait(srv.submit(fid, 1e-4, h_out))
    ref = standalone(P, comp, cont, 1e-4).cpu().numpy()
    assert np.array_equal(h_out, ref)
    assert not info["from_cache"]
    # the same request again is served from the resident reconstruction
    h2 = np.empty_like(h_out)
    info2 = srv.wait(srv.submit(fid, 1e-4, h2))
    assert info2["from_cache"] and np.array_equal(h2, ref)
    srv.close()


def test_server_budget_is_enforced(env):
    torch, P, flds = env
    ctx, cont, _ = flds[0]
    srv = P.Server(1024, slots=1)
    with pytest.raises(P.PrismError):
        srv.add_field(ctx, cont)
    srv.close()
