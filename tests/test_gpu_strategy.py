"""Progressive strategy search on the GPU against the oracle's literal
restatement of findStrategy_h (dataloader.cu:179-334): per-thread scans,
per-block and cross-block tree reductions.  Plane-size tables with many
equal-valued candidates make the tie order decide the result, so these cases
check that the GPU's single-key reduction picks the same plane counts."""
import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    import prism_b200 as P
    assert torch.cuda.is_available()
    return torch, P, P.Handle()


def gpu_strategy(torch, P, h, cs, eb, target, begin, end):
    b = (C.c_int * 4)(*begin)
    e = (C.c_int * 4)(*end)
    ml = C.c_int(4)
    c = np.ascontiguousarray(cs, dtype=np.uint64)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    h.check(P.lib().prism_find_strategy(h.ptr, c.ctypes.data_as(C.c_void_p), C.c_double(eb), C.c_double(target), b,
                                        e, C.byref(ml), st), "prism_find_strategy")
    return list(b), list(e), ml.value


def tables():
    rng = np.random.default_rng(7)
    out = []
    # every plane of every level the same size: a huge number of ties
    out.append(np.tile(np.arange(1, 33, dtype=np.uint64) * 1000, 4))
    # two sizes per level, some empty planes
    for _ in range(3):
        per = rng.choice([0, 64, 128], size=(4, 32)).astype(np.uint64)
        out.append(np.cumsum(per, axis=1).reshape(-1))
    # realistic: leading planes small, trailing planes large, level 0 largest
    for _ in range(4):
        per = np.zeros((4, 32), dtype=np.uint64)
        for lv in range(4):
            scale = [2000, 8000, 60000, 500000][lv]
            w = np.exp(np.linspace(-6, 0, 32)) * scale * rng.uniform(0.5, 1.5)
            per[3 - lv] = np.maximum(w, 2).astype(np.uint64)
        out.append(np.cumsum(per, axis=1).reshape(-1))
    return out


RATIOS = [0.9, 1.0, 1.1, 2.0, 10.0, 123.0, 1e3, 5e4, 1e6, 3e8]


def test_strategy_matches_oracle_single_steps(env):
    torch, P, h = env
    eb = 1e-6
    n = 0
    for cs in tables():
        for r in RATIOS:
            got = gpu_strategy(torch, P, h, cs, eb, r * eb, [0] * 4, [0] * 4)
            want = O.find_strategy(cs, eb, r * eb, [0] * 4, [0] * 4)
            assert got == want, (cs[:4], r, got, want)
            n += 1
    assert n == len(RATIOS) * 8


def test_strategy_matches_oracle_in_sequence(env):
    torch, P, h = env
    eb = 2.5e-7
    for cs in tables():
        gb, ge = [0] * 4, [0] * 4
        ob, oe = [0] * 4, [0] * 4
        for r in [1e7, 1e5, 3e3, 40.0, 1.0]:
            gb, ge, gml = gpu_strategy(torch, P, h, cs, eb, r * eb, gb, ge)
            ob, oe, oml = O.find_strategy(cs, eb, r * eb, ob, oe)
            assert (gb, ge, gml) == (ob, oe, oml), (r, gb, ge, gml, ob, oe, oml)


def test_batched_strategy_matches_oracle(env):
    """prism_find_strategy_batch: every (table, ratio) search of the single-step
    test plus searches from mid-sequence states, all in one call, each equal to
    the oracle's step."""
    torch, P, h = env
    eb = 1e-6
    cases = []
    for cs in tables():
        for r in RATIOS:
            cases.append((cs, eb, r * eb, [0] * 4, [0] * 4))
        b, e = [0] * 4, [0] * 4
        for r in [1e7, 1e5, 3e3]:
            b, e, _ = O.find_strategy(cs, eb, r * eb, b, e)
        for r in [40.0, 1.0]:
            cases.append((cs, eb, r * eb, list(b), list(e)))
    n = len(cases)
    cs_all = np.ascontiguousarray(np.stack([c[0] for c in cases]), dtype=np.uint64)
    ebs = np.array([c[1] for c in cases], dtype=np.float64)
    tgs = np.array([c[2] for c in cases], dtype=np.float64)
    begin = np.array([c[3] for c in cases], dtype=np.int32).reshape(-1)
    end = np.array([c[4] for c in cases], dtype=np.int32).reshape(-1)
    ml = np.full(n, 4, dtype=np.int32)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    h.check(P.lib().prism_find_strategy_batch(h.ptr, n, vp(cs_all), vp(ebs), vp(tgs), vp(begin), vp(end), vp(ml),
                                              st), "prism_find_strategy_batch")
    for i, (cs, e_b, tg, b0, e0) in enumerate(cases):
        want = O.find_strategy(cs, e_b, tg, b0, e0)
        got = (list(begin[4 * i: 4 * i + 4]), list(end[4 * i: 4 * i + 4]), int(ml[i]))
        assert got == (list(want[0]), list(want[1]), want[2]), (i, got, want)


def test_batched_strategy_rejects_bad_arguments(env):
    torch, P, h = env
    z = np.zeros(128, dtype=np.uint64)
    one = np.ones(1)
    b = np.zeros(4, dtype=np.int32)
    ml = np.zeros(1, dtype=np.int32)
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    assert P.lib().prism_find_strategy_batch(h.ptr, 0, vp(z), vp(one), vp(one), vp(b), vp(b), vp(ml), None) != 0
    assert P.lib().prism_find_strategy_batch(h.ptr, 1, vp(z), vp(np.zeros(1)), vp(one), vp(b), vp(b), vp(ml),
                                             None) != 0
