"""CPU tests: the oracle against the reference's golden vectors, and the
oracle's own invariants.  No GPU needed."""
import os

import numpy as np
import pytest

import golden_util as gu
import oracle as O

SMALL = ["clean_f32", "clean_f64", "short_f32", "sparse_f32", "line1d_f32", "plane2d_f32", "spill_a"]
SMALL_PROG = ["clean_f32_prog", "clean_f64_prog", "sparse_f32_prog"]


def mode_of(c):
    return 1 if c["mode"] == "R" else 0


@pytest.mark.parametrize("name", SMALL + SMALL_PROG)
def test_oracle_container_matches_reference(name):
    """Compress with the reference's interpolation flags: the container bytes
    equal the reference build's (byte parity, every stage)."""
    c = gu.CASES[name]
    md, rv = gu.flags(name)
    cont, _, _ = O.compress(gu.field(name), mode_of(c), c["bound"], 1 if c["bt"] == "SM" else 0,
                            force=O.intp(md, rv))
    size, digest = gu.digests(name)["cmp.bin"]
    assert len(cont) == size
    assert gu.sha(np.frombuffer(cont, np.uint8)) == digest


@pytest.mark.parametrize("name", SMALL)
def test_oracle_autotune_flags_match_reference(name):
    c = gu.CASES[name]
    _, flags, _ = O.compress(gu.field(name), mode_of(c), c["bound"], 1 if c["bt"] == "SM" else 0)
    md, rv = gu.flags(name)
    assert flags == (tuple(md), tuple(rv))


@pytest.mark.parametrize("name", [n for n in SMALL if gu.CASES[n]["bt"] == "SM"])
def test_oracle_decompress_matches_reference(name):
    c = gu.CASES[name]
    nx, ny, nz = c["dims"]
    cont = gu.raw(name, "cmp.bin")
    out = O.decompress(cont, (nz, ny, nx), gu.dtype_of(c), mode_of(c), c["bound"])
    assert gu.sha(out) == gu.digests(name)["dec.bin"][1]


@pytest.mark.parametrize("name", SMALL_PROG)
def test_oracle_progressive_matches_reference(name):
    c = gu.CASES[name]
    nx, ny, nz = c["dims"]
    cont = gu.raw(name, "cmp.bin")
    st = O.ProgressiveState()
    ref_steps = gu.steps(name)
    dg = gu.digests(name)
    for i, t in enumerate(c["targets"]):
        out, (b, e, ml) = O.progressive_step(cont, (nz, ny, nx), gu.dtype_of(c), mode_of(c), c["bound"], t, st)
        assert (b, e, ml) == (ref_steps[i][1], ref_steps[i][2], ref_steps[i][3])
        assert gu.sha(out) == dg[f"prog{i}.bin"][1]


def test_shuffle_network_closed_form():
    """The reference's 8-lane shuffle network is a plain bit transpose: bit
    7-l of plane byte p is bit 31-p of word l."""
    rng = np.random.default_rng(0)
    for _ in range(300):
        w = rng.integers(0, 2**32, 8, dtype=np.uint64).astype(np.uint32)
        o = O.shuffle_network(w)
        for p in range(32):
            k, j = divmod(p, 4)
            byte = (int(o[k]) >> (24, 8, 16, 0)[j]) & 0xFF
            want = sum(((int(w[l]) >> (31 - p)) & 1) << (7 - l) for l in range(8))
            assert byte == want


def test_zbpc_chunk_roundtrip_and_format():
    rng = np.random.default_rng(1)
    for osize in (16384, 8, 4096 + 8, 12480):
        for density in (0.0, 0.001, 0.05, 0.5, 1.0):
            chunk = np.where(rng.random(osize) < density, rng.integers(1, 256, osize), 0).astype(np.uint8)
            enc = O.zbpc_encode_chunk(chunk)
            assert len(enc) <= osize
            if density == 0.0:
                assert enc == bytes([osize & 0xFF, osize >> 8])
            assert O.zbpc_decode_chunk(enc, osize) == chunk.tobytes()


def test_strategy_costs_exact():
    """cost[l][b] = ceil(2^(32-b) * sum of three powers of 1.25) is exact."""
    from fractions import Fraction
    cost = O.strategy_costs()
    for l in range(4):
        p = Fraction(1) if l == 0 else Fraction(5, 4)
        s = p ** (11 - 3 * l) + p ** (10 - 3 * l) + p ** (9 - 3 * l)
        for b in range(33):
            v = 0 if b == 32 else Fraction(2 ** (32 - b)) * s
            assert int(cost[l][b]) == -((-v.numerator) // v.denominator)


def test_oracle_roundtrip_bound_random_shapes():
    """Non-progressive round trip honours the bound on shapes the reference
    handles without its last-block quirks."""
    rng = np.random.default_rng(5)
    checked = 0
    for shape in [(20, 33, 17), (64, 40, 17), (31, 45, 18), (16, 32, 32), (64, 56, 33)]:
        g = O.geometry(shape[2], shape[1], shape[0])
        tail = g.n % 16384 or 16384
        covered = (g.sh_grid - 1) * 16384 + tail >= g.n + g.align_dev
        if not (g.align_dev == 0 and tail % 8 == 0 and covered):
            continue
        data = rng.standard_normal(shape).cumsum(axis=2).astype(np.float32)
        cont, _, _ = O.compress(data, 0, 1e-2, 1)
        out = O.decompress(cont, shape, np.float32, 0, 1e-2)
        # float32 arithmetic: the bound holds up to a few ulps of the data
        slack = 8 * np.finfo(np.float32).eps * float(np.abs(data).max())
        assert np.abs(out.astype(np.float64) - data).max() <= 1e-2 + slack
        checked += 1
    assert checked >= 1


def test_oracle_predictor_bound_every_shape():
    """The predictor alone (codes straight back into the reconstruction, no
    bit planes) honours the bound on every shape, including those where the
    reference's last shuffle block alters codes; progressive reconstruction
    at maxlevel 4 adds the previous values."""
    rng = np.random.default_rng(9)
    for shape in [(64, 32, 48), (16, 33, 17), (33, 45, 70), (5, 3, 129), (1, 1, 300)]:
        for dtype in (np.float32, np.float64):
            data = (rng.standard_normal(shape).cumsum(axis=2) * 0.1).astype(dtype)
            for md, rv in (([1] * 4, [0] * 4), ([0] * 4, [1] * 4), ([0, 1, 0, 1], [1, 0, 0, 1])):
                anchors, qc, _ = O.predict(data, 1e-3, md, rv, 0.0)
                out = O.reconstruct(qc, anchors, shape, dtype, 1e-3, md, rv, 0.0)
                slack = 8 * np.finfo(dtype).eps * float(np.abs(data).max())
                assert np.abs(out.astype(np.float64) - data).max() <= 1e-3 + slack
                old = np.ones(shape, dtype=dtype)
                prog = O.reconstruct(qc, anchors, shape, dtype, 1e-3, md, rv, 0.0, 4, old)
                assert np.array_equal(prog, (out + old).astype(dtype))


def test_exact_refinement_equals_one_step():
    """The oracle's exact refinement (the chunks of plane begin - 1 decoded
    as well) ends every chain within a few ulps of the one-step retrieval to
    the same planes, while the reference's chain 1e-2 -> 1e-4 on a double
    field with 8-byte-multiple planes misses the head of the first new plane
    and ends far outside the 1e-4 bound."""
    from prism_b200 import fields
    data = fields.make("grf", (40, 48, 64), np.float64, 30)
    shape, rng = data.shape, float(data.max() - data.min())
    cont, _, _ = O.compress(data, 1, 1e-6, 0)
    ulp = float(np.spacing(np.abs(data).max()))
    one, _ = O.progressive_step(cont, shape, np.float64, 1, 1e-6, 1e-4, O.ProgressiveState())
    for exact in (False, True):
        st = O.ProgressiveState()
        O.progressive_step(cont, shape, np.float64, 1, 1e-6, 1e-2, st, exact=exact)
        two, (b, e, ml) = O.progressive_step(cont, shape, np.float64, 1, 1e-6, 1e-4, st, exact=exact)
        d = np.abs(two - one).max()
        if exact:
            assert d <= 16 * ulp and np.abs(two - data).max() <= 1e-4 * rng
        else:
            assert d > 1e-3 * rng and np.abs(two - data).max() > 1e-3 * rng


@pytest.mark.parametrize("kind,shape,dtype,mode,bound", [
    ("grf", (24, 40, 56), np.float64, 1, 1e-6),
    ("sinusoid", (33, 40, 48), np.float32, 1, 1e-5),
    ("voronoi", (30, 45, 50), np.float32, 0, 1e-4),
    ("grf", (17, 33, 65), np.float32, 1, 1e-5),
])
def test_exact_chains_equal_one_step(kind, shape, dtype, mode, bound):
    """Chains of three exact-refinement steps end every step within a few
    ulps of the largest magnitude of the one-step retrieval to the same
    planes, on shapes with and without 8-byte-multiple planes."""
    from prism_b200 import fields
    data = fields.make(kind, shape, dtype, 7)
    cont, _, _ = O.compress(data, mode, bound, 0)
    scale = 1.0 if mode == 1 else float(np.abs(data).max())
    ulp = float(np.spacing(np.array(np.abs(data).max(), dtype=dtype)))
    st = O.ProgressiveState()
    for t in (1e-1, 1e-3, 1e-5):
        got, (b, e, ml) = O.progressive_step(cont, shape, dtype, mode, bound, t * scale, st, exact=True)
        one, (b1, e1, ml1) = O.progressive_step(cont, shape, dtype, mode, bound, t * scale, O.ProgressiveState())
        assert e == e1
        assert np.abs(got.astype(np.float64) - one).max() <= 16 * ulp, (t, np.abs(got.astype(np.float64) - one).max() / ulp)
