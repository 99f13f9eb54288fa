"""CPU tests of prism_lost_codes: the level-0 codes whose bits the reference's
last bit-plane shuffle block does not carry, counted from the dimensions
alone, against the oracle's restatement of that block (pinned to the
reference's own bytes): a round trip codes -> planes -> codes of a code array
with every magnitude bit set changes exactly that many level-0 codes and no
coarser one."""
import numpy as np
import pytest

import golden_util as gu
import oracle as O
import prism_b200 as P

SHAPES = [(48, 32, 64), (79, 44, 33), (194, 762, 1), (64, 40, 30), (100, 37, 1), (33, 56, 64), (17, 47, 64),
          (10, 116, 113), (97, 11, 22), (4, 14, 54), (1, 82, 27), (7293, 1, 1), (30113, 1, 1), (191, 83, 1),
          (242, 315, 1), (128, 128, 16), (5000, 1, 1)]


def oracle_lost(dims):
    nx, ny, nz = dims
    g = O.geometry(nx, ny, nz, 4)
    n, na = int(g.n), int(g.anchors)
    grid0 = ((nx + 1) // 2) * ((ny + 1) // 2) * ((nz + 1) // 2)
    lm0, c0 = int(g.lm_prefix[0]), n - grid0
    qc = np.zeros(n + na + 2 * 16384 + 64, dtype=np.int32)
    qc[na:lm0 + c0] = 0x7FFFFFFF  # level segments' pad slots included: harmless
    planes = O.bitshuffle(qc, g, 1, np.zeros(int(g.aligned_size) + (1 << 20), dtype=np.uint8))
    back = O.inverse_bitshuffle(planes, g, 1)
    coarse = int(np.count_nonzero(qc[na:lm0] != back[na:lm0]))
    return int(np.count_nonzero(qc[lm0:lm0 + c0] != back[lm0:lm0 + c0])), coarse


@pytest.mark.parametrize("dims", SHAPES)
def test_lost_codes_match_oracle(dims):
    lost, coarse = oracle_lost(dims)
    assert coarse == 0
    assert P.lost_codes(*dims) == lost


def test_reference_reconstruction_misses_the_bound_only_at_lost_codes():
    """The reference's own reconstruction of a short-last-block shape
    (79x44x33 float, REL 1e-3) misses the bound at some points, and at no
    more points than the lost codes."""
    name = "short_f32"
    c = gu.CASES[name]
    nx, ny, nz = c["dims"]
    lost = P.lost_codes(nx, ny, nz)
    assert lost > 0
    data = gu.field(name).astype(np.float64)
    # the oracle's decode of the reference's container is the reference's own
    # reconstruction (same SHA-256 as the reference's dec.bin)
    dec32 = O.decompress(gu.raw(name, "cmp.bin"), (nz, ny, nx), np.float32, 1, c["bound"])
    assert gu.sha(dec32) == gu.digests(name)["dec.bin"][1]
    dec = dec32.astype(np.float64)
    eb = float(gu.meta(name)["eb"][0][0])
    over = int(np.count_nonzero(np.abs(dec - data) > eb * (1 + 1e-6)))
    assert 0 < over <= lost


def test_benchmark_shapes_lose_nothing():
    assert P.lost_codes(384, 384, 256) == 0
    assert P.lost_codes(128, 128, 128) == 0
    assert P.lost_codes(1024, 1024, 1024) == 0
