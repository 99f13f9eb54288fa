"""The command-line flows on the GPU against the reference's own outputs.

Two binaries run the same command lines: this library's `prism` CLI, and the
reference's examples/prism.cpp compiled unchanged against this library's C++
headers (prism.hpp, compressor.hpp: prism::Compressor<T,E>, StatBuffer,
prism_context, parse_argv, initialize) and linked with it -- the check that a
reference caller recompiles unchanged.  The container and the decompressed
files must carry the reference build's SHA-256 digests."""
import hashlib
import os
import subprocess

import numpy as np
import pytest

import golden_util as gu

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINARIES = {"cli": os.path.join(ROOT, "prism_b200", "bin", "prism"),
            "reference_example": os.path.join(ROOT, "prism_b200", "bin", "prism_ref_example")}


def sha_file(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for blk in iter(lambda: f.read(1 << 22), b""):
            h.update(blk)
    return h.hexdigest()


def binary(kind):
    b = BINARIES[kind]
    if not os.path.exists(b):
        pytest.skip(f"{b} not built (the reference example needs the reference sources at build time)")
    return b


def run(cmd):
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    return p.stdout


@pytest.mark.parametrize("kind", ["cli", "reference_example"])
def test_progressive_flow_f64_384x384x256(kind, tmp_path):
    """-d -3 384 384 256 -R 1e-6 -prog -errors -5 1e-2 .. 1e-6 -z -x: the
    container and the final retrieval equal the reference's; with --report
    time,cr every step prints its statistics and retrieved bytes."""
    c = gu.CASES["c1"]
    nx, ny, nz = c["dims"]
    src = tmp_path / "c1.f64"
    gu.field("c1").tofile(src)
    cmd = [binary(kind), "-i", str(src), "-d", "-3", str(nx), str(ny), str(nz), "-R", repr(c["bound"]),
           "-prog", "-errors", "-%d" % len(c["targets"])] + [repr(t) for t in c["targets"]] + ["-z", "-x"]
    if kind == "reference_example":
        cmd += ["--report", "time,cr"]
    out = run(cmd)
    dg = gu.digests("c1")
    assert sha_file(str(src) + ".prisma") == dg["cmp.bin"][1]
    last = len(c["targets"]) - 1
    assert sha_file(str(src) + ".prisma.out") == dg[f"prog{last}.bin"][1]
    if kind == "reference_example":
        assert out.count("Total Retrieved size") == len(c["targets"])
        assert out.count("PSNR") == len(c["targets"])
        assert "compression ratio" in out


@pytest.mark.parametrize("kind", ["cli", "reference_example"])
@pytest.mark.parametrize("name", ["clean_f32", "clean_f64", "short_f32"])
def test_decompress_reference_container_files(kind, name, tmp_path):
    """-x on the reference's own container file writes the reference's
    reconstruction."""
    c = gu.CASES[name]
    nx, ny, nz = c["dims"]
    base = tmp_path / name
    (tmp_path / (name + ".prisma")).write_bytes(gu.raw(name, "cmp.bin"))
    mode = "-R" if c["mode"] == "R" else "-A"
    run([binary(kind), "-i", str(base), "-" + c["dtype"], "-3", str(nx), str(ny), str(nz), mode, repr(c["bound"]),
         "-x"])
    assert sha_file(str(base) + ".prisma.out") == gu.digests(name)["dec.bin"][1]


@pytest.mark.parametrize("kind", ["cli", "reference_example"])
def test_compress_file_matches_reference(kind, tmp_path):
    name = "short_f32"
    c = gu.CASES[name]
    nx, ny, nz = c["dims"]
    src = tmp_path / "f.f32"
    gu.field(name).tofile(src)
    run([binary(kind), "-i", str(src), "-f", "-3", str(nx), str(ny), str(nz), "-R", repr(c["bound"]), "-z"])
    assert sha_file(str(src) + ".prisma") == gu.digests(name)["cmp.bin"][1]


def test_extrema_minmax_matches_numpy():
    """prism_extrema_minmax (the two results of extrema_scan) on an odd-sized
    double array."""
    import ctypes as C
    import torch
    import prism_b200 as P
    h = P.Handle()
    a = np.random.default_rng(3).standard_normal(1_000_003)
    d = torch.from_numpy(a).cuda()
    mm = (C.c_double * 2)()
    h.check(P.lib().prism_extrema_minmax(h.ptr, C.c_void_p(d.data_ptr()), 8, a.size, mm,
                                         C.c_void_p(torch.cuda.current_stream().cuda_stream)), "minmax")
    assert (mm[0], mm[1]) == (float(a.min()), float(a.max()))
    h.close()
