"""Generate golden vectors by running the reference PRISM build on a GPU.

Test infrastructure only.  Needs the binaries that ``oracle/ref/Makefile``
builds from the reference sources into ``oracle/_ref/`` (``ref_harness``,
``prism`` and their compute_90-PTX twins), plus a CUDA GPU.  Inputs come from
the seeded generators in ``prism_b200.fields``, so only the reference's
outputs need storing.

For every case the harness dumps each pipeline stage (auto-tune error sums,
chosen interpolation flags, level-major quant codes, the predictor's linear
scratch, bit planes, the container, decoded planes/codes and reconstructions,
and each progressive step with its strategy result).  This script keeps small
buffers raw (gzip) and reduces large ones to SHA-256 digests, then writes

    <out>/<case>/meta.txt, errors.bin, cmp.bin.gz, *.bin.gz | digests.txt

``cases.json`` (next to this file) lists the cases.  Run:

    python tests/golden/make_golden.py --out <dir> [--big]

and copy the case folders into ``tests/golden/``.
"""
from __future__ import annotations

import argparse
import gzip
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from prism_b200 import fields  # noqa: E402

REF_DIR = os.path.join(ROOT, "oracle", "_ref")
KEEP_RAW_LIMIT = 4 << 20  # raw (gzip) copies of the listed buffers up to 4 MiB


def sha256_file(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for blk in iter(lambda: f.read(1 << 22), b""):
            h.update(blk)
    return h.hexdigest()


def run_case(case, out_root, harness, tmp, keep_all):
    name = case["name"]
    nx, ny, nz = case["dims"]
    dtype = np.float32 if case["dtype"] == "f" else np.float64
    data = fields.make(case["gen"], (nz, ny, nx), dtype, case["seed"])
    inp = os.path.join(tmp, name + ".raw")
    data.tofile(inp)
    odir = os.path.join(tmp, name)
    os.makedirs(odir, exist_ok=True)
    cmd = [harness, case["dtype"], str(nx), str(ny), str(nz), case["mode"], repr(case["bound"]),
           case["bt"], inp, odir] + [repr(t) for t in case.get("targets", [])]
    env = dict(os.environ)
    if case.get("small_dumps"):
        env["HARNESS_SMALL"] = "1"
    t0 = time.time()
    p = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=600)
    dt = time.time() - t0
    dest = os.path.join(out_root, name)
    os.makedirs(dest, exist_ok=True)
    with open(os.path.join(dest, "run.log"), "w") as f:
        f.write(" ".join(cmd) + "\n" + p.stdout + p.stderr + f"\nrc={p.returncode} seconds={dt:.2f}\n")
    if p.returncode != 0:
        print(f"[golden] {name}: harness rc={p.returncode}\n{p.stderr[-2000:]}", flush=True)
        return False
    digests = []
    for fn in sorted(os.listdir(odir)):
        src = os.path.join(odir, fn)
        if fn.endswith(".txt"):
            shutil.copy(src, os.path.join(dest, fn))
            continue
        size = os.path.getsize(src)
        digests.append(f"{fn} {size} {sha256_file(src)}")
        raw = case.get("raw", ["cmp.bin", "errors.bin"])
        if keep_all or (fn in raw and size <= KEEP_RAW_LIMIT):
            with open(src, "rb") as fi, gzip.open(os.path.join(dest, fn + ".gz"), "wb") as fo:
                shutil.copyfileobj(fi, fo)
        os.remove(src)
    with open(os.path.join(dest, "digests.txt"), "w") as f:
        f.write("\n".join(digests) + "\n")
    os.remove(inp)
    print(f"[golden] {name}: ok in {dt:.2f}s", flush=True)
    return True


def run_cli(case, out_root, prism, tmp, tag):
    """Run the unmodified reference CLI (timing + output digests)."""
    name = case["name"]
    nx, ny, nz = case["dims"]
    dtype = np.float32 if case["dtype"] == "f" else np.float64
    data = fields.make(case["gen"], (nz, ny, nx), dtype, case["seed"])
    inp = os.path.join(tmp, name + ".raw")
    data.tofile(inp)
    cmpf, decf = inp + ".prisma", inp + ".prisma.out"
    mode = "-A" if case["mode"] == "A" else "-R"
    cmd = [prism, "-i", inp, "-" + case["dtype"], "-3", str(nx), str(ny), str(nz), mode,
           repr(case["bound"]), "-z", cmpf, "-x", decf, "--report", "time,cr"]
    if case.get("targets"):
        cmd += ["-prog", "-errors", "-%d" % len(case["targets"])] + [repr(t) for t in case["targets"]]
    t0 = time.time()
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    dt = time.time() - t0
    dest = os.path.join(out_root, "cli_" + tag + "_" + name)
    os.makedirs(dest, exist_ok=True)
    lines = [" ".join(cmd), p.stdout[-20000:], p.stderr[-4000:], f"rc={p.returncode} wall={dt:.2f}s"]
    for fn in (cmpf, decf):
        if os.path.exists(fn):
            lines.append(f"{os.path.basename(fn)} {os.path.getsize(fn)} {sha256_file(fn)}")
            os.remove(fn)
    with open(os.path.join(dest, "cli.log"), "w") as f:
        f.write("\n".join(lines) + "\n")
    os.remove(inp)
    print(f"[golden] cli {tag} {name}: rc={p.returncode} {dt:.2f}s", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="output folder for the case dumps")
    ap.add_argument("--cases", default=os.path.join(HERE, "cases.json"))
    ap.add_argument("--only", default="")
    ap.add_argument("--big", action="store_true", help="also run the large configurations")
    ap.add_argument("--cli", action="store_true", help="also run the unmodified CLI")
    ap.add_argument("--jit", action="store_true", help="also run the compute_90-PTX build")
    args = ap.parse_args()
    with open(args.cases) as f:
        cases = json.load(f)
    os.makedirs(args.out, exist_ok=True)
    tmp = tempfile.mkdtemp(prefix="golden_")
    ok = True
    for case in cases:
        if args.only and case["name"] not in args.only.split(","):
            continue
        if case.get("big") and not args.big:
            continue
        ok &= run_case(case, args.out, os.path.join(REF_DIR, "ref_harness"), tmp, False)
        if args.jit and case.get("jit"):
            jc = dict(case, name=case["name"] + "_jit")
            ok &= run_case(jc, args.out, os.path.join(REF_DIR, "ref_harness_jit"), tmp, False)
        if args.cli and case.get("cli"):
            run_cli(case, args.out, os.path.join(REF_DIR, "prism"), tmp, "sass")
    shutil.rmtree(tmp, ignore_errors=True)
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
