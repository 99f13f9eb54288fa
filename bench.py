"""Benchmark of the PRISM hot path on B200 (one JSON line on rank 0).

Workload (one step): the progressive double-precision configuration -- a
256x384x384 float64 field (a[z][y][x], seeded k^-5/3 Gaussian random field
mapped to [0.9, 3.0], standing in for the README's Miranda density) is
compressed with negabinary planes at REL 1e-6 (`-prog`), then retrieved
progressively at REL 1e-2, 1e-3, 1e-4, 1e-5, 1e-6, each step refining the
previous reconstruction in place.

value = field bytes x (1 compression + 5 retrievals) / step time, all ranks
summed (weak scaling: every rank works on its own field -- replicas, there is
no data-path collective).  `e2e` is the same workflow through the C ABI with
host buffers and every host<->device copy inside the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl prism|reference]

--impl reference times the CPU restatement of the reference pipeline (the
reference has no CPU implementation of its own) with all host threads on a
bounded slab of the same field.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cmp/dec GB/s & %HBM peak at ref-equal CR; batched GB/s; p99 retrieval ms"
DIMS = (384, 384, 256)  # nx, ny, nz
TARGETS = [1e-2, 1e-3, 1e-4, 1e-5, 1e-6]
REL_EB = 1e-6
SAMPLE_Z = 64  # CPU baseline slab: the first 64 z-planes
L2_BYTES = 126 * 1024 * 1024


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            return float(json.load(open(p))["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None
        self.skip = 0

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # wait for the first sample so that the timed region is covered
        t0 = time.time()
        while time.time() - t0 < 3.0 and os.path.getsize(self.path) == 0:
            time.sleep(0.01)
        self.skip = sum(1 for _ in open(self.path))

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = open(self.path).read().splitlines()
        # samples taken before the timed region started are dropped, unless
        # the region was shorter than one sampling interval
        lines = lines[self.skip:] or lines[-1:]
        for line in lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_field(rank):
    from prism_b200 import fields
    nx, ny, nz = DIMS
    return fields.make("grf", (nz, ny, nx), np.float64, 1 + rank)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---------------------------------------------------------------- CPU arm
def cpu_sample_run(data_slab, steps):
    """Oracle (C, OpenMP over tiles and chunks) on the slab; returns seconds
    per workflow and the core count."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        cont, _, _ = O.compress(data_slab, 1, REL_EB, 0)
        st = O.ProgressiveState()
        for t in TARGETS:
            O.progressive_step(cont, data_slab.shape, np.float64, 1, REL_EB, t, st)
        times.append(time.perf_counter() - t0)
    return times, os.cpu_count()


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    data = make_field(0)[:SAMPLE_Z].copy()
    bytes_per = data.nbytes * (1 + len(TARGETS))
    cpu_sample_run(data, max(1, min(args.warmup, 1)))  # warm-up (page cache, thread pool)
    times, cores = cpu_sample_run(data, args.steps)
    per = sum(times) / len(times)
    value = bytes_per / per / 1e9
    sample = f"first {SAMPLE_Z} of 256 z-planes of the 384x384x256 field ({data.nbytes} B), full workflow"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "progressive f64 384x384x256 REL 1e-6 -prog, retrieval 1e-2..1e-6",
                   "sample": sample},
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU arm
STAGE_BYTES = None


def stage_algorithmic_bytes(n, tsize, aligned, cont_bytes, loaded_fraction):
    """Algorithmic HBM bytes per launch of each stage: what the stage must read
    and write at least (inputs once, outputs once)."""
    codes = 4 * n
    return {
        "extrema": n * tsize,
        "autotune": 0,
        "predict": n * tsize + codes,
        "shuffle": codes + aligned,
        "encode": aligned + cont_bytes,
        "trailer": 0,
        "strategy": 0,
        "decode": loaded_fraction * (cont_bytes + aligned),
        "inverse_shuffle": aligned + codes,
        "reconstruct": codes + 2 * n * tsize,
    }


def run_prism(args, world, rank, local):
    import torch
    import torch.distributed as dist
    import prism_b200 as P

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    nx, ny, nz = DIMS
    host = make_field(rank)
    n = host.size
    field_bytes = host.nbytes
    d_in = torch.from_numpy(host).cuda()
    ctx = P.Context(nx, ny, nz, np.dtype(np.float64), P.REL, REL_EB, True)
    h = P.Handle()
    comp = P.Compressor(ctx, h)
    d_cont = torch.empty(comp.max_container_size(), dtype=torch.uint8, device="cuda")
    values = torch.empty((nz, ny, nx), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    lib = P.lib()
    import ctypes as C

    def workflow():
        cont = comp.compress_pipeline(d_in, d_cont)
        ptr = C.c_void_p()
        st_ = C.c_void_p(stream.cuda_stream)
        h.check(lib.prism_progressive_open(h.ptr, C.c_void_p(cont.data_ptr()), cont.numel(), 8, nx, ny, nz,
                                           P.REL, REL_EB, C.byref(ptr)), "prism_progressive_open")
        for t in TARGETS:
            h.check(lib.prism_progressive_step(ptr, t, C.c_void_p(values.data_ptr()), st_), "prism_progressive_step")
        b, e, ml = (C.c_int * 4)(), (C.c_int * 4)(), C.c_int()
        lib.prism_progressive_state(ptr, b, e, C.byref(ml), None)
        lib.prism_progressive_close(ptr)
        return cont.numel(), (list(b), list(e), ml.value)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    # warm-up
    for _ in range(args.warmup):
        cont_bytes, _ = workflow()
    barrier()
    # ---- device-resident timed region ----
    h.profile(True)
    h.stage_times(reset=True)
    launches0 = h.launches()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        cont_bytes, state = workflow()
    ev1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    stage = h.stage_times(reset=True)
    launches = h.launches() - launches0
    h.profile(False)
    ms_t = torch.tensor([ms], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    bytes_step = field_bytes * (1 + len(TARGETS))
    value = bytes_step * args.steps * world / (ms_max / 1e3) / 1e9

    # ---- end-to-end through host buffers (C ABI, copies inside the region) ----
    h_in = torch.from_numpy(host).pin_memory()
    cap = comp.max_container_size()
    h_cont = torch.empty(cap, dtype=torch.uint8).pin_memory()
    h_vals = torch.empty((nz, ny, nx), dtype=torch.float64).pin_memory()
    d_cont2 = torch.empty(cap, dtype=torch.uint8, device="cuda")
    size = C.c_uint64()
    st = C.c_void_p(stream.cuda_stream)

    def e2e_workflow():
        h.check(lib.prism_compress_host(h.ptr, C.c_void_p(h_in.data_ptr()), 8, nx, ny, nz, P.REL, REL_EB, 1,
                                        C.c_void_p(h_cont.data_ptr()), cap, C.byref(size), st), "compress_host")
        csz = size.value
        d_cont2[:csz].copy_(h_cont[:csz], non_blocking=True)
        ptr = C.c_void_p()
        h.check(lib.prism_progressive_open(h.ptr, C.c_void_p(d_cont2.data_ptr()), csz, 8, nx, ny, nz, P.REL,
                                           REL_EB, C.byref(ptr)), "open")
        for t in TARGETS:
            h.check(lib.prism_progressive_step(ptr, t, C.c_void_p(values.data_ptr()), st), "step")
            h_vals.copy_(values, non_blocking=True)
        lib.prism_progressive_close(ptr)
        torch.cuda.current_stream().synchronize()
        return csz

    for _ in range(max(1, args.warmup)):
        csz = e2e_workflow()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        csz = e2e_workflow()
    e1.record(stream)
    barrier()
    e2e_ms = torch.tensor([e0.elapsed_time(e1)], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(e2e_ms, op=dist.ReduceOp.MAX)
    e2e_value = bytes_step * args.steps * world / (float(e2e_ms.item()) / 1e3) / 1e9

    # ---- roofline of the dominant stage ----
    peak, peak_kind = measured_peak()
    aligned = int(lib.prism_plane_buffer_size(nx, ny, nz))
    alg = stage_algorithmic_bytes(n, 8, aligned, cont_bytes, 1.0)
    dom = max((k for k in stage if stage[k][1] > 0), key=lambda k: stage[k][0])
    dom_ms, dom_n = stage[dom]
    achieved = alg[dom] * dom_n / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else 0.0
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": f"{peak_kind} copy bandwidth",
                "traffic": None, "bytes_per_launch": alg[dom], "launches": dom_n,
                "ms_per_launch": dom_ms / max(dom_n, 1)}
    stages = {k: {"ms_per_step": v[0] / args.steps, "launches_per_step": v[1] / args.steps,
                  "GBps": (alg[k] * v[1] / (v[0] / 1e3) / 1e9) if v[0] > 0 and alg[k] else None}
              for k, v in stage.items() if v[1] > 0}

    # ---- CPU baseline (rank 0, bounded slab of the same field) ----
    cpu = None
    if rank == 0 and not args.no_cpu:
        slab = host[:SAMPLE_Z].copy()
        cpu_sample_run(slab, 1)
        times, cores = cpu_sample_run(slab, 2)
        per = sum(times) / len(times)
        cpu = {"value": slab.nbytes * (1 + len(TARGETS)) / per / 1e9, "unit": "GB/s", "cores": cores,
               "kind": "port",
               "sample": f"first {SAMPLE_Z} z-planes ({slab.nbytes} B) of the field, full workflow, 2 runs"}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "progressive f64 384x384x256 (x,y,z) k^-5/3 GRF, compress REL 1e-6 -prog + "
                               "retrieval at REL 1e-2,1e-3,1e-4,1e-5,1e-6 refined in place",
                   "field_bytes": field_bytes, "container_bytes": cont_bytes,
                   "compression_ratio": field_bytes / cont_bytes,
                   "bytes_per_step": bytes_step, "l2": "inputs larger than L2 (302 MB field, 126 MB L2)",
                   "parallelism": f"replicas x{world}", "final_planes": state[1]},
        "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": field_bytes + csz,
                "d2h_bytes_per_step": csz + len(TARGETS) * field_bytes},
        "roofline": roofline, "stages": stages, "cpu_baseline": cpu, "gpu_launches": launches,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="prism", choices=["prism", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, world, rank)
    return run_prism(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
