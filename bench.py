#!/usr/bin/env python
"""Batch-decode benchmark: decompressed GB/s on B200 with its HBM roofline.

Workload (the headline configuration): 1,024 independent LZ4 blocks of
64 KiB each (64 MiB out, ~36 MB in), content from the seeded generator in
cudec_b200/csrc/workload.c (64-symbol Zipf(1.1) literal runs of mean 8,
copies of length 4-255 / mean 16 at offsets uniform in 1..min(pos, 65535),
copy probability 0.5), each block compressed with liblz4
LZ4_compress_default. The reference's corpora (Silesia, enwik8) are not
available; these synthetic chunks stand in for them.

A step is one cudec_lz4_decompress_batch launch over the whole batch with
inputs resident in HBM. The working set (~100 MB) would fit in the 126 MB
L2, so L2 is flushed (a 256 MiB memset) before every timed launch and only
the launch itself is bracketed by CUDA events on its stream.

  value     decompressed bytes / mean launch time (whole job: all ranks)
  e2e       the same metric through the C ABI with host buffers: each step
            copies the compressed chunks and the chunk tables host->device
            from pinned memory, decodes, and reads the 16-byte results back
  roofline  (compressed + decompressed bytes) per launch / launch time,
            against the measured HBM copy bandwidth
  cpu_baseline  the reference's own host decoder (its twin, compiled from
            its sources) on all host cores, same chunks

`--impl reference` times that reference CPU decoder alone, same metric.
Multi-GPU: replicas (chunks are independent; no exchange step).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIG_SEED = 0xC0DEC
N_CHUNKS = 1024
CHUNK = 65536
METRIC = "decompressed GB/s per format + % HBM roofline; serve p50/p99 latency"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="CPU-baseline sample length")
    return ap.parse_args()


def workload():
    from cudec_b200 import workload as W
    seeds = np.array([W.chunk_seed(CONFIG_SEED, 1, i) for i in range(N_CHUNKS)],
                     dtype=np.uint64)
    buf, offs = W.generate([CHUNK] * N_CHUNKS, W.lz_params(0.5), seeds=seeds)
    raws = [buf[int(o):int(o) + CHUNK] for o in offs]
    comps = [W.lz4_compress(r) for r in raws]
    return raws, comps


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_per_launch():
    """dram bytes per launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "lz4_batch_64KiBx1024.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch="):
                return int(line.split("=", 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sample(kind, comps, caps, seconds, threads):
    """Decode the whole batch repeatedly on host cores for ~`seconds`."""
    import oracle
    hb = oracle.HostBatch(comps, caps)
    oracle.decode_batch(kind, hb, threads)  # warm + verify
    assert (hb.status == 0).all(), kind
    reps, t0 = 0, time.perf_counter()
    while True:
        used = oracle.decode_batch(kind, hb, threads)
        reps += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    out = float(sum(caps)) * reps
    return out / el / 1e9, used, reps


def run_reference(args, rank):
    if rank != 0:
        return
    import oracle
    raws, comps = workload()
    caps = [CHUNK] * N_CHUNKS
    kind = "ref_lz4" if oracle.ref_twin_lib() is not None else "oracle_lz4"
    threads = os.cpu_count() or 1
    hb = oracle.HostBatch(comps, caps)
    for _ in range(args.warmup):
        oracle.decode_batch(kind, hb, threads)
    assert (hb.status == 0).all()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.decode_batch(kind, hb, threads)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    out_bytes = float(sum(caps))
    value = out_bytes * len(times) / total / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / len(times), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "lz4 block batch decode, 1024 x 64 KiB chunks (64 MiB out)",
                   "format": "lz4", "chunks": N_CHUNKS, "chunk_bytes": CHUNK,
                   "l2": "host decode (no GPU)"},
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads,
                         "kind": "reference" if kind == "ref_lz4" else "port",
                         "sample": "whole batch (64 MiB) per step, tests/lz4_twin.h over "
                                   "src/lz4_block.h on a std::thread pool"},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import torch.distributed as dist
    import cudec_b200 as cd
    from cudec_b200.device import DeviceBatch

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    cd.lib()

    raws, comps = workload()
    caps = [CHUNK] * N_CHUNKS
    in_bytes = sum(len(c) for c in comps)
    out_bytes = CHUNK * N_CHUNKS
    batch = DeviceBatch(comps, caps, device=dev, poison=None)
    stream = torch.cuda.Stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    # correctness gate before timing
    with torch.cuda.stream(stream):
        assert batch.run("lz4", stream) == 0
    stream.synchronize()
    res = batch.results()
    assert (res["status"] == 0).all() and (res["bytes_written"] == CHUNK).all()
    dst = batch.dst_host()
    for i in range(0, N_CHUNKS, 97):
        assert batch.output(i, dst, CHUNK) == raws[i].tobytes()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            for _ in range(max(args.warmup, 3)):
                flush.zero_()
                batch.run("lz4", stream)
            barrier()
            for k in range(args.steps):
                flush.zero_()
                starts[k].record(stream)
                rc = batch.run("lz4", stream)
                ends[k].record(stream)
                assert rc == 0
            barrier()
    kernel_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    mean_ms = sum(kernel_ms) / len(kernel_ms)
    if world > 1:
        t = torch.tensor([mean_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        mean_ms = float(t.item())
    value = world * out_bytes / (mean_ms * 1e-3) / 1e9

    # ---- end to end through the C ABI with host buffers ----------------
    pinned_src = torch.empty(batch.d_src.numel(), dtype=torch.uint8).pin_memory()
    pinned_src.copy_(batch.d_src.cpu())
    meta_dev = torch.cat([batch.d_src_ptrs, batch.d_src_sizes, batch.d_dst_ptrs, batch.d_caps])
    pinned_meta = meta_dev.cpu().pin_memory()
    meta_dev2 = torch.empty_like(meta_dev)
    n = N_CHUNKS
    pinned_res = torch.empty(16 * n, dtype=torch.uint8).pin_memory()
    e_starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e_ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        for k in range(max(args.warmup, 3) + args.steps):
            flush.zero_()
            if k >= max(args.warmup, 3):
                e_starts[k - max(args.warmup, 3)].record(stream)
            batch.d_src.copy_(pinned_src, non_blocking=True)
            meta_dev2.copy_(pinned_meta, non_blocking=True)
            p = meta_dev2.data_ptr()
            rc = cd.lz4_decompress_batch(p, p + 8 * n, p + 16 * n, p + 24 * n, n,
                                         batch.d_results.data_ptr(), stream.cuda_stream)
            pinned_res.copy_(batch.d_results, non_blocking=True)
            if k >= max(args.warmup, 3):
                e_ends[k - max(args.warmup, 3)].record(stream)
            assert rc == 0
    stream.synchronize()
    e2e_ms = sum(s.elapsed_time(e) for s, e in zip(e_starts, e_ends)) / args.steps
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    r2 = np.frombuffer(pinned_res.numpy().tobytes(), dtype=[("s", "<i4"), ("r", "<u4"), ("w", "<u8")])
    assert (r2["s"] == 0).all()
    e2e = world * out_bytes / (e2e_ms * 1e-3) / 1e9

    peak, peak_kind = peaks()
    achieved = (in_bytes + out_bytes) / (mean_ms * 1e-3) / 1e9
    line = None
    if rank == 0:
        cpu = {}
        if world == 1:
            import oracle
            kind = "ref_lz4" if oracle.ref_twin_lib() is not None else "oracle_lz4"
            threads = os.cpu_count() or 1
            v, used, reps = cpu_sample(kind, comps, caps, args.cpu_seconds, threads)
            cpu = {"value": round(v, 3), "unit": "GB/s", "cores": used,
                   "kind": "reference" if kind == "ref_lz4" else "port",
                   "sample": "%d passes over the same 1024 x 64 KiB batch (~%.0f s), "
                             "reference twin tests/lz4_twin.h on a std::thread pool"
                             % (reps, args.cpu_seconds)}
            cv, cused, creps = cpu_sample("codec_lz4", comps, caps, min(args.cpu_seconds, 5.0),
                                          threads)
            codec = {"value": round(cv, 3), "unit": "GB/s", "cores": cused,
                     "library": "liblz4 %d LZ4_decompress_safe" % oracle.oracle_lib().codec_lz4_version()}
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(mean_ms, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8", "data": "synthetic",
            "config": {"workload": "lz4 block batch decode, 1024 x 64 KiB chunks (64 MiB out)",
                       "format": "lz4", "chunks": N_CHUNKS, "chunk_bytes": CHUNK,
                       "compressed_bytes": in_bytes, "parallelism": "replicas x%d" % world,
                       "l2": "flushed before every timed launch (256 MiB memset)"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic_per_launch(), "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": in_bytes + out_bytes},
            "e2e": {"value": round(e2e, 3), "unit": "GB/s",
                    "h2d_bytes_per_step": int(batch.d_src.numel() + meta_dev.numel() * 8),
                    "d2h_bytes_per_step": 16 * n},
            "gpu_launches": args.steps,
            "clocks": clocks.summary(),
        }
        if cpu:
            line["cpu_baseline"] = cpu
            line["cpu_codec"] = codec
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
