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
  e2e       the same metric through the C ABI with host buffers:
            cudec_lz4_decompress_stream_ctx with the compressed chunks in
            pinned host memory and destinations in HBM (the decode kernel
            reads the chunks over the host link in place; table upload,
            decode and result readback inside the synchronous call);
            e2e.staged repeats it with the chunks in pageable memory, which
            the call copies to the device before decoding
  roofline  (compressed + decompressed bytes) per launch / launch time,
            against the measured HBM copy bandwidth
  cpu_baseline  the reference's own host decoder (its twin, compiled from
            its sources) on all host cores, same chunks
  mixed     the uneven mixed batch: 100,000 chunks, sizes lognormal (median
            16 KiB, sigma 1.2, clamped to 256 B - 4 MiB), copy probability
            uniform 0.2-0.8 per chunk, 5 % incompressible chunks, half LZ4 and
            half Snappy; the persistent work-stealing plan (tuned once, CUDA
            graph) against the plain path (one batch launch per format)
  gdeflate  4 GiB as 65,536 pages of 64 KiB in 16,384 TileStreams of
            256 KiB (content: 256-symbol Zipf(1.3) literals, matches 3-258,
            offsets up to 32 KiB), encoded by this library's GDeflate encoder at
            its highest effort (dynamic Huffman blocks); `--gdeflate-unique`
            distinct streams are encoded and laid out repeatedly, every page
            its own copy in HBM; one page-batch launch
  serve     the served mixed-format stream: Poisson arrivals, each request
            1-4,096 chunks (log-uniform), 40 % LZ4 / 20 % Snappy / 30 % Zstd
            level 3 / 10 % GDeflate (one page each, so capped at 64 KiB),
            sizes lognormal (median 32 KiB, sigma 1.0, 512 B - 2 MiB), a
            32 GiB device budget, outputs kept on the device; p50 /
            p99 latency and aggregate GB/s of the continuous-batching server
            against the plain path (one request at a time, one launch per
            format)
  per_format    the same measurement for raw Snappy (same content) and for
            Zstd: 4,096 frames of 1 MiB (1 MiB window, 128 KiB blocks, 10%
            repeated-byte runs, back-references up to 1 MiB), libzstd level 3
            and level 19 as two batches; `--zstd-unique` distinct frames are
            compressed and laid out repeatedly so the batch fills 4 GiB of
            output (every frame is its own copy in HBM; L2 flushed)

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
WORKLOAD = "lz4 block batch decode, %d x 64 KiB chunks"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="CPU-baseline sample length (0 skips the CPU leg)")
    ap.add_argument("--chunks", type=int, default=N_CHUNKS,
                    help="chunk count (the headline workload is 1024; smaller "
                         "counts are for profiler captures)")
    ap.add_argument("--mixed-chunks", type=int, default=100000,
                    help="chunks of the uneven mixed LZ4+Snappy batch (0 skips it)")
    ap.add_argument("--serve-requests", type=int, default=160,
                    help="requests of the served mixed-format stream (0 skips it)")
    ap.add_argument("--serve-rate", type=float, default=200.0,
                    help="Poisson arrival rate of the served stream (requests/s)")
    ap.add_argument("--gdeflate-streams", type=int, default=16384,
                    help="256 KiB TileStreams of the GDeflate leg (0 skips it)")
    ap.add_argument("--gdeflate-unique", type=int, default=512,
                    help="distinct TileStreams encoded for the GDeflate leg")
    ap.add_argument("--zstd-frames", type=int, default=4096,
                    help="Zstd frames per batch (0 skips the Zstd legs)")
    ap.add_argument("--zstd-unique", type=int, default=128,
                    help="distinct Zstd frames compressed per level")
    return ap.parse_args()


ZSTD_FRAME = 1 << 20


def _zstd_job(job):
    from cudec_b200 import workload as W
    seed, level = job
    buf, offs = W.generate([ZSTD_FRAME], [W.zstd_params(0.5, 0.1)],
                           seeds=np.array([seed], dtype=np.uint64))
    raw = buf[:ZSTD_FRAME].tobytes()
    return raw, W.zstd_compress(raw, level, 20, False)


def zstd_workload(unique, level):
    """`unique` distinct 1 MiB frames at `level`, compressed in worker
    processes (spawned, so no CUDA state is forked)."""
    import multiprocessing as mp
    from cudec_b200 import workload as W
    jobs = [(W.chunk_seed(CONFIG_SEED, 3, i), level) for i in range(unique)]
    with mp.get_context("spawn").Pool(min(os.cpu_count() or 1, 32)) as pool:
        out = pool.map(_zstd_job, jobs)
    return [o[0] for o in out], [o[1] for o in out]


def workload(n, fmt="lz4"):
    from cudec_b200 import workload as W
    seeds = np.array([W.chunk_seed(CONFIG_SEED, 1, i) for i in range(n)],
                     dtype=np.uint64)
    buf, offs = W.generate([CHUNK] * n, W.lz_params(0.5), seeds=seeds)
    raws = [buf[int(o):int(o) + CHUNK] for o in offs]
    comp = W.lz4_compress if fmt == "lz4" else W.snappy_compress
    return raws, [comp(r) for r in raws]


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_per_launch():
    """DRAM bytes per launch from the committed ncu summary, if any."""
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
    return float(sum(caps)) * reps / el / 1e9, used, reps


def run_reference(args, rank):
    """The reference's own CPU decoder (its host twin over its parser), on
    all host cores, same chunks and metric. Rank 0 only."""
    if rank != 0:
        return
    import oracle
    n = args.chunks
    _, comps = workload(n)
    caps = [CHUNK] * n
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
    value = float(sum(caps)) * len(times) / total / 1e9
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / len(times), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": WORKLOAD % n, "format": "lz4", "chunks": n,
                   "chunk_bytes": CHUNK, "l2": "host decode (no GPU)"},
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads,
                         "kind": "reference" if kind == "ref_lz4" else "port",
                         "sample": "whole batch per step: tests/lz4_twin.h over "
                                   "src/lz4_block.h on a std::thread pool"},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def time_region(torch, stream, flush, steps, warmup, body):
    """Mean device time (ms) of body() on `stream`, L2 flushed before each."""
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            flush.zero_()
            body()
        for k in range(steps):
            flush.zero_()
            starts[k].record(stream)
            body()
            ends[k].record(stream)
    stream.synchronize()
    return sum(s.elapsed_time(e) for s, e in zip(starts, ends)) / steps


MIXED_SEED = 0xC0DEC2


def run_mixed(torch, cd, DeviceBatch, args, dev, stream, flush, max_over_ranks, world, warm):
    """Uneven LZ4+Snappy batch: persistent tuned plan vs per-format launches."""
    from cudec_b200 import workload as W
    n = args.mixed_chunks
    raws, comps, fmts = W.mixed_batch(n, MIXED_SEED, formats=("lz4", "snappy"))
    caps = [len(r) for r in raws]
    out_bytes = int(sum(caps))
    in_bytes = int(sum(len(c) for c in comps))
    allb = DeviceBatch(comps, caps, device=dev, poison=None)
    plan = cd.MixedPlan()
    s = stream.cuda_stream
    with torch.cuda.stream(stream):
        assert allb.run_mixed(plan, fmts, stream, tune=True) == 0
    tuning = plan.tuning()
    res = allb.results()
    assert (res["status"] == 0).all() and (res["bytes_written"] == np.array(caps)).all()
    for i in range(0, n, max(n // 64, 1)):
        o = int(allb.dst_offs[i])
        assert allb.d_dst[o:o + caps[i]].cpu().numpy().tobytes() == raws[i].tobytes()
    steps = max(args.steps // 50, 3)
    p_ms = max_over_ranks(time_region(torch, stream, flush, steps, warm,
                                      lambda: allb.run_mixed(plan, fmts, stream)))
    res = allb.results()
    assert (res["status"] == 0).all()
    plan.close()
    del allb
    torch.cuda.empty_cache()
    subs = []
    for f in ("lz4", "snappy"):
        idx = [i for i, x in enumerate(fmts) if x == f]
        subs.append((f, DeviceBatch([comps[i] for i in idx], [caps[i] for i in idx],
                                    device=dev, poison=None)))

    def plain():
        for f, b in subs:
            assert b.run(f, stream) == 0

    q_ms = max_over_ranks(time_region(torch, stream, flush, steps, warm, plain))
    for f, b in subs:
        assert (b.results()["status"] == 0).all()
    del subs
    torch.cuda.empty_cache()
    sizes = np.array(caps)
    return {
        "value": round(world * out_bytes / (p_ms * 1e-3) / 1e9, 3), "unit": "GB/s",
        "ms_per_step": round(p_ms, 3),
        "plain_per_format_value": round(world * out_bytes / (q_ms * 1e-3) / 1e9, 3),
        "plain_per_format_ms": round(q_ms, 3),
        "chunks": n, "decompressed_bytes": out_bytes, "compressed_bytes": in_bytes,
        "largest_chunk": int(sizes.max()), "median_chunk": int(np.median(sizes)),
        "roofline_frac": round((in_bytes + out_bytes) / (p_ms * 1e-3) / 1e9 / peaks()[0], 5),
        "tuning_per_bucket": [list(t) for t in tuning],
        "path": "cudec_mixed_decompress (graph: order + persistent work-stealing kernel) vs "
                "cudec_lz4_decompress_batch + cudec_snappy_decompress_batch",
    }


GD_SEED = 0xC0DEC3


def _gd_job(i):
    from cudec_b200 import workload as W
    sizes = [65536] * 4
    buf, _ = W.generate(sizes, [W.gdeflate_params(0.5)],
                        seeds=np.array([W.chunk_seed(GD_SEED, 3, 4 * i + k) for k in range(4)],
                                       dtype=np.uint64))
    raw = buf.tobytes()
    return raw, W.gdeflate_tilestream(raw, 12, 32768)


def run_gdeflate(torch, cd, DeviceBatch, args, dev, stream, flush, max_over_ranks, world, warm):
    """65,536 GDeflate pages (16,384 TileStreams x 4 tiles) in one launch."""
    import multiprocessing as mp
    unique = min(args.gdeflate_unique, args.gdeflate_streams)
    with mp.get_context("spawn").Pool(min(os.cpu_count() or 1, 32)) as pool:
        made = pool.map(_gd_job, range(unique))
    pages, raws = [], []
    for raw, ts in made:
        st, tiles, total = cd.tilestream_parse(ts, 4)
        assert st == 0 and total == len(raw)
        for k, (off, sz, dsz) in enumerate(tiles):
            pages.append(ts[off:off + sz])
            raws.append(raw[65536 * k:65536 * k + dsz])
    n = 4 * args.gdeflate_streams
    comps = [pages[i % len(pages)] for i in range(n)]
    b = DeviceBatch(comps, [65536] * n, device=dev, poison=None)
    ms = max_over_ranks(time_device(torch, b, "gdeflate", stream, flush,
                                    max(args.steps // 50, 3), warm))
    res = b.results()
    assert (res["status"] == 0).all() and (res["bytes_written"] == 65536).all()
    for i in range(0, n, max(n // 32, 1)):
        o = int(b.dst_offs[i])
        assert b.d_dst[o:o + 65536].cpu().numpy().tobytes() == raws[i % len(raws)]
    out_bytes = 65536 * n
    in_bytes = b.src_bytes
    del b
    torch.cuda.empty_cache()
    return {"value": round(world * out_bytes / (ms * 1e-3) / 1e9, 3), "ms_per_step": round(ms, 3),
            "pages": n, "streams": args.gdeflate_streams, "unique_streams": unique,
            "compressed_bytes": in_bytes, "decompressed_bytes": out_bytes,
            "roofline_frac": round((in_bytes + out_bytes) / (ms * 1e-3) / 1e9 / peaks()[0], 5),
            "encoder": "this library's GDeflate encoder, level 12, 32 KiB window",
            "parity": "vs this library's CPU decoder; GDeflate reference decoder unpinned"}


SERVE_SEED = 0xC0DEC5
SERVE_SLOTS = 32


def serve_requests(k):
    """The served stream's requests (seeded): packed input + per-chunk arrays."""
    from cudec_b200 import workload as W
    rng = np.random.default_rng(SERVE_SEED)
    counts = np.rint(np.exp(rng.uniform(0, np.log(4096), k))).astype(int)
    reqs = []
    for i, n in enumerate(counts):
        raws, comps, fmts = W.mixed_batch(int(n), SERVE_SEED * 7919 + i,
                                          formats=("lz4", "snappy", "zstd", "gdeflate"),
                                          weights=(4, 2, 3, 1),
                                          median=32768, sigma=1.0, lo=512, hi=2 << 20)
        sizes = np.array([len(c) for c in comps], dtype=np.uint64)
        offs = np.zeros(len(sizes), dtype=np.uint64)
        offs[1:] = np.cumsum(sizes[:-1])
        packed = np.frombuffer(b"".join(bytes(c) for c in comps), dtype=np.uint8)
        import torch
        pinned = torch.empty(len(packed), dtype=torch.uint8).pin_memory()
        pinned.numpy()[:] = packed
        reqs.append(dict(packed=pinned.numpy(), pin=pinned, offs=offs, sizes=sizes,
                         caps=[len(r) for r in raws], fmts=fmts,
                         check=(raws[0].tobytes(), raws[-1].tobytes())))
    return reqs


def serve_once(cd, reqs, mode, slots, rate):
    """Replay the stream at `rate` requests/s into a fresh server."""
    import threading
    from cudec_b200.device import read_device
    srv = cd.Server(32 << 30, max_inflight=slots, mode=mode, max_chunks=4096)
    arrivals = np.cumsum(np.random.default_rng(SERVE_SEED + 1).exponential(1.0 / rate,
                                                                            len(reqs)))
    tickets = [None] * len(reqs)
    late = []
    t0 = time.perf_counter() + 0.05

    def submitter():
        for i, r in enumerate(reqs):
            wait = t0 + arrivals[i] - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            late.append(max(0.0, time.perf_counter() - (t0 + arrivals[i])))
            st, t = srv.submit(r["packed"], r["offs"], r["sizes"], r["caps"], r["fmts"])
            assert st == 0, st
            tickets[i] = t

    th = threading.Thread(target=submitter)
    th.start()
    lats, t_end = [], 0.0
    for i, r in enumerate(reqs):
        while tickets[i] is None:
            time.sleep(0.0002)
        st, recs, ptrs, lat = srv.wait(tickets[i])
        assert st == 0 and (recs["status"] == 0).all()
        assert read_device(int(ptrs[0]), r["caps"][0]) == r["check"][0]
        assert read_device(int(ptrs[-1]), r["caps"][-1]) == r["check"][1]
        lats.append(lat)
        t_end = time.perf_counter()
        srv.release(tickets[i])
    th.join()
    srv.close()
    total = float(sum(sum(r["caps"]) for r in reqs))
    return {"p50_ms": round(float(np.percentile(lats, 50)), 3),
            "p99_ms": round(float(np.percentile(lats, 99)), 3),
            "mean_ms": round(float(np.mean(lats)), 3),
            "value": round(total / (t_end - t0) / 1e9, 3),
            "unit": "GB/s", "submit_late_p99_ms": round(1e3 * float(np.percentile(late, 99)), 3)}


def run_serve(cd, args, dev):
    reqs = serve_requests(args.serve_requests)
    total = float(sum(sum(r["caps"]) for r in reqs))
    mixed = serve_once(cd, reqs, cd.SERVER_MIXED, SERVE_SLOTS, args.serve_rate)
    plain = serve_once(cd, reqs, cd.SERVER_PLAIN, 1, args.serve_rate)
    return {"continuous_batching": mixed, "plain_queue": plain,
            "requests": len(reqs), "rate_per_s": args.serve_rate,
            "chunks": int(sum(len(r["caps"]) for r in reqs)),
            "decompressed_bytes": int(total),
            "offered_GBps": round(total / len(reqs) * args.serve_rate / 1e9, 3),
            "budget_bytes": 32 << 30, "slots": SERVE_SLOTS,
            "formats": "40 % LZ4 / 20 % Snappy / 30 % Zstd L3 / 10 % GDeflate (pages <= 64 KiB)",
            "latency": "submit to completion, measured by the server"}


def time_device(torch, batch, fmt, stream, flush, steps, warmup):
    """Mean launch time (ms) of the batch entry, L2 flushed before each."""
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            flush.zero_()
            assert batch.run(fmt, stream) == 0
        for k in range(steps):
            flush.zero_()
            starts[k].record(stream)
            rc = batch.run(fmt, stream)
            ends[k].record(stream)
            assert rc == 0
    stream.synchronize()
    return sum(s.elapsed_time(e) for s, e in zip(starts, ends)) / steps


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

    from cudec_b200 import replicas
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    replicas.init("nccl", dev)
    cd.lib()
    n = args.chunks
    warm = max(args.warmup, 3)
    raws, comps = workload(n)
    caps = [CHUNK] * n
    in_bytes = sum(len(c) for c in comps)
    out_bytes = CHUNK * n
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
    for i in range(0, n, 97):
        assert batch.output(i, dst, CHUNK) == raws[i].tobytes()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, dev)

    barrier()
    with ClockSampler(local) as clocks:
        mean_ms = time_device(torch, batch, "lz4", stream, flush, args.steps, warm)
        barrier()
    mean_ms = max_over_ranks(mean_ms)
    value = world * out_bytes / (mean_ms * 1e-3) / 1e9

    # ---- Snappy, same content -------------------------------------------
    _, scomps = workload(n, "snappy")
    sbatch = DeviceBatch(scomps, caps, device=dev, poison=None)
    s_ms = max_over_ranks(time_device(torch, sbatch, "snappy", stream, flush,
                                      max(args.steps // 4, 1), warm))
    sres = sbatch.results()
    assert (sres["status"] == 0).all()
    s_in = sum(len(c) for c in scomps)
    del sbatch

    # ---- uneven mixed batch: persistent plan vs one launch per format ----
    mixed_line = None
    if args.mixed_chunks > 0:
        mixed_line = run_mixed(torch, cd, DeviceBatch, args, dev, stream, flush,
                               max_over_ranks, world, warm)

    # ---- GDeflate pages (TileStream tiles) ------------------------------
    gd_line = None
    if args.gdeflate_streams > 0:
        gd_line = run_gdeflate(torch, cd, DeviceBatch, args, dev, stream, flush,
                               max_over_ranks, world, warm)

    # ---- served stream: continuous batching vs the plain queue --------
    serve_line = None
    if args.serve_requests > 0:
        serve_line = run_serve(cd, args, dev)

    # ---- Zstd, 1 MiB frames at levels 3 and 19 ------------------------
    zstd_lines = {}
    if args.zstd_frames > 0:
        for level in (3, 19):
            zraws, zuniq = zstd_workload(min(args.zstd_unique, args.zstd_frames), level)
            zn = args.zstd_frames
            zcomps = [zuniq[i % len(zuniq)] for i in range(zn)]
            zbatch = DeviceBatch(zcomps, [ZSTD_FRAME] * zn, device=dev, poison=None)
            z_ms = max_over_ranks(time_device(torch, zbatch, "zstd", stream, flush,
                                              max(args.steps // 20, 3), warm))
            zres = zbatch.results()
            assert (zres["status"] == 0).all() and (zres["bytes_written"] == ZSTD_FRAME).all()
            zdst = zbatch.dst_host() if zn <= 1024 else None
            for i in range(0, zn, max(zn // 16, 1)):
                got = zbatch.output(i, zdst, ZSTD_FRAME) if zdst is not None else \
                    zbatch.d_dst[int(zbatch.dst_offs[i]):int(zbatch.dst_offs[i]) + ZSTD_FRAME].cpu().numpy().tobytes()
                assert got == zraws[i % len(zraws)]
            z_in = zbatch.src_bytes
            z_out = ZSTD_FRAME * zn
            zstd_lines["zstd_l%d" % level] = {
                "value": round(world * z_out / (z_ms * 1e-3) / 1e9, 3),
                "ms_per_step": round(z_ms, 4), "frames": zn, "unique_frames": len(zuniq),
                "frame_bytes": ZSTD_FRAME, "compressed_bytes": z_in,
                "roofline_frac": round((z_in + z_out) / (z_ms * 1e-3) / 1e9 / peaks()[0], 5)}
            del zbatch
            torch.cuda.empty_cache()

    # ---- end to end through the C ABI with host buffers ----------------
    # cudec_lz4_decompress_stream_ctx: compressed chunks in pinned host memory
    # (read in place by the kernel) or pageable memory (copied up by the
    # call), destinations in HBM; the synchronous call covers the transfer,
    # the decode and the 16-byte result readback, so it is timed with the
    # host clock around the call (L2 flushed before each).
    blob = b"".join(comps)
    pinned_src = torch.empty(len(blob), dtype=torch.uint8).pin_memory()
    pinned_src.numpy()[:] = np.frombuffer(blob, dtype=np.uint8)
    sizes_h = np.array([len(c) for c in comps], dtype=np.uint64)
    offs_h = np.zeros(n, dtype=np.uint64)
    offs_h[1:] = np.cumsum(sizes_h[:-1])
    src_ptrs_h = (offs_h + pinned_src.data_ptr()).astype(np.uint64)
    dst_ptrs_h = batch.d_dst_ptrs.cpu().numpy().astype(np.uint64)
    caps_h = np.array(caps, dtype=np.uint64)
    res_h = np.zeros(n, dtype=[("s", "<i4"), ("r", "<u4"), ("w", "<u8")])
    pageable_src = np.frombuffer(blob, dtype=np.uint8).copy()
    staged_ptrs_h = (offs_h + np.uint64(pageable_src.ctypes.data)).astype(np.uint64)

    def e2e_ms_for(ptrs):
        batch.d_dst.fill_(0)
        ctx = cd.StreamContext()
        times = []
        for k in range(warm + args.steps):
            flush.zero_()
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            rc = ctx.decode(ptrs.ctypes.data, sizes_h.ctypes.data, dst_ptrs_h.ctypes.data,
                            caps_h.ctypes.data, n, cd.MEM_DEVICE, res_h.ctypes.data)
            t1 = time.perf_counter()
            assert rc == 0 and (res_h["s"] == 0).all()
            if k >= warm:
                times.append(t1 - t0)
        ctx.close()
        dst = batch.dst_host()
        for i in range(0, n, 101):
            assert batch.output(i, dst, CHUNK) == raws[i].tobytes()
        return max_over_ranks(1e3 * sum(times) / len(times))

    e2e_staged_ms = e2e_ms_for(staged_ptrs_h)
    e2e_ms = e2e_ms_for(src_ptrs_h)
    e2e = world * out_bytes / (e2e_ms * 1e-3) / 1e9
    e2e_staged = world * out_bytes / (e2e_staged_ms * 1e-3) / 1e9

    peak, peak_kind = peaks()
    achieved = (in_bytes + out_bytes) / (mean_ms * 1e-3) / 1e9
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(mean_ms, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8", "data": "synthetic",
            "config": {"workload": WORKLOAD % n, "format": "lz4", "chunks": n,
                       "chunk_bytes": CHUNK, "compressed_bytes": in_bytes,
                       "parallelism": "replicas x%d" % world,
                       "l2": "flushed before every timed launch (256 MiB memset)"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 5),
                         "traffic": traffic_per_launch(), "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": in_bytes + out_bytes},
            "e2e": {"value": round(e2e, 3), "unit": "GB/s",
                    "h2d_bytes_per_step": int(in_bytes + 32 * n),
                    "d2h_bytes_per_step": 16 * n,
                    "api": "cudec_lz4_decompress_stream_ctx, pinned host chunks read in "
                           "place -> HBM, host clock around the synchronous call",
                    "ms_per_step": round(e2e_ms, 4),
                    "staged": {"value": round(e2e_staged, 3),
                               "ms_per_step": round(e2e_staged_ms, 4),
                               "source": "pageable host chunks, copied up by the call"}},
            "per_format": {
                "lz4": {"value": round(value, 3), "ms_per_step": round(mean_ms, 5)},
                "snappy": {"value": round(world * out_bytes / (s_ms * 1e-3) / 1e9, 3),
                           "ms_per_step": round(s_ms, 5),
                           "roofline_frac": round((s_in + out_bytes) / (s_ms * 1e-3) / 1e9 / peak, 5)},
                **zstd_lines,
                **({"gdeflate": gd_line} if gd_line else {}),
            },
            **({"mixed": mixed_line} if mixed_line else {}),
            **({"serve": serve_line} if serve_line else {}),
            "gpu_launches": args.steps,
            "clocks": clocks.summary(),
        }
        if world == 1 and args.cpu_seconds > 0:
            import oracle
            kind = "ref_lz4" if oracle.ref_twin_lib() is not None else "oracle_lz4"
            threads = os.cpu_count() or 1
            v, used, reps = cpu_sample(kind, comps, caps, args.cpu_seconds, threads)
            line["cpu_baseline"] = {
                "value": round(v, 3), "unit": "GB/s", "cores": used,
                "kind": "reference" if kind == "ref_lz4" else "port",
                "sample": "%d passes over the same %d x 64 KiB batch (~%.0f s); reference "
                          "twin tests/lz4_twin.h on a std::thread pool" % (reps, n, args.cpu_seconds)}
            cv, cused, _ = cpu_sample("codec_lz4", comps, caps, min(args.cpu_seconds, 5.0), threads)
            line["cpu_codec"] = {"value": round(cv, 3), "unit": "GB/s", "cores": cused,
                                 "library": "liblz4 %d LZ4_decompress_safe"
                                            % oracle.oracle_lib().codec_lz4_version()}
        print(json.dumps(line), flush=True)
    replicas.finish()


if __name__ == "__main__":
    main()
