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
  l2_unscrubbed  the same launches back to back without the flush (a
            repeated launch finds much of its ~100 MB in L2; not the
            headline)
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
            its highest effort (dynamic Huffman blocks), every stream distinct;
            one page-batch launch
  serve     the served mixed-format stream: Poisson arrivals, each request
            1-4,096 chunks (log-uniform), 40 % LZ4 / 20 % Snappy / 30 % Zstd
            level 3 / 10 % GDeflate (one page each, so capped at 64 KiB),
            sizes lognormal (median 32 KiB, sigma 1.0, 512 B - 2 MiB), a
            32 GiB device budget, outputs kept on the device; p50 /
            p99 latency and aggregate GB/s of the continuous-batching server
            against the plain path (one request at a time, one launch per
            format), at the default rate and at the `--serve-sweep` rates
  per_format    the same measurement for raw Snappy (same content) and for
            Zstd: 4,096 frames of 1 MiB (1 MiB window, 128 KiB blocks, 10%
            repeated-byte runs, back-references up to 1 MiB), libzstd level 3
            and level 19 as two batches, every frame distinct (4 GiB of output
            per batch; L2 flushed)
  reference_gpu the reference library's own sm_100a LZ4 kernel on the same
            device batch, flush and events (a baseline leg)

Every leg checks every chunk: statuses and lengths, and the decoded bytes
against the generator's bytes (or their BLAKE2b digests, taken when the
input was generated); each leg reports `verified_chunks`.

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
    ap.add_argument("--serve-sweep", default="25,50,100",
                    help="further arrival rates (requests/s, comma-separated) replayed "
                         "for the latency sweep, below the saturating default rate")
    ap.add_argument("--gdeflate-streams", type=int, default=16384,
                    help="256 KiB TileStreams of the GDeflate leg (0 skips it)")
    ap.add_argument("--gdeflate-unique", type=int, default=0,
                    help="distinct TileStreams encoded for the GDeflate leg (0: all "
                         "of them; a smaller count is laid out repeatedly)")
    ap.add_argument("--zstd-frames", type=int, default=4096,
                    help="Zstd frames per batch (0 skips the Zstd legs)")
    ap.add_argument("--zstd-unique", type=int, default=0,
                    help="distinct Zstd frames compressed per level (0: all of them; "
                         "a smaller count is laid out repeatedly)")
    return ap.parse_args()


ZSTD_FRAME = 1 << 20


def digest(b):
    """16-byte BLAKE2b digest of a chunk's expected (or decoded) bytes."""
    import hashlib
    return hashlib.blake2b(b, digest_size=16).digest()


def _zstd_job(job):
    from cudec_b200 import workload as W
    seed, level = job
    buf, offs = W.generate([ZSTD_FRAME], [W.zstd_params(0.5, 0.1)],
                           seeds=np.array([seed], dtype=np.uint64))
    raw = buf[:ZSTD_FRAME].tobytes()
    return digest(raw), W.zstd_compress(raw, level, 20, False)


def start_generation(args):
    """Compress the Zstd frames (both levels) and encode the GDeflate
    TileStreams in spawned worker processes (no CUDA state is forked), all
    host cores, while the device legs run. Returns {name: AsyncResult}."""
    import multiprocessing as mp
    from cudec_b200 import workload as W
    jobs = {}
    if args.zstd_frames <= 0 and args.gdeflate_streams <= 0:
        return None, jobs
    pool = mp.get_context("spawn").Pool(min(os.cpu_count() or 1, 64))
    if args.gdeflate_streams > 0:
        jobs["gdeflate"] = pool.map_async(
            _gd_job, range(min(args.gdeflate_unique or args.gdeflate_streams,
                               args.gdeflate_streams)), chunksize=8)
    if args.zstd_frames > 0:
        unique = min(args.zstd_unique or args.zstd_frames, args.zstd_frames)
        for level in (19, 3):
            jobs["zstd_l%d" % level] = pool.map_async(
                _zstd_job, [(W.chunk_seed(CONFIG_SEED, 3, i), level) for i in range(unique)],
                chunksize=4)
    pool.close()
    return pool, jobs


def verify_outputs(batch, lengths, expect=None, digests=None, window=256 << 20):
    """Every chunk's decoded bytes against its expected bytes (`expect[k]`)
    or digest (`digests[k]`), copied back in windows of whole chunks. Returns
    the number of chunks verified (all of them, or an AssertionError)."""
    from concurrent.futures import ThreadPoolExecutor
    offs = batch.dst_offs
    n = len(lengths)
    i = done = 0
    with ThreadPoolExecutor(max_workers=min(os.cpu_count() or 1, 16)) as ex:
        while i < n:
            lo = int(offs[i])
            j = i + 1
            while j < n and int(offs[j]) + int(lengths[j]) - lo <= window:
                j += 1
            hi = int(offs[j - 1]) + int(lengths[j - 1])
            host = batch.d_dst[lo:hi].cpu().numpy()

            def check(k):
                o = int(offs[k]) - lo
                got = host[o:o + int(lengths[k])]
                if digests is not None:
                    return digest(got) == digests[k]
                e = expect[k]
                e = np.frombuffer(e, dtype=np.uint8) if isinstance(e, (bytes, bytearray)) else e
                return np.array_equal(got, e)

            ok = list(ex.map(check, range(i, j), chunksize=256))
            bad = [k for k, v in zip(range(i, j), ok) if not v]
            assert not bad, "chunk %d: decoded bytes differ from the expected output" % bad[0]
            done += j - i
            i = j
    return done


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


TRAFFIC_PROFILE = os.path.join("profiles", "lz4_cta_kernel_64KiBx1024.txt")


def traffic_per_launch():
    """(DRAM bytes, L2 write bytes, build) per headline launch from the
    committed ncu summary (Nones where absent)."""
    vals = {}
    try:
        for line in open(os.path.join(ROOT, TRAFFIC_PROFILE)):
            for key in ("dram_bytes_per_launch=", "l2_write_bytes_per_launch=", "build:"):
                if line.startswith(key):
                    vals[key] = line.split(key[-1], 1)[1].strip()
    except OSError:
        pass
    num = lambda k: int(vals[k].split()[0]) if k in vals else None
    return num("dram_bytes_per_launch="), num("l2_write_bytes_per_launch="), vals.get("build:")


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
    default_shape = plan.shape()  # compiled in: the same on every run
    with torch.cuda.stream(stream):
        assert allb.run_mixed(plan, fmts, stream) == 0
    stream.synchronize()
    res = allb.results()
    assert (res["status"] == 0).all() and (res["bytes_written"] == np.array(caps)).all()
    steps = max(args.steps // 50, 3)
    p_ms = max_over_ranks(time_region(torch, stream, flush, steps, warm,
                                      lambda: allb.run_mixed(plan, fmts, stream)))
    res = allb.results()
    assert (res["status"] == 0).all() and (res["bytes_written"] == np.array(caps)).all()
    verified = verify_outputs(allb, caps, expect=raws)
    # the autotuner's shape for this batch, measured the same way
    with torch.cuda.stream(stream):
        assert allb.run_mixed(plan, fmts, stream, tune=True) == 0
    tuned_shape = plan.shape()
    t_ms = max_over_ranks(time_region(torch, stream, flush, steps, warm,
                                      lambda: allb.run_mixed(plan, fmts, stream)))
    res = allb.results()
    assert (res["status"] == 0).all() and (res["bytes_written"] == np.array(caps)).all()
    assert verify_outputs(allb, caps, expect=raws) == n
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
        idx = [i for i, x in enumerate(fmts) if x == f]
        assert verify_outputs(b, [caps[i] for i in idx], expect=[raws[i] for i in idx]) == len(idx)
    del subs
    torch.cuda.empty_cache()
    sizes = np.array(caps)
    return {
        "value": round(world * out_bytes / (p_ms * 1e-3) / 1e9, 3), "unit": "GB/s",
        "ms_per_step": round(p_ms, 3),
        "plain_per_format_value": round(world * out_bytes / (q_ms * 1e-3) / 1e9, 3),
        "plain_per_format_ms": round(q_ms, 3),
        "chunks": n, "verified_chunks": verified,
        "decompressed_bytes": out_bytes, "compressed_bytes": in_bytes,
        "largest_chunk": int(sizes.max()), "median_chunk": int(np.median(sizes)),
        "roofline_frac": round((in_bytes + out_bytes) / (p_ms * 1e-3) / 1e9 / peaks()[0], 5),
        "shape_per_bucket": [list(t) for t in default_shape],
        "shape_source": "compiled-in default (warps per LZ4/Snappy chunk, then the one-warp "
                        "parse reach, lookahead, ring batch; buckets <4K,<16K,<64K,<256K,<1M,"
                        "larger)",
        "tuned": {"value": round(world * out_bytes / (t_ms * 1e-3) / 1e9, 3),
                  "ms_per_step": round(t_ms, 3),
                  "shape_per_bucket": [list(t) for t in tuned_shape]},
        "path": "cudec_mixed_decompress (graph: order + persistent work-stealing warp grid beside "
                "a CTA-per-chunk grid) vs "
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
    return [digest(raw[65536 * k:65536 * (k + 1)]) for k in range(4)], \
        W.gdeflate_tilestream(raw, 12, 32768)


def run_gdeflate(torch, cd, DeviceBatch, args, dev, stream, flush, max_over_ranks, world, warm,
                 made):
    """65,536 GDeflate pages (16,384 TileStreams x 4 tiles) in one launch."""
    unique = len(made)
    pages, digs = [], []
    for dg, ts in made:
        st, tiles, total = cd.tilestream_parse(ts, 4)
        assert st == 0 and total == 4 * 65536
        for k, (off, sz, dsz) in enumerate(tiles):
            assert dsz == 65536
            pages.append(ts[off:off + sz])
            digs.append(dg[k])
    n = 4 * args.gdeflate_streams
    comps = [pages[i % len(pages)] for i in range(n)]
    b = DeviceBatch(comps, [65536] * n, device=dev, poison=None)
    ms = max_over_ranks(time_device(torch, b, "gdeflate", stream, flush,
                                    max(args.steps // 50, 3), warm))
    res = b.results()
    assert (res["status"] == 0).all() and (res["bytes_written"] == 65536).all()
    verified = verify_outputs(b, [65536] * n, digests=[digs[i % len(digs)] for i in range(n)])
    out_bytes = 65536 * n
    in_bytes = b.src_bytes
    del b
    torch.cuda.empty_cache()
    return {"value": round(world * out_bytes / (ms * 1e-3) / 1e9, 3), "ms_per_step": round(ms, 3),
            "pages": n, "streams": args.gdeflate_streams, "unique_streams": unique,
            "verified_chunks": verified,
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
                         digests=[digest(r) for r in raws]))
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
    lats, t_end, outs = [], 0.0, []
    for i, r in enumerate(reqs):
        while tickets[i] is None:
            time.sleep(0.0002)
        st, recs, ptrs, lat = srv.wait(tickets[i])
        assert st == 0 and (recs["status"] == 0).all()
        assert (recs["bytes_written"] == np.array(r["caps"])).all()
        lats.append(lat)
        t_end = time.perf_counter()
        outs.append(ptrs)
    th.join()
    # every chunk of every request, read back from the arena after the
    # replay (outputs stay resident until released; the 32 GiB budget holds
    # the whole stream, so holding them changes no admission)
    verified = 0
    for i, r in enumerate(reqs):
        for k, cap in enumerate(r["caps"]):
            assert digest(read_device(int(outs[i][k]), cap)) == r["digests"][k], (i, k)
            verified += 1
        srv.release(tickets[i])
    srv.close()
    total = float(sum(sum(r["caps"]) for r in reqs))
    return {"verified_chunks": verified,
            "p50_ms": round(float(np.percentile(lats, 50)), 3),
            "p99_ms": round(float(np.percentile(lats, 99)), 3),
            "mean_ms": round(float(np.mean(lats)), 3),
            "value": round(total / (t_end - t0) / 1e9, 3),
            "unit": "GB/s", "submit_late_p99_ms": round(1e3 * float(np.percentile(late, 99)), 3)}


def run_serve(cd, args, dev):
    reqs = serve_requests(args.serve_requests)
    total = float(sum(sum(r["caps"]) for r in reqs))
    mixed = serve_once(cd, reqs, cd.SERVER_MIXED, SERVE_SLOTS, args.serve_rate)
    plain = serve_once(cd, reqs, cd.SERVER_PLAIN, 1, args.serve_rate)
    sweep = []
    for rate in [float(r) for r in args.serve_sweep.split(",") if r]:
        m = serve_once(cd, reqs, cd.SERVER_MIXED, SERVE_SLOTS, rate)
        q = serve_once(cd, reqs, cd.SERVER_PLAIN, 1, rate)
        sweep.append({"rate_per_s": rate,
                      "offered_GBps": round(total / len(reqs) * rate / 1e9, 3),
                      "continuous_batching": {k: m[k] for k in ("p50_ms", "p99_ms", "value")},
                      "plain_queue": {k: q[k] for k in ("p50_ms", "p99_ms", "value")}})
    return {"continuous_batching": mixed, "plain_queue": plain, "sweep": sweep,
            "requests": len(reqs), "rate_per_s": args.serve_rate,
            "chunks": int(sum(len(r["caps"]) for r in reqs)),
            "decompressed_bytes": int(total),
            "offered_GBps": round(total / len(reqs) * args.serve_rate / 1e9, 3),
            "budget_bytes": 32 << 30, "slots": SERVE_SLOTS,
            "formats": "40 % LZ4 / 20 % Snappy / 30 % Zstd L3 / 10 % GDeflate (pages <= 64 KiB)",
            "latency": "submit to completion, measured by the server"}


def run_reference_gpu(torch, batch, caps, raws, stream, flush, steps, warm, alg_bytes):
    """The reference library's own sm_100a LZ4 kernel (its src/batch.cu,
    compiled from its sources into oracle/_ref) on the same device batch,
    flush and events: the GPU kernel this library is measured against. A
    baseline leg outside the headline timed region."""
    import oracle
    ref = oracle.ref_gpu_lib()
    if ref is None:
        return {"unavailable": "reference library not built (oracle/_ref/libcudec_ref.so)"}

    def body():
        assert ref.cudec_lz4_decompress_batch(*batch.args(), stream.cuda_stream) == 0

    with torch.cuda.stream(stream):
        body()
    stream.synchronize()
    res = batch.results()
    assert (res["status"] == 0).all() and (res["bytes_written"] == np.array(caps)).all()
    verified = verify_outputs(batch, caps, expect=raws)
    ms = time_region(torch, stream, flush, steps, warm, body)
    out = float(sum(caps))
    return {"value": round(out / (ms * 1e-3) / 1e9, 3), "unit": "GB/s",
            "ms_per_step": round(ms, 5), "steps": steps, "verified_chunks": verified,
            "roofline_frac": round(alg_bytes / (ms * 1e-3) / 1e9 / peaks()[0], 5),
            "kernel": "reference lz4_decode_batch<false> (src/lz4_decode.cuh:29-173) "
                      "built for sm_100a, through its cudec_lz4_decompress_batch"}


def pyarrow_version():
    import pyarrow
    return pyarrow.__version__


def snappy_cpu(comps, caps, seconds, threads):
    """snappy's raw decompressor (bundled in pyarrow; it releases the GIL)
    over the batch from a thread pool, for ~`seconds`."""
    from concurrent.futures import ThreadPoolExecutor
    from cudec_b200 import workload as W
    codec = W.snappy_codec()

    def one(k):
        return codec.decompress(comps[k], decompressed_size=caps[k])

    with ThreadPoolExecutor(max_workers=threads) as ex:
        outs = list(ex.map(one, range(len(comps))))
        assert all(o.size == c for o, c in zip(outs, caps))
        reps, t0 = 0, time.perf_counter()
        while True:
            for _ in ex.map(one, range(len(comps)), chunksize=16):
                pass
            reps += 1
            el = time.perf_counter() - t0
            if el >= seconds:
                break
    return float(sum(caps)) * reps / el / 1e9, threads, reps


def time_device(torch, batch, fmt, stream, flush, steps, warmup):
    """Mean launch time (ms) of the batch entry, L2 flushed before each
    (flush None: back to back, the L2 left as the previous launch left it)."""
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            if flush is not None:
                flush.zero_()
            assert batch.run(fmt, stream) == 0
        for k in range(steps):
            if flush is not None:
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

    # Zstd / GDeflate inputs are compressed on all host cores while the
    # device legs below run (spawned workers, started before CUDA is used)
    gen_pool, gen_jobs = start_generation(args)

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
    verified = verify_outputs(batch, caps, expect=raws)

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
    res = batch.results()
    assert (res["status"] == 0).all() and (res["bytes_written"] == CHUNK).all()
    assert verify_outputs(batch, caps, expect=raws) == n
    # the same launches without the flush: input and output (~100 MB) fit in
    # the 126 MB L2, so a repeated launch finds much of them there
    warm_ms = max_over_ranks(time_device(torch, batch, "lz4", stream, None,
                                         max(args.steps // 2, 3), warm))
    assert (batch.results()["status"] == 0).all()

    # ---- the reference's own kernel on the same batch (a baseline leg) --
    ref_gpu = None
    if world == 1 and rank == 0:
        ref_gpu = run_reference_gpu(torch, batch, caps, raws, stream, flush,
                                    max(args.steps // 4, 3), warm, in_bytes + out_bytes)

    # ---- Snappy, same content -------------------------------------------
    _, scomps = workload(n, "snappy")
    sbatch = DeviceBatch(scomps, caps, device=dev, poison=None)
    s_ms = max_over_ranks(time_device(torch, sbatch, "snappy", stream, flush,
                                      max(args.steps // 4, 1), warm))
    sres = sbatch.results()
    assert (sres["status"] == 0).all() and (sres["bytes_written"] == CHUNK).all()
    s_verified = verify_outputs(sbatch, caps, expect=raws)
    s_in = sum(len(c) for c in scomps)
    del sbatch

    # ---- uneven mixed batch: persistent plan vs one launch per format ----
    mixed_line = None
    if args.mixed_chunks > 0:
        mixed_line = run_mixed(torch, cd, DeviceBatch, args, dev, stream, flush,
                               max_over_ranks, world, warm)

    # ---- served stream: continuous batching vs the plain queue --------
    serve_line = None
    if args.serve_requests > 0:
        serve_line = run_serve(cd, args, dev)

    # ---- GDeflate pages (TileStream tiles) ------------------------------
    gd_line = None
    if args.gdeflate_streams > 0:
        gd_line = run_gdeflate(torch, cd, DeviceBatch, args, dev, stream, flush,
                               max_over_ranks, world, warm, gen_jobs["gdeflate"].get())

    # ---- Zstd, 1 MiB frames at levels 3 and 19 ------------------------
    zstd_lines = {}
    zstd_sample = None
    if args.zstd_frames > 0:
        for level in (3, 19):
            made = gen_jobs["zstd_l%d" % level].get()
            zdig, zuniq = [m[0] for m in made], [m[1] for m in made]
            zn = args.zstd_frames
            zcomps = [zuniq[i % len(zuniq)] for i in range(zn)]
            if level == 3:
                zstd_sample = zuniq[:256]
            zbatch = DeviceBatch(zcomps, [ZSTD_FRAME] * zn, device=dev, poison=None)
            z_ms = max_over_ranks(time_device(torch, zbatch, "zstd", stream, flush,
                                              max(args.steps // 20, 3), warm))
            zres = zbatch.results()
            assert (zres["status"] == 0).all() and (zres["bytes_written"] == ZSTD_FRAME).all()
            zver = verify_outputs(zbatch, [ZSTD_FRAME] * zn,
                                  digests=[zdig[i % len(zdig)] for i in range(zn)])
            z_in = zbatch.src_bytes
            z_out = ZSTD_FRAME * zn
            zstd_lines["zstd_l%d" % level] = {
                "value": round(world * z_out / (z_ms * 1e-3) / 1e9, 3),
                "ms_per_step": round(z_ms, 4), "frames": zn, "unique_frames": len(zuniq),
                "verified_chunks": zver,
                "frame_bytes": ZSTD_FRAME, "compressed_bytes": z_in,
                "roofline_frac": round((z_in + z_out) / (z_ms * 1e-3) / 1e9 / peaks()[0], 5)}
            del zbatch
            torch.cuda.empty_cache()
    if gen_pool is not None:
        gen_pool.join()

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
        assert verify_outputs(batch, caps, expect=raws) == n
        return max_over_ranks(1e3 * sum(times) / len(times))

    e2e_staged_ms = e2e_ms_for(staged_ptrs_h)
    e2e_ms = e2e_ms_for(src_ptrs_h)

    # host output: the same call with every destination in pinned host
    # memory (the decoded bytes are copied back inside the call)
    host_out = torch.empty(out_bytes, dtype=torch.uint8).pin_memory()
    host_dst_h = (np.arange(n, dtype=np.uint64) * np.uint64(CHUNK) +
                  np.uint64(host_out.data_ptr())).astype(np.uint64)
    ctx = cd.StreamContext()
    ho_times = []
    for k in range(warm + args.steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        rc = ctx.decode(src_ptrs_h.ctypes.data, sizes_h.ctypes.data, host_dst_h.ctypes.data,
                        caps_h.ctypes.data, n, cd.MEM_HOST, res_h.ctypes.data)
        t1 = time.perf_counter()
        assert rc == 0 and (res_h["s"] == 0).all()
        if k >= warm:
            ho_times.append(t1 - t0)
    ctx.close()
    hnp = host_out.numpy()
    assert all(np.array_equal(hnp[CHUNK * i:CHUNK * (i + 1)], raws[i]) for i in range(n))
    ho_ms = max_over_ranks(1e3 * sum(ho_times) / len(ho_times))

    # the .lz4 frame entry, host to host: the whole batch's content as one
    # frame of independent 4 MiB blocks with block and content checksums
    from cudec_b200 import workload as W
    content = np.concatenate(raws).tobytes()
    frame = W.lz4f_compress(content, block_size_id=7, independent=True, content_checksum=True,
                            block_checksum=True)
    import ctypes
    f_src = np.frombuffer(frame, dtype=np.uint8).copy()
    f_out = np.empty(len(content), dtype=np.uint8)
    f_written = ctypes.c_size_t(0)
    f_times = []
    for k in range(warm + max(args.steps // 4, 3)):
        t0 = time.perf_counter()
        st = cd.lib().cudec_lz4f_decompress(f_src.ctypes.data, len(frame), f_out.ctypes.data,
                                            len(content), ctypes.byref(f_written))
        t1 = time.perf_counter()
        assert st == 0 and f_written.value == len(content)
        if k >= warm:
            f_times.append(t1 - t0)
    assert f_out.tobytes() == content
    f_ms = max_over_ranks(1e3 * sum(f_times) / len(f_times))
    e2e = world * out_bytes / (e2e_ms * 1e-3) / 1e9
    e2e_staged = world * out_bytes / (e2e_staged_ms * 1e-3) / 1e9

    peak, peak_kind = peaks()
    traffic = traffic_per_launch()
    achieved = (in_bytes + out_bytes) / (mean_ms * 1e-3) / 1e9
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(mean_ms, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8", "data": "synthetic",
            "config": {"workload": WORKLOAD % n, "format": "lz4", "chunks": n,
                       "chunk_bytes": CHUNK, "compressed_bytes": in_bytes,
                       "verified_chunks": verified,
                       "parallelism": "replicas x%d" % world,
                       "l2": "flushed before every timed launch (256 MiB memset)"},
            "l2_unscrubbed": {"value": round(world * out_bytes / (warm_ms * 1e-3) / 1e9, 3),
                              "unit": "GB/s", "ms_per_step": round(warm_ms, 5),
                              "l2": "launches back to back, no flush (not the headline)"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 5),
                         "traffic": traffic[0], "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": in_bytes + out_bytes,
                         "l2_write_bytes_per_launch": traffic[1],
                         "traffic_source": "%s (%s)" % (TRAFFIC_PROFILE, traffic[2])},
            "e2e": {"value": round(e2e, 3), "unit": "GB/s",
                    "h2d_bytes_per_step": int(in_bytes + 32 * n),
                    "d2h_bytes_per_step": 16 * n,
                    "api": "cudec_lz4_decompress_stream_ctx, pinned host chunks read in "
                           "place -> HBM, host clock around the synchronous call",
                    "ms_per_step": round(e2e_ms, 4),
                    "staged": {"value": round(e2e_staged, 3),
                               "ms_per_step": round(e2e_staged_ms, 4),
                               "source": "pageable host chunks, copied up by the call"},
                    "host_out": {"value": round(world * out_bytes / (ho_ms * 1e-3) / 1e9, 3),
                                 "ms_per_step": round(ho_ms, 4),
                                 "d2h_bytes_per_step": out_bytes,
                                 "dst": "pinned host memory, every decoded byte copied back "
                                        "inside the call"},
                    "frame": {"value": round(world * out_bytes / (f_ms * 1e-3) / 1e9, 3),
                              "ms_per_step": round(f_ms, 4),
                              "api": "cudec_lz4f_decompress, host frame -> host buffer",
                              "frame": "the batch's 64 MiB as one .lz4 frame: independent "
                                       "4 MiB blocks, block and content checksums (liblz4 "
                                       "LZ4F_compressFrame)",
                              "compressed_bytes": len(frame)}},
            "per_format": {
                "lz4": {"value": round(value, 3), "ms_per_step": round(mean_ms, 5)},
                "snappy": {"value": round(world * out_bytes / (s_ms * 1e-3) / 1e9, 3),
                           "ms_per_step": round(s_ms, 5), "verified_chunks": s_verified,
                           "roofline_frac": round((s_in + out_bytes) / (s_ms * 1e-3) / 1e9 / peak, 5)},
                **zstd_lines,
                **({"gdeflate": gd_line} if gd_line else {}),
            },
            **({"reference_gpu": ref_gpu} if ref_gpu else {}),
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
            csec = min(args.cpu_seconds, 5.0)
            cv, cused, _ = cpu_sample("codec_lz4", comps, caps, csec, threads)
            line["cpu_codec"] = {"value": round(cv, 3), "unit": "GB/s", "cores": cused,
                                 "library": "liblz4 %d LZ4_decompress_safe"
                                            % oracle.oracle_lib().codec_lz4_version()}
            # the same measurement for the other formats' codec libraries
            if oracle.ref_twin_lib() is not None:
                rv, rused, rreps = cpu_sample("ref_snappy", scomps, caps, csec, threads)
                line["per_format"]["snappy"]["cpu_baseline"] = {
                    "value": round(rv, 3), "unit": "GB/s", "cores": rused, "kind": "reference",
                    "sample": "%d passes over the %d x 64 KiB batch; reference twin "
                              "tests/snappy_twin.h on a std::thread pool" % (rreps, n)}
            sv, sused, sreps = snappy_cpu(scomps, caps, csec, threads)
            line["per_format"]["snappy"]["cpu_codec"] = {
                "value": round(sv, 3), "unit": "GB/s", "cores": sused,
                "library": "snappy (pyarrow %s) raw decompress, one call per chunk on a "
                           "thread pool" % pyarrow_version(),
                "sample": "%d passes over the %d x 64 KiB batch" % (sreps, n)}
            if zstd_sample:
                zv, zused, zreps = cpu_sample("codec_zstd", zstd_sample,
                                              [ZSTD_FRAME] * len(zstd_sample), csec, threads)
                line["per_format"]["zstd_l3"]["cpu_codec"] = {
                    "value": round(zv, 3), "unit": "GB/s", "cores": zused,
                    "library": "libzstd %d ZSTD_decompressDCtx, one DCtx per thread"
                               % oracle.oracle_lib().codec_zstd_version(),
                    "sample": "%d passes over %d of the level-3 1 MiB frames"
                              % (zreps, len(zstd_sample))}
        print(json.dumps(line), flush=True)
    replicas.finish()


if __name__ == "__main__":
    main()
