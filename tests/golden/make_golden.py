"""Generate the golden fixtures for the LZ4 and Snappy block parity tests.

Run where the reference tree is mounted, with CUDEC_REFERENCE naming it,
after oracle/_ref has been built (`make -f oracle/Makefile REF=<tree>`):

    CUDEC_REFERENCE=<tree> python tests/golden/make_golden.py

Sources of the vectors:
  * the reference's own fuzz seeds, fuzz/corpus/fuzz_lz4_block/* (framing:
    2-byte big-endian capacity, then the block; fuzz/fuzz_lz4_block.cpp:69-74)
    and fuzz/corpus/fuzz_snappy_block/* (the whole input is the stream,
    capacity 1<<22; fuzz/fuzz_snappy_block.cpp:41-47);
  * the hand-built hostile LZ4 shapes of tests/adversarial_blocks.h:22-101,
    rebuilt here from their description (extension runs, zero offset,
    offset past the output, self-referential matches).

Expected verdicts come from running the reference's own host twins
(tests/lz4_twin.h, tests/snappy_twin.h, compiled from its sources into
oracle/_ref/libref_twin.so) and are cross-checked against the codec libraries
(liblz4 LZ4_decompress_safe; snappy via pyarrow). The written JSON is what the
tests compare against; the tests never read the reference tree.
"""
import hashlib
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from cudec_b200 import workload  # noqa: E402

REF = os.environ.get("CUDEC_REFERENCE", "")
OUT = os.path.dirname(os.path.abspath(__file__))


def _record(name, fmt, data, cap, twin, codec_ok, codec_bytes):
    st, out = twin
    rec = {
        "name": name,
        "format": fmt,
        "input_hex": data.hex(),
        "capacity": cap,
        "expect_status": st,
        "expect_len": len(out) if st == 0 else 0,
        "expect_sha256": hashlib.sha256(out).hexdigest() if st == 0 else None,
        "codec_accepts": codec_ok,
    }
    if st == 0 and codec_ok:
        assert codec_bytes == out, name
    return rec


def lz4_vectors():
    vecs = []
    d = os.path.join(REF, "fuzz", "corpus", "fuzz_lz4_block")
    for f in sorted(os.listdir(d)):
        raw = open(os.path.join(d, f), "rb").read()
        cap = (raw[0] << 8) | raw[1]
        body = raw[2:2 + (1 << 14)]
        vecs.append(("seed/" + f, body, cap))

    def lit_ext_run(run):
        return bytes([0xF0]) + b"\xff" * run + b"\x00" + b"\x41" * 64

    def match_ext_run(run):
        return bytes([0x4F, 0x41, 0x42, 0x43, 0x44, 0x01, 0x00]) + b"\xff" * run + \
            b"\x00" + b"\x41" * 64

    mb = 1 << 20
    vecs += [
        ("adversarial/empty", b"", 64),
        ("adversarial/lone-zero-token", b"\x00", 64),
        ("adversarial/lone-max-token", b"\xff", 64),
        ("adversarial/all-ff-4096", b"\xff" * 4096, mb),
        ("adversarial/all-zero-4096", b"\x00" * 4096, mb),
        ("adversarial/literal-extension-run-1", lit_ext_run(1), mb),
        ("adversarial/literal-extension-run-4096", lit_ext_run(4096), mb),
        ("adversarial/match-extension-run-1", match_ext_run(1), mb),
        ("adversarial/match-extension-run-4096", match_ext_run(4096), mb),
        ("adversarial/zero-offset", bytes([0x40, 0x41, 0x42, 0x43, 0x44, 0, 0]) + b"\x41" * 64, mb),
        ("adversarial/offset-past-output", bytes([0x40, 0x41, 0x42, 0x43, 0x44, 0xFF, 0xFF]) + b"\x41" * 64, mb),
        ("adversarial/self-referential-rle", workload.lz4_compress(b"\x5a" * 65536), 65536),
        ("adversarial/self-referential-period-2",
         workload.lz4_compress(bytes((0x00, 0xFF)) * 32768), 65536),
        ("edge/capacity-zero-accepts-lone-zero", b"\x00", 0),
        ("edge/capacity-zero-rejects-lone-ten", b"\x10", 0),
    ]
    out = []
    for name, body, cap in vecs:
        twin = oracle.ref_lz4_decode(body, cap)
        got = workload.lz4_decompress_ref(body, cap) if body else None
        out.append(_record(name, "lz4", body, cap, twin, got is not None, got))
    return out


def snappy_vectors():
    out = []
    d = os.path.join(REF, "fuzz", "corpus", "fuzz_snappy_block")
    cap = 1 << 22
    for f in sorted(os.listdir(d)):
        body = open(os.path.join(d, f), "rb").read()[: 1 << 14]
        twin = oracle.ref_snappy_decode(body, cap)
        declared = _declared(body)
        got = workload.snappy_decompress_ref(body, declared) if declared is not None \
            and declared <= cap else None
        out.append(_record("seed/" + f, "snappy", body, cap, twin, got is not None, got))
    # The one deliberate strictness (src/snappy_block.h:345-358): a literal
    # whose length-1 is spelled 0xFFFFFFFF wraps to zero in snappy's 32-bit
    # arithmetic and is accepted there; refused here.
    body = bytes([0x00, 0xF0]) + b"\xff\xff\xff\xff"
    twin = oracle.ref_snappy_decode(body, cap)
    got = workload.snappy_decompress_ref(body, 0)
    out.append(_record("edge/literal-length-wrap", "snappy", body, cap, twin,
                       got is not None, None))
    return out


def zstd_vectors():
    """fuzz/corpus/fuzz_zstd_frame/* (the whole input is the frame,
    fuzz/fuzz_zstd_frame.cpp) decoded whole with capacity 1 MiB, plus small
    libzstd frames (levels 1/19, checksum on) kept as bytes so the vectors do
    not depend on the compressor version; verdicts from the reference's twin
    driver (tests/zstd_twin_driver.h)."""
    out = []
    d = os.path.join(REF, "fuzz", "corpus", "fuzz_zstd_frame")
    cap = 1 << 20
    for f in sorted(os.listdir(d)):
        body = open(os.path.join(d, f), "rb").read()[: 1 << 14]
        twin = oracle.ref_zstd_decode(body, cap)
        got = workload.zstd_decompress_ref(body, cap)
        out.append(_record("seed/" + f, "zstd", body, cap, twin, got is not None, got))
    import numpy as np
    buf, offs = workload.generate([3000, 20000], [workload.zstd_params(0.5, 0.1)],
                                  seeds=np.array([11, 12], dtype=np.uint64))
    for i, (o, n) in enumerate(zip(offs, [3000, 20000])):
        raw = buf[int(o):int(o) + n].tobytes()
        for lvl in (1, 19):
            body = workload.zstd_compress(raw, lvl, 20, True)
            twin = oracle.ref_zstd_decode(body, n)
            got = workload.zstd_decompress_ref(body, n)
            out.append(_record("libzstd/%d-L%d" % (n, lvl), "zstd", body, n, twin,
                               got is not None, got))
    return out


def tilestream_vectors():
    """fuzz/corpus/fuzz_gdeflate_tilestream/* (framing per
    fuzz/fuzz_gdeflate_tilestream.cpp: byte 0 selects the tile-array capacity
    - odd: the declared count minus byte0 >> 1, floored at 0 - and the rest is
    the stream); verdicts and tile tables from the reference's own walker
    (src/tilestream.h, compiled into oracle/_ref/libref_twin.so)."""
    out = []
    d = os.path.join(REF, "fuzz", "corpus", "fuzz_gdeflate_tilestream")
    for f in sorted(os.listdir(d)):
        raw = open(os.path.join(d, f), "rb").read()
        if not raw:
            continue
        sel, stream = raw[0], raw[1:1 + (1 << 13)]
        declared = stream[2] | (stream[3] << 8) if len(stream) >= 4 else 0
        cap = declared
        if sel & 1:
            cap = max(declared - (sel >> 1), 0)
        st, tiles, total = oracle.ref_tilestream_parse(stream, cap)
        out.append({"name": "seed/" + f, "input_hex": stream.hex(), "tiles_capacity": cap,
                    "expect_status": st, "expect_tiles": tiles, "expect_total": total})
    return out


def gdeflate_vectors():
    """Pages from this library's own encoder with their decoded digests. No
    GDeflate reference decoder or vector exists in the reference tree, so
    these pin this library's format decisions against later change; they are
    not parity with the GDeflate reference."""
    import numpy as np
    out = []
    sizes = [0, 1, 100, 4096, 65536, 65536]
    buf, offs = workload.generate(sizes, [workload.gdeflate_params(0.5)],
                                  seeds=np.arange(40, 40 + len(sizes), dtype=np.uint64))
    raws = [buf[int(o):int(o) + n].tobytes() for o, n in zip(offs, sizes)]
    raws += [bytes(range(256)) * 256, b"\x00" * 65536,
             bytes(np.random.default_rng(3).integers(0, 256, 3000, dtype=np.uint8))]
    for i, raw in enumerate(raws):
        for lvl in (1, 12):
            page = workload.gdeflate_compress(raw, lvl)
            st, dec = oracle.gdeflate_decode(page, len(raw))
            assert st == 0 and dec == raw
            out.append({"name": "page/%d-%d-L%d" % (i, len(raw), lvl), "input_hex": page.hex(),
                        "capacity": len(raw), "expect_status": 0, "expect_len": len(raw),
                        "expect_sha256": hashlib.sha256(raw).hexdigest()})
    return out


def _declared(body):
    v = 0
    for k in range(5):
        if k >= len(body):
            return None
        b = body[k]
        if k == 4 and b >= 16:
            return None
        v |= (b & 0x7F) << (7 * k)
        if not b & 0x80:
            return v
    return None


def main():
    if not REF or not os.path.isdir(os.path.join(REF, "fuzz")):
        sys.exit("CUDEC_REFERENCE must name the reference tree")
    if oracle.ref_twin_lib() is None:
        sys.exit("oracle/_ref/libref_twin.so missing: run make -f oracle/Makefile")
    for name, vecs in (("lz4_block.json", lz4_vectors()),
                       ("snappy_block.json", snappy_vectors()),
                       ("zstd_frame.json", zstd_vectors()),
                       ("tilestream.json", tilestream_vectors()),
                       ("gdeflate_page.json", gdeflate_vectors())):
        with open(os.path.join(OUT, name), "w") as f:
            json.dump({"generated_by": "tests/golden/make_golden.py",
                       "lz4_version": workload.lz4_version(),
                       "vectors": vecs}, f, indent=1)
        print(name, len(vecs), "vectors")


if __name__ == "__main__":
    main()
