"""Device-resident batches for the C-ABI batch entries.

A DeviceBatch packs a list of compressed chunks into one device buffer,
builds the five device tables the batch entries take (source pointers,
source sizes, destination pointers, capacities, 16-byte results), and gives
each chunk a destination slot. torch provides device memory and streams only;
the decode itself is the library's kernel.
"""
import numpy as np
import torch

import cudec_b200 as cd

RESULT_DTYPE = np.dtype([("status", "<i4"), ("reserved", "<u4"),
                         ("bytes_written", "<u8")])


def _ptr(t):
    return t.data_ptr()


class DeviceBatch:
    """Chunks + tables on one device.

    dst_align / dst_skew place every destination slot at an address that is
    dst_skew bytes past a dst_align-aligned boundary (to exercise unaligned
    outputs); poison fills destinations and `result_poison` the result
    records before each run, so a test can see exactly which bytes a decode
    touched.
    """

    def __init__(self, comps, caps, device="cuda", dst_align=256, dst_skew=0,
                 poison=0xA5, result_poison=0xFF, src_skew=0):
        self.n = len(comps)
        self.device = torch.device(device)
        self.caps = np.asarray(caps, dtype=np.uint64)
        sizes = np.array([len(c) for c in comps], dtype=np.uint64)
        self.src_sizes_h = sizes
        src_offs = np.zeros(self.n, dtype=np.uint64)
        if self.n > 1:
            src_offs[1:] = np.cumsum(sizes[:-1])
        src_offs += src_skew
        blob = b"\0" * src_skew + b"".join(comps)
        self.src_bytes = int(sizes.sum())
        host = torch.frombuffer(bytearray(blob + b"\0" * 16), dtype=torch.uint8)
        self.d_src = host.to(self.device)
        slot = ((self.caps + dst_align - 1) // dst_align) * dst_align + dst_align
        dst_offs = np.zeros(self.n, dtype=np.uint64)
        if self.n > 1:
            dst_offs[1:] = np.cumsum(slot[:-1])
        dst_offs += dst_skew
        self.dst_offs = dst_offs
        self.poison = poison
        self.result_poison = result_poison
        self.d_dst = torch.empty(int(slot.sum()) + dst_align + 16, dtype=torch.uint8,
                                 device=self.device)
        base_src, base_dst = _ptr(self.d_src), _ptr(self.d_dst)
        self.d_src_ptrs = torch.from_numpy((src_offs + base_src).astype(np.int64)).to(self.device)
        self.d_src_sizes = torch.from_numpy(sizes.astype(np.int64)).to(self.device)
        self.d_dst_ptrs = torch.from_numpy((dst_offs + base_dst).astype(np.int64)).to(self.device)
        self.d_caps = torch.from_numpy(self.caps.astype(np.int64)).to(self.device)
        self.d_results = torch.empty(self.n * 16, dtype=torch.uint8, device=self.device)
        self.reset()

    def reset(self):
        if self.poison is not None:
            self.d_dst.fill_(self.poison)
        self.d_results.fill_(self.result_poison)

    def args(self):
        return (_ptr(self.d_src_ptrs), _ptr(self.d_src_sizes), _ptr(self.d_dst_ptrs),
                _ptr(self.d_caps), self.n, _ptr(self.d_results))

    def run(self, fmt, stream=None):
        """Launch the format's batch entry on `stream` (torch stream or None =
        current stream). Returns the synchronous status."""
        s = (stream or torch.cuda.current_stream(self.device)).cuda_stream
        if fmt in ("zstd", "zstd_multi"):
            ws = self.workspace()
            fn = cd.zstd_decompress_batch if fmt == "zstd" else cd.zstd_decompress_batch_multi
            return fn(*self.args(), ws.data_ptr(), ws.numel(), s)
        return cd.BATCH_ENTRIES[fmt](*self.args(), s)

    def run_mixed(self, plan, formats, stream=None, tune=False):
        """Decode through a MixedPlan; `formats` = one format code per chunk."""
        s = (stream or torch.cuda.current_stream(self.device)).cuda_stream
        if getattr(self, "_fmt_codes", None) is None or len(self._fmt_codes_src) != self.n or \
                list(self._fmt_codes_src) != list(formats):
            self._fmt_codes_src = list(formats)
            self._fmt_codes = torch.tensor([cd.FORMAT_CODES.get(f, f) if isinstance(f, str) else f
                                            for f in formats], dtype=torch.uint8).to(self.device)
        fn = plan.tune if tune else plan.decode
        return fn(*self.args()[:4], self._fmt_codes.data_ptr(), self.n, _ptr(self.d_results), s)

    def workspace(self):
        """Device workspace for the Zstd entry (allocated once per batch)."""
        if getattr(self, "_ws", None) is None:
            self._ws = torch.empty(cd.zstd_workspace_bytes(self.n), dtype=torch.uint8,
                                   device=self.device)
        return self._ws

    def results(self):
        raw = self.d_results.cpu().numpy().tobytes()
        return np.frombuffer(raw, dtype=RESULT_DTYPE)

    def dst_host(self):
        return self.d_dst.cpu().numpy()

    def output(self, i, dst=None, length=None):
        dst = self.dst_host() if dst is None else dst
        o = int(self.dst_offs[i])
        n = int(self.caps[i]) if length is None else length
        return dst[o:o + n].tobytes()


class _DevView:
    """A raw device byte range, viewable by torch without a copy."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "|u1",
                                         "data": (int(ptr), False), "version": 3}


def read_device(ptr, n, device="cuda"):
    """Copy n bytes at device address ptr to host bytes."""
    if n == 0:
        return b""
    return torch.as_tensor(_DevView(ptr, n), device=device).cpu().numpy().tobytes()
