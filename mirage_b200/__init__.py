"""mirage_b200: B200-native MirAge classification hot path (Python host mirror of the C ABI).

The compute path is the CUDA library libmirage_b200.so (include/mirage_b200.h); this module
only marshals buffers through ctypes. There is no CPU fallback: if the library is missing the
import of any entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmirage_b200.so")

READ_DTYPE = np.dtype([("highest", "<f4"), ("cand_off", "<u4"), ("n_fwd", "<u2"), ("n_rc", "<u2"),
                       ("strand", "u1"), ("reported", "u1"), ("n_top", "<u2")])
CAND_DTYPE = np.dtype([("ref", "<u4"), ("rel", "<f4"), ("score", "<f4"), ("pct", "<f4")])
assert READ_DTYPE.itemsize == 16 and CAND_DTYPE.itemsize == 16

MG_OK = 0
ERRORS = {-1: "MG_ERR_IO", -2: "MG_ERR_BADFMT", -3: "MG_ERR_OOM", -4: "MG_ERR_LIMIT", -5: "MG_ERR_CUDA",
          -6: "MG_ERR_BADINPUT", -7: "MG_ERR_TIMEOUT", -8: "MG_ERR_INVAL", -9: "MG_ERR_BUSY"}

EXPORTS = ["mg_open", "mg_open_image", "mg_close", "mg_index_get_info", "mg_inspect_image", "mg_eval_logf",
           "mg_set_timing", "mg_set_probe_slots", "mg_set_tuning", "mg_get_tuning", "mg_last_kernel_times", "mg_last_tier_counts", "mg_bucket_sizes", "mg_gather_bandwidth",
           "mg_build_image", "mg_build_image_device", "mg_parse_fasta_device", "mg_seqs_free", "mg_free",
           "mg_score_batch", "mg_classify", "mg_classify_device", "mg_classify_device_sync",
           "mg_score_candidates", "mg_score_candidates_noalloc", "mg_server_create", "mg_server_submit", "mg_server_submit_into", "mg_server_register_host",
           "mg_server_get_stats", "mg_server_poll",
           "mg_server_wait", "mg_server_destroy", "mg_strerror", "mg_last_error", "mg_logs_open", "mg_logs_write",
           "mg_logs_close", "mg_make_results_dir", "mg_index_reference"]


class MirageError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {ERRORS.get(code, code)} ({msg})")
        self.code = code


class _Batch(C.Structure):
    _fields_ = [("n_reads", C.c_uint64), ("offsets", C.c_void_p), ("bases", C.c_void_p)]


class _Seqs(C.Structure):
    _fields_ = [("n_seqs", C.c_uint64), ("offsets", C.POINTER(C.c_uint64)), ("bases", C.POINTER(C.c_uint8)),
                ("header_at", C.POINTER(C.c_uint64)), ("header_len", C.POINTER(C.c_uint32))]


class _Result(C.Structure):
    _fields_ = [("reads", C.c_void_p), ("cands", C.c_void_p), ("cand_cap", C.c_uint64), ("n_cands", C.c_uint64)]


class _Info(C.Structure):
    _fields_ = [("n_hashes", C.c_uint64), ("n_postings", C.c_uint64), ("n_refs", C.c_uint64),
                ("ref_bases", C.c_uint64), ("device_bytes", C.c_uint64), ("k", C.c_int32), ("word", C.c_int32),
                ("load_seconds", C.c_double), ("upload_seconds", C.c_double), ("probe_slots", C.c_int32)]


TUNING_FIELDS = ("dual_blocks_per_sm", "steal_chunk", "first_tier", "second_blocks_per_sm", "finish_blocks_per_sm",
                 "long_blocks_per_sm", "chunks", "weighted_chunks", "third_blocks_per_sm", "pack_bases")


class _Tuning(C.Structure):
    _fields_ = [(f, C.c_uint32) for f in TUNING_FIELDS]


class _ServerConfig(C.Structure):
    _fields_ = [("max_inflight_reads", C.c_uint32), ("max_requests", C.c_uint32), ("device_budget", C.c_uint64),
                ("step_slots", C.c_uint32)]


class _ServerStats(C.Structure):
    _fields_ = [("steps", C.c_uint64), ("reads", C.c_uint64), ("requests", C.c_uint64), ("ring_bytes", C.c_uint64),
                ("direct_bytes", C.c_uint64), ("submit_copy_s", C.c_double), ("launch_s", C.c_double),
                ("device_s", C.c_double), ("deliver_s", C.c_double), ("idle_s", C.c_double), ("step_s", C.c_double)]


_lib = None


def lib() -> C.CDLL:
    """Load the native library (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m mirage_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, u64, i32, f32p = C.c_void_p, C.c_uint64, C.c_int, C.POINTER(C.c_float)
        L.mg_open.argtypes = [C.c_char_p, i32, i32, C.POINTER(vp)]
        L.mg_open_image.argtypes = [vp, u64, i32, i32, C.POINTER(vp)]
        L.mg_close.argtypes = [vp]
        L.mg_close.restype = None
        L.mg_index_get_info.argtypes = [vp, C.POINTER(_Info)]
        L.mg_build_image.argtypes = [vp, vp, C.c_uint32, C.POINTER(C.c_char_p), vp, i32, i32,
                                     C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(u64)]
        L.mg_build_image_device.argtypes = [i32, vp, vp, C.c_uint32, C.POINTER(C.c_char_p), vp, i32, i32,
                                            C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(u64)]
        L.mg_parse_fasta_device.argtypes = [i32, vp, u64, i32, C.POINTER(_Seqs)]
        L.mg_seqs_free.argtypes = [C.POINTER(_Seqs)]
        L.mg_seqs_free.restype = None
        L.mg_free.argtypes = [vp]
        L.mg_free.restype = None
        L.mg_score_batch.argtypes = [vp, C.POINTER(_Batch), C.POINTER(_Result)]
        L.mg_classify.argtypes = [vp, C.POINTER(_Batch), C.POINTER(_Result)]
        L.mg_classify_device.argtypes = [vp, u64, vp, vp, vp, vp, u64, vp, vp]
        L.mg_classify_device_sync.argtypes = [vp, vp, C.POINTER(u64)]
        L.mg_score_candidates.argtypes = [vp, u64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.mg_score_candidates_noalloc.argtypes = [vp, u64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.mg_server_create.argtypes = [vp, C.POINTER(_ServerConfig), C.POINTER(vp)]
        L.mg_server_submit.argtypes = [vp, C.POINTER(_Batch), C.POINTER(u64)]
        L.mg_server_submit_into.argtypes = [vp, C.POINTER(_Batch), C.POINTER(_Result), C.POINTER(u64)]
        L.mg_server_register_host.argtypes = [vp, vp, u64]
        L.mg_server_get_stats.argtypes = [vp, C.POINTER(_ServerStats)]
        L.mg_server_poll.argtypes = [vp, u64, C.POINTER(_Result)]
        L.mg_server_wait.argtypes = [vp, u64, C.POINTER(_Result), C.c_uint32]
        L.mg_server_destroy.argtypes = [vp]
        L.mg_server_destroy.restype = None
        L.mg_set_timing.argtypes = [vp, i32]
        L.mg_set_probe_slots.argtypes = [vp, i32]
        L.mg_set_tuning.argtypes = [vp, C.POINTER(_Tuning)]
        L.mg_get_tuning.argtypes = [vp, C.POINTER(_Tuning), C.c_char_p, u64]
        L.mg_gather_bandwidth.argtypes = [i32, u64, C.POINTER(C.c_double)]
        L.mg_last_kernel_times.argtypes = [vp, vp]
        L.mg_last_tier_counts.argtypes = [vp, vp]
        L.mg_bucket_sizes.argtypes = [vp, vp, vp, u64]
        L.mg_inspect_image.argtypes = [vp, u64, i32, C.POINTER(_Info)]
        L.mg_eval_logf.argtypes = [vp, vp, vp, u64]
        L.mg_logs_open.argtypes = [C.c_char_p, i32, C.c_float, C.c_float, C.c_float, C.POINTER(vp)]
        L.mg_logs_write.argtypes = [vp, vp, vp, u64, vp, C.POINTER(C.c_char_p), C.POINTER(C.c_char_p), vp, i32]
        L.mg_logs_close.argtypes = [vp]
        L.mg_logs_close.restype = None
        L.mg_make_results_dir.argtypes = [C.c_char_p, C.c_char_p, u64]
        L.mg_index_reference.argtypes = [vp, C.c_uint32, C.POINTER(C.c_char_p), C.POINTER(C.c_int32),
                                         C.POINTER(C.c_uint32)]
        L.mg_strerror.argtypes = [i32]
        L.mg_strerror.restype = C.c_char_p
        L.mg_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def _check(rc: int, where: str) -> int:
    if rc < 0:
        raise MirageError(rc, where, (lib().mg_last_error() or b"").decode(errors="replace"))
    return rc


def _u8(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint8)


def _u64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint64)


def gather_bandwidth(device: int = 0, buffer_bytes: int = 1 << 30) -> float:
    """Measured random 32-byte-sector gather bandwidth of `device` in GB/s (mg_gather_bandwidth)."""
    out = C.c_double()
    _check(lib().mg_gather_bandwidth(device, buffer_bytes, C.byref(out)), "mg_gather_bandwidth")
    return out.value


def parse_fasta(text, device: int = 0, uppercase: bool = True):
    """Parse a FASTA text on `device` as the reference's loader does; returns (bases, offsets,
    headers) with the bases and offsets as numpy arrays and the header lines as bytes."""
    t = _u8(np.frombuffer(text, np.uint8) if isinstance(text, (bytes, bytearray)) else text)
    s = _Seqs()
    _check(lib().mg_parse_fasta_device(device, t.ctypes.data, len(t), 1 if uppercase else 0, C.byref(s)),
           "mg_parse_fasta_device")
    try:
        n = int(s.n_seqs)
        offs = np.ctypeslib.as_array(s.offsets, shape=(n + 1,)).copy()
        total = int(offs[-1])
        bases = np.ctypeslib.as_array(s.bases, shape=(total,)).copy() if total else np.zeros(0, np.uint8)
        heads = []
        if n:
            at = np.ctypeslib.as_array(s.header_at, shape=(n,))
            ln = np.ctypeslib.as_array(s.header_len, shape=(n,))
            tb = t.tobytes()
            heads = [tb[int(a):int(a) + int(b)] for a, b in zip(at, ln)]
        return bases, offs, heads
    finally:
        lib().mg_seqs_free(C.byref(s))


def build_image(bases, offsets, names, k: int = 31, word: int = 0, taxids=None, device: int | None = None) -> np.ndarray:
    """Build a .mhm image (the reference's index format) from references; on the host, or with
    GPU kernels on `device` (the same bytes)."""
    L = lib()
    bases, offsets = _u8(bases), _u64(offsets)
    n = len(offsets) - 1
    arr = (C.c_char_p * max(1, n))(*[(x if isinstance(x, bytes) else str(x).encode()) for x in names])
    tax = None if taxids is None else np.ascontiguousarray(taxids, dtype=np.int32)
    out = C.POINTER(C.c_uint8)()
    ln = C.c_uint64()
    if device is None:
        rc = L.mg_build_image(bases.ctypes.data, offsets.ctypes.data, n, arr, None if tax is None else tax.ctypes.data,
                              k, word, C.byref(out), C.byref(ln))
    else:
        rc = L.mg_build_image_device(device, bases.ctypes.data, offsets.ctypes.data, n, arr,
                                     None if tax is None else tax.ctypes.data, k, word, C.byref(out), C.byref(ln))
    _check(rc, "mg_build_image")
    try:
        return np.ctypeslib.as_array(out, shape=(ln.value,)).copy()
    finally:
        L.mg_free(C.cast(out, C.c_void_p))


def inspect_image(image, k: int = 31) -> dict:
    """Parse and validate a .mhm image on the host (no GPU); returns its counts."""
    img = _u8(image)
    inf = _Info()
    _check(lib().mg_inspect_image(img.ctypes.data, len(img), k, C.byref(inf)), "mg_inspect_image")
    return {f: getattr(inf, f) for f, _ in _Info._fields_}


def write_logs(out_dir: str, results: "Results", input_ids, input_headers, ref_headers, taxids,
               first_group_only: bool = True, thresholds=(0.4, 0.7, 1.0), high_precision: bool = True) -> None:
    """Append results to the reference-format logs in out_dir (created with their headers when
    this call opens them). Headers are bytes including '>'."""
    L = lib()
    h = C.c_void_p()
    _check(L.mg_logs_open(os.fspath(out_dir).encode(), 1 if high_precision else 0, thresholds[0], thresholds[1],
                          thresholds[2], C.byref(h)), "mg_logs_open")
    try:
        n = len(results.reads)
        ids = np.ascontiguousarray(input_ids, dtype=np.uint64)
        ih = (C.c_char_p * max(1, n))(*input_headers)
        rh = (C.c_char_p * max(1, len(ref_headers)))(*ref_headers)
        tx = np.ascontiguousarray(taxids, dtype=np.int32)
        reads = np.ascontiguousarray(results.reads)
        cands = np.ascontiguousarray(results.cands) if len(results.cands) else np.zeros(1, CAND_DTYPE)
        _check(L.mg_logs_write(h, reads.ctypes.data, cands.ctypes.data, n, ids.ctypes.data, ih, rh, tx.ctypes.data,
                               1 if first_group_only else 0), "mg_logs_write")
    finally:
        L.mg_logs_close(h)


class Results:
    """Per-read results (READ_DTYPE) and the scored candidates (CAND_DTYPE), as the C ABI
    returns them."""

    def __init__(self, reads: np.ndarray, cands: np.ndarray):
        self.reads = reads
        self.cands = cands

    def strand_cands(self, i: int, strand: int) -> np.ndarray:
        r = self.reads[i]
        o = int(r["cand_off"])
        if strand == 0:
            return self.cands[o : o + int(r["n_fwd"])]
        return self.cands[o + int(r["n_fwd"]) : o + int(r["n_fwd"]) + int(r["n_rc"])]

    def top(self, i: int) -> list[int]:
        """Top-scoring reference group of read i (ascending refID)."""
        r = self.reads[i]
        if not r["reported"]:
            return []
        c = self.strand_cands(i, int(r["strand"]))
        return sorted(int(x["ref"]) for x in c if x["rel"] == r["highest"])


class Index:
    """An HBM-resident MirAge index (one .mhm file)."""

    def __init__(self, source, k: int = 31, device: int = 0):
        L = lib()
        h = C.c_void_p()
        if isinstance(source, (str, os.PathLike)):
            _check(L.mg_open(os.fspath(source).encode(), k, device, C.byref(h)), "mg_open")
        else:
            img = _u8(source)
            _check(L.mg_open_image(img.ctypes.data, len(img), k, device, C.byref(h)), "mg_open_image")
        self.h = h
        self.k = k

    def close(self):
        if getattr(self, "h", None):
            lib().mg_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        inf = _Info()
        _check(lib().mg_index_get_info(self.h, C.byref(inf)), "mg_index_get_info")
        return {f: getattr(inf, f) for f, _ in _Info._fields_}

    def _run(self, fn, name, bases, offsets, cand_cap=None):
        bases, offsets = _u8(bases), _u64(offsets)
        n = len(offsets) - 1
        cap = cand_cap if cand_cap is not None else max(1024, 8 * n)
        reads = np.zeros(n, dtype=READ_DTYPE)
        cands = np.zeros(cap, dtype=CAND_DTYPE)
        b = _Batch(n, offsets.ctypes.data, bases.ctypes.data)
        r = _Result(reads.ctypes.data, cands.ctypes.data, cap, 0)
        rc = fn(self.h, C.byref(b), C.byref(r))
        if rc == -3 and r.n_cands > cap and cand_cap is None:
            return self._run(fn, name, bases, offsets, int(r.n_cands))
        _check(rc, name)
        return Results(reads, cands[: r.n_cands].copy())

    def classify(self, bases, offsets, form: str = "batched", cand_cap: int | None = None) -> Results:
        """Classify a batch of reads (raw FASTA bytes, CSR offsets). form: 'batched' (fused
        persistent kernel) or 'plain' (one block per read)."""
        L = lib()
        fn = L.mg_classify if form == "batched" else L.mg_score_batch
        return self._run(fn, "mg_classify" if form == "batched" else "mg_score_batch", bases, offsets, cand_cap)

    def set_probe_slots(self, on: bool = True) -> None:
        """Build (or drop) the hash-slot table the dual-strand tiers probe (mg_set_probe_slots)."""
        _check(lib().mg_set_probe_slots(self.h, 1 if on else 0), "mg_set_probe_slots")

    def set_tuning(self, **fields) -> None:
        """Launch shapes (mg_set_tuning); unnamed fields (and zeros) keep the defaults."""
        t = _Tuning(*[int(fields.get(f, 0)) for f in TUNING_FIELDS])
        _check(lib().mg_set_tuning(self.h, C.byref(t)), "mg_set_tuning")

    def get_tuning(self) -> tuple[dict, str]:
        """The launch shapes in effect and the index's density class (mg_get_tuning)."""
        t = _Tuning()
        cls = C.create_string_buffer(32)
        _check(lib().mg_get_tuning(self.h, C.byref(t), cls, 32), "mg_get_tuning")
        return {f: int(getattr(t, f)) for f in TUNING_FIELDS}, cls.value.decode()

    def set_timing(self, on: bool = True) -> None:
        _check(lib().mg_set_timing(self.h, 1 if on else 0), "mg_set_timing")

    def last_kernel_times(self) -> np.ndarray:
        """Device ms of the last call: [dual-strand warp tier or plain kernel, general warp tier,
        block tier, global tier, output compaction]."""
        ms = np.zeros(5, np.float32)
        _check(lib().mg_last_kernel_times(self.h, ms.ctypes.data), "mg_last_kernel_times")
        return ms

    def last_tier_counts(self) -> dict:
        """Reads each tier of the last one-piece batched call handed on (mg_last_tier_counts)."""
        c = np.zeros(7, np.uint32)
        _check(lib().mg_last_tier_counts(self.h, c.ctypes.data), "mg_last_tier_counts")
        names = ["dual64", "dual128", "dual256", "warp", "long_small", "long_large", "block"]
        return {n: int(v) for n, v in zip(names, c)}

    def bucket_sizes(self, hashes) -> np.ndarray:
        h = np.ascontiguousarray(hashes, dtype=np.uint32)
        out = np.empty_like(h)
        _check(lib().mg_bucket_sizes(self.h, h.ctypes.data, out.ctypes.data, len(h)), "mg_bucket_sizes")
        return out

    def classify_ptrs(self, n: int, offs_ptr: int, bases_ptr: int, reads_ptr: int, cands_ptr: int,
                      cand_cap: int, form: str = "batched") -> int:
        """Classify with caller-provided host pointers (e.g. pinned buffers); returns the number
        of candidates written."""
        L = lib()
        fn = L.mg_classify if form == "batched" else L.mg_score_batch
        b = _Batch(n, offs_ptr, bases_ptr)
        r = _Result(reads_ptr, cands_ptr, cand_cap, 0)
        _check(fn(self.h, C.byref(b), C.byref(r)), "mg_classify")
        return int(r.n_cands)

    def classify_device(self, n: int, d_offs: int, d_bases: int, d_reads: int, d_cands: int, cand_cap: int,
                        d_n_cands: int, stream: int = 0) -> None:
        """Queue the batched form on device buffers (no host copies) on `stream`."""
        _check(lib().mg_classify_device(self.h, n, d_offs, d_bases, d_reads, d_cands, cand_cap, d_n_cands,
                                        stream or None), "mg_classify_device")

    def device_sync(self, stream: int = 0) -> int:
        n = C.c_uint64()
        _check(lib().mg_classify_device_sync(self.h, stream or None, C.byref(n)), "mg_classify_device_sync")
        return int(n.value)

    def eval_logf(self, x) -> np.ndarray:
        """The device logarithm of the relative score at the points x (float32)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.empty_like(x)
        _check(lib().mg_eval_logf(self.h, x.ctypes.data, out.ctypes.data, len(x)), "mg_eval_logf")
        return out

    def score_candidates(self, q_off, bases, c_off, cand_ref, r_off, runs):
        """Scoring-only drop-in: Score, percentageMatch, relative score per candidate and
        HighestScore per strand, for candidate lists and runs produced elsewhere."""
        q_off, bases, c_off, r_off = _u64(q_off), _u8(bases), _u64(c_off), _u64(r_off)
        cand_ref = np.ascontiguousarray(cand_ref, dtype=np.uint32)
        runs = np.ascontiguousarray(runs, dtype=np.uint32)
        ns = len(q_off) - 1
        nc = int(c_off[-1])
        score = np.zeros(nc, np.float32)
        pct = np.zeros(nc, np.float32)
        rel = np.zeros(nc, np.float32)
        hi = np.zeros(ns, np.float32)
        _check(lib().mg_score_candidates(self.h, ns, q_off.ctypes.data, bases.ctypes.data, c_off.ctypes.data,
                                         cand_ref.ctypes.data, r_off.ctypes.data, runs.ctypes.data,
                                         score.ctypes.data, pct.ctypes.data, rel.ctypes.data, hi.ctypes.data),
               "mg_score_candidates")
        return score, pct, rel, hi


class Server:
    """Served form: continuous batching of requests against a resident index."""

    def __init__(self, index: Index, max_inflight_reads: int = 0, max_requests: int = 0, device_budget: int = 0,
                 step_slots: int = 0):
        self.index = index
        cfg = _ServerConfig(max_inflight_reads, max_requests, device_budget, step_slots)
        h = C.c_void_p()
        _check(lib().mg_server_create(index.h, C.byref(cfg), C.byref(h)), "mg_server_create")
        self.h = h
        self._pending: dict[int, int] = {}
        self._into: dict[int, tuple] = {}  # ticket -> (reads, cands, result struct) of submit_into
        self._registered: list = []  # arrays page-locked by register_host (kept alive with the server)

    def register_host(self, array) -> None:
        """Page-lock a host array for the server (mg_server_register_host): requests whose bases
        lie in it are copied to the device from it, without the copy into the request ring. The
        array must stay unchanged while such requests are outstanding."""
        a = np.ascontiguousarray(array)
        if a is not array and isinstance(array, np.ndarray):
            raise ValueError("register_host needs a contiguous array")
        _check(lib().mg_server_register_host(self.h, a.ctypes.data, a.nbytes), "mg_server_register_host")
        self._registered.append(a)

    def stats(self) -> dict:
        """Counters and the server thread's time per phase since creation (mg_server_get_stats)."""
        st = _ServerStats()
        _check(lib().mg_server_get_stats(self.h, C.byref(st)), "mg_server_get_stats")
        return {f: getattr(st, f) for f, _ in _ServerStats._fields_}

    def submit(self, bases, offsets) -> int | None:
        """Submit a request; returns its ticket, or None when it cannot be admitted now."""
        bases, offsets = _u8(bases), _u64(offsets)
        n = len(offsets) - 1
        b = _Batch(n, offsets.ctypes.data, bases.ctypes.data)
        t = C.c_uint64()
        rc = lib().mg_server_submit(self.h, C.byref(b), C.byref(t))
        if rc == -9:
            return None
        _check(rc, "mg_server_submit")
        self._pending[t.value] = n
        return t.value

    def submit_into(self, bases, offsets, cand_cap: int | None = None) -> int | None:
        """Submit a request whose results the server writes straight into buffers made here
        (mg_server_submit_into); returns its ticket, or None when it cannot be admitted now."""
        bases, offsets = _u8(bases), _u64(offsets)
        n = len(offsets) - 1
        cap = cand_cap if cand_cap is not None else max(1024, 8 * n)
        reads = np.empty(n, dtype=READ_DTYPE)
        cands = np.empty(cap, dtype=CAND_DTYPE)
        res = _Result(reads.ctypes.data, cands.ctypes.data, cap, 0)
        b = _Batch(n, offsets.ctypes.data, bases.ctypes.data)
        t = C.c_uint64()
        rc = lib().mg_server_submit_into(self.h, C.byref(b), C.byref(res), C.byref(t))
        if rc == -9:
            return None
        _check(rc, "mg_server_submit_into")
        self._into[t.value] = (reads, cands, res)
        return t.value

    def _result(self, ticket: int, fn, *extra):
        if ticket in self._into:
            reads, cands, res = self._into[ticket]
            rc = fn(self.h, ticket, None, *extra)
            if rc != 0:
                self._into.pop(ticket, None)
            _check(rc, "mg_server_poll")
            if rc == 0:
                return None
            return Results(reads, cands[: res.n_cands].copy())
        n = self._pending.get(ticket, 0)
        cap = max(1024, 8 * n)
        while True:
            reads = np.empty(n, dtype=READ_DTYPE)
            cands = np.empty(cap, dtype=CAND_DTYPE)
            r = _Result(reads.ctypes.data, cands.ctypes.data, cap, 0)
            rc = fn(self.h, ticket, C.byref(r), *extra)
            if rc == -3 and r.n_cands > cap:
                cap = int(r.n_cands)
                continue
            if rc < 0 and rc != -8:
                self._pending.pop(ticket, None)  # the server no longer tracks a failed request
            _check(rc, "mg_server_poll")
            if rc == 0:
                return None
            self._pending.pop(ticket, None)
            return Results(reads, cands[: r.n_cands].copy())

    def poll(self, ticket: int) -> Results | None:
        return self._result(ticket, lib().mg_server_poll)

    def wait(self, ticket: int, timeout_ms: int = 60000) -> Results:
        res = self._result(ticket, lib().mg_server_wait, timeout_ms)
        if res is None:
            raise MirageError(-7, "mg_server_wait", "timed out")
        return res

    def close(self):
        if getattr(self, "h", None):
            lib().mg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
