"""TEST INFRASTRUCTURE ONLY -- Python access to the CPU restatement (liboracle.so) and to the
reference harness dumps. Imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg; the product never imports this module."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
HARNESS = os.path.join(REF_DIR, "mg_ref_harness")
MIRAGE_REF = os.path.join(REF_DIR, "mirage_ref")


class _Cand(C.Structure):
    _fields_ = [("ref", C.c_uint32), ("n_runs", C.c_uint32), ("run_off", C.c_uint32),
                ("score", C.c_float), ("pct", C.c_float), ("rel", C.c_float)]


class _Run(C.Structure):
    _fields_ = [("start_ref", C.c_uint32), ("start_q", C.c_uint32), ("last_ref", C.c_uint32),
                ("last_q", C.c_uint32)]


class _Strand(C.Structure):
    _fields_ = [("cand_off", C.c_uint32), ("n_cand", C.c_uint32), ("highest", C.c_float)]


class _Read(C.Structure):
    _fields_ = [("highest", C.c_float), ("strand", C.c_int32), ("reported", C.c_int32),
                ("n_top", C.c_uint32)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.mgo_open.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]
        L.mgo_close.argtypes = [C.c_void_p]
        L.mgo_n_refs.argtypes = [C.c_void_p]
        L.mgo_n_refs.restype = C.c_uint32
        L.mgo_ref_size.argtypes = [C.c_void_p, C.c_uint32]
        L.mgo_ref_size.restype = C.c_uint32
        L.mgo_hash28.argtypes = [C.c_char_p, C.c_int]
        L.mgo_hash28.restype = C.c_uint32
        L.mgo_relative_score.argtypes = [C.c_float, C.c_float, C.c_float]
        L.mgo_relative_score.restype = C.c_float
        L.mgo_classify.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_int,
                                   C.c_void_p, C.c_void_p, C.POINTER(C.POINTER(_Cand)),
                                   C.POINTER(C.c_uint64), C.POINTER(C.POINTER(_Run)),
                                   C.POINTER(C.c_uint64), C.c_void_p, C.c_void_p, C.c_uint64]
        L.mgo_classify_count.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_int]
        L.mgo_classify_count.restype = C.c_int64
        L.mgo_free.argtypes = [C.c_void_p]
        L.mgo_logf_bits.argtypes = [C.c_uint32, C.c_uint64, C.c_void_p]
        L.mgo_logf_bits.restype = None
        _lib = L
    return _lib


def logf_bits(lo_bits: int, n: int) -> np.ndarray:
    """Host libm logf at n consecutive float bit patterns from lo_bits."""
    out = np.empty(n, dtype=np.float32)
    lib().mgo_logf_bits(lo_bits, n, out.ctypes.data)
    return out


def fbits(x: float) -> int:
    return int(np.array([x], dtype=np.float32).view(np.uint32)[0])


@dataclass
class Strand:
    slot: int
    length: int
    cands: list = field(default_factory=list)  # (ref, n_runs, score_bits, pct_bits|None, runs)
    highest: int = 0                           # float bits
    scores: list = field(default_factory=list)  # (rel_bits, ref) in candidate order


@dataclass
class Result:
    strands: list
    merged: list  # (read, strand, highest_bits, top refIDs sorted)


class Index:
    def __init__(self, path: str, k: int = 31):
        self.L = lib()
        h = C.c_void_p()
        rc = self.L.mgo_open(path.encode(), k, C.byref(h))
        if rc != 0:
            raise RuntimeError(f"mgo_open({path}) failed: {rc}")
        self.h = h

    def close(self):
        if self.h:
            self.L.mgo_close(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def n_refs(self) -> int:
        return self.L.mgo_n_refs(self.h)

    def classify(self, bases: np.ndarray, offs: np.ndarray, threads: int = 1) -> Result:
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.uint64)
        n = len(offs) - 1
        strands = (_Strand * (2 * n + 1))()
        reads = (_Read * (n + 1))()
        cp = C.POINTER(_Cand)()
        rp = C.POINTER(_Run)()
        nc = C.c_uint64()
        nr = C.c_uint64()
        cap = 64 * n + 1024
        top = np.zeros(cap, dtype=np.uint32)
        top_off = np.zeros(n + 1, dtype=np.uint64)
        rc = self.L.mgo_classify(self.h, bases.ctypes.data, offs.ctypes.data, n, threads,
                                 C.cast(strands, C.c_void_p), C.cast(reads, C.c_void_p),
                                 C.byref(cp), C.byref(nc), C.byref(rp), C.byref(nr),
                                 top.ctypes.data, top_off.ctypes.data, cap)
        if rc != 0:
            raise RuntimeError(f"mgo_classify failed: {rc}")
        try:
            res_strands = []
            for i in range(n):
                L = int(offs[i + 1] - offs[i])
                for s in range(2):
                    st = strands[2 * i + s]
                    S = Strand(2 * i + s, L)
                    for c in range(st.n_cand):
                        cd = cp[st.cand_off + c]
                        runs = [(rp[cd.run_off + j].start_ref, rp[cd.run_off + j].start_q,
                                 rp[cd.run_off + j].last_ref, rp[cd.run_off + j].last_q)
                                for j in range(cd.n_runs)]
                        scored = cd.score > -1
                        S.cands.append((cd.ref, cd.n_runs, fbits(cd.score),
                                        fbits(cd.pct) if scored else None, runs))
                        if scored:
                            S.scores.append((fbits(cd.rel), cd.ref))
                    S.highest = fbits(st.highest)
                    res_strands.append(S)
            merged = []
            for i in range(n):
                rd = reads[i]
                t0 = int(top_off[i])
                merged.append((i, rd.strand, fbits(rd.highest),
                               sorted(int(x) for x in top[t0 : t0 + rd.n_top])))
            return Result(res_strands, merged)
        finally:
            self.L.mgo_free(C.cast(cp, C.c_void_p))
            self.L.mgo_free(C.cast(rp, C.c_void_p))

    def count(self, bases: np.ndarray, offs: np.ndarray, threads: int = 1) -> int:
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.uint64)
        r = self.L.mgo_classify_count(self.h, bases.ctypes.data, offs.ctypes.data, len(offs) - 1, threads)
        if r < 0:
            raise RuntimeError(f"mgo_classify_count failed: {r}")
        return int(r)


def parse_dump(path: str) -> Result:
    """Parse a dump written by ref_harness.cpp (the reference's own results)."""
    strands: list[Strand] = []
    merged = []
    cur = None
    cand = None
    import gzip
    with (gzip.open(path, "rt") if path.endswith(".gz") else open(path)) as f:
        for line in f:
            t = line.split()
            if not t or t[0] == "#":
                continue
            if t[0] == "S":
                cur = Strand(int(t[1]), int(t[3]))
                strands.append(cur)
            elif t[0] == "C":
                cand = (int(t[1]), int(t[2]), int(t[3], 16), None if t[4] == "-" else int(t[4], 16), [])
                cur.cands.append(cand)
            elif t[0] == "R":
                cand[4].append(tuple(int(x) for x in t[1:5]))
            elif t[0] == "H":
                cur.highest = int(t[1], 16)
            elif t[0] == "P":
                cur.scores.append((int(t[1], 16), int(t[2])))
            elif t[0] == "M":
                n_top = int(t[4])
                merged.append((int(t[1]), int(t[2]), int(t[3], 16), sorted(int(x) for x in t[5 : 5 + n_top])))
    return Result(strands, merged)


def compare(a: Result, b: Result, max_report: int = 10) -> list[str]:
    """Field-by-field differences between two results (empty list = identical)."""
    diffs = []
    if len(a.strands) != len(b.strands):
        return [f"strand count {len(a.strands)} != {len(b.strands)}"]
    for sa, sb in zip(a.strands, b.strands):
        if sa.cands != sb.cands or sa.highest != sb.highest or sa.scores != sb.scores:
            diffs.append(f"strand {sa.slot}: {sa.cands} H={sa.highest:08x} vs {sb.cands} H={sb.highest:08x}")
            if len(diffs) >= max_report:
                return diffs
    if a.merged != b.merged:
        for ma, mb in zip(a.merged, b.merged):
            if ma != mb:
                diffs.append(f"merged {ma} vs {mb}")
                if len(diffs) >= max_report:
                    break
    return diffs


def run_harness(mhm: str, reads_fasta: str, out: str | None = None, job: int = 1,
                threads: int = 1, logdir: str | None = None, time_only: bool = False,
                limit: int | None = None, word: int = 4, scheme: str | None = None, repeat: int = 1,
                all_lines: bool = False):
    """Run the reference harness (oracle/_ref/mg_ref_harness); returns its last timing JSON
    line (all of them, one per repetition, as dicts when all_lines). scheme "stock": the stock
    program's worker count and job size instead of job / threads (see ref_harness.cpp)."""
    cmd = [HARNESS if word == 4 else HARNESS + "64", "--mhm", mhm, "--reads", reads_fasta, "--job", str(job), "--threads", str(threads)]
    if scheme:
        cmd += ["--scheme", scheme]
    if repeat > 1:
        cmd += ["--repeat", str(repeat)]
    if out:
        cmd += ["--out", out]
    if logdir:
        cmd += ["--logdir", logdir]
    if time_only:
        cmd += ["--time"]
    if limit is not None:
        cmd += ["--limit", str(limit)]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"harness failed: {p.stderr[-2000:]}")
    lines = [l for l in p.stderr.splitlines() if l.startswith("{")]
    if all_lines:
        import json

        return [json.loads(l) for l in lines]
    return lines[-1] if lines else ""


def build_mhm_with_reference(ref_fasta: str, workdir: str, word: int = 4) -> str:
    """Build a .mhm from FASTA with the reference's own builder (the stock program)."""
    workdir = os.path.abspath(workdir)
    os.makedirs(os.path.join(workdir, "mirage", "data"), exist_ok=True)
    os.makedirs(os.path.join(workdir, "x"), exist_ok=True)
    os.makedirs(os.path.join(workdir, "out"), exist_ok=True)
    cfg = os.path.join(workdir, "mirage", "data", "mirage.identifier.cfg")
    with open(cfg, "w") as f:
        f.write(_BUILD_CFG)
    q = os.path.join(workdir, "q.fasta")
    with open(q, "w") as f:
        f.write(">q\n" + "ACGT" * 40 + "\n")
    p = subprocess.run([MIRAGE_REF if word == 4 else MIRAGE_REF + "64", "-query", q, "-reference", os.path.abspath(ref_fasta), "-outputpath",
                        os.path.abspath(os.path.join(workdir, "out"))], cwd=os.path.join(workdir, "x"),
                       capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(p.stdout[-2000:] + p.stderr[-2000:])
    found = []
    for root, _, files in os.walk(os.path.join(workdir, "out")):
        found += [os.path.join(root, f) for f in files if f.endswith(".mhm")]
    if len(found) != 1:
        raise RuntimeError(f"expected one .mhm, got {found}")
    return found[0]


# The sample configuration's hot-path keys (the reference's data/mirage.identifier.cfg
# values), enough for the stock program to build and load an index.
_BUILD_CFG = """Query:./q.fasta
Reference:./r.fasta
ReferenceDatabaseSort:0
considerthreshold:31
OutputPath:/tmp
Hardware_Auto_Detect:1
Hardware_BlockSize_Default_CPU:7500
Hardware_BlockSize_Default_GPU:20000
Hardware_BlockSize_AutoIncrease_Enabled_Default:1
Hardware_BlockSize_AutoIncrease_IncreasePercentage:130
Hardware_maxCPUThreads:200000
Hardware_MANUAL_Types:CPU
Hardware_MANUAL_Enabled:1
Hardware_MANUAL_BlockSize:200
Hardware_MANUAL_BlockSize_AutoIncrease_Enabled:1
Hashmap_Use_Experimental_LazyLoading:1
Reference_Divide:0
Reference_Divideby:80
hashmap_threshold_percentage:0
Hashmap_LazyLoading_Cache_FreeMemory_Percentage_Threshold:10
Hashmap_LazyLoading_Cache_FreeMemory_Percentage_Tidy:20
Hashmap_Performance_Boost:0
hashmap_generate_proportiondatabase_percentage:100
Hashmap_Save_Hashmap_During_Build_Below_Free_Memory:0
Hashmap_Load_Hashmap_From_File_After_Build:1
Hashmap_Load_Hashmap_Percentage:100
hashmap_load_hashmap_skip_on_failure:1
Hardware_Device_Queue_MaxSize:1
Hashmap_Load_Reference_Memory_UsageMode:extreme
LogThreshold_HighSensitivity:0.4
LogThreshold_HighPrecision:1
LogThreshold_Balanced:0.7
UltraFastMode:Sensitive
OutputMode:silent
output_firstresults_only:1
output_save_hashmap_database:1
MultiNode_CombineResult_AllNodes:1
Screen_Resize:0
Screen_COLS:160
Screen_ROWS:60
"""
