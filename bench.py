#!/usr/bin/env python
"""Benchmark of the MirAge classification hot path on B200.

Workload ("uneven", the largest configuration quoted that fits one GPU): 5,000 synthetic references with
log-normal lengths (median 50 kb, sigma 0.8, ~344 Mbp, GC per reference uniform in [0.3, 0.7]),
1,000,000 reads per GPU of uniform length 75-300 bp with 0.5% substitutions, 0.1% single-base
indels and 20% unrelated reads; seeded synthetic data (no public read set is named). A step is
the classification of one batch of 1,000,000 reads (both strands, seed lookup through best
reference pick). Inputs (index ~4.6 GB, reads ~187 MB) are larger than the 126 MB L2, so no
flush is needed between steps.

  value       reads/s with the batch already resident in HBM (fused batched form), device-timed
              with CUDA events on the launching stream, max over ranks.
  e2e         reads/s through the C ABI (mg_classify) from pinned host buffers: host->device
              copy of the reads and device->host copy of every result inside the timed region.
  plain       the same e2e measurement of the plain form (mg_score_batch, one block per read).
  served      the served form (mg_server_*): saturated reads/s with requests of log-uniform
              size in [1, 50000] reads, then p50/p99 request latency under Poisson arrivals at
              25/50/75/90% of that rate.
  roofline    the warp tiers (the dual-strand kernel and the general warp kernel, which take
              every read once between them; 97% of a step): algorithmic bytes per step / their
              CUDA-event time, against the measured HBM copy bandwidth (peak) and against the
              random 32-byte-sector gather bandwidth measured in the same run (gather_peak).
  cpu_baseline the reference's own CPU path (oracle/_ref harness) when built, else the CPU
              restatement, on a bounded sample with all host threads.

--impl reference times the reference's CPU implementation of the path (see above) on the same
workload, one bounded sample per step.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 2024
N_READS = 1_000_000
# kernels one batched call launches: dual-strand tier, second dual-strand tier (its leftovers),
# the finishing pass, general warp tier, block tier, global tier, candidate count, scan, scatter
LAUNCHES_PER_BATCH = 9
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one k_classify_dual launch on the
# default workload (1,000,000 reads, scale 1.0): a constant from one ncu capture of this kernel,
# not a measurement of this run
# dram__bytes_read.sum + dram__bytes_write.sum of k_classify_dual and of k_finish_dual, one launch each
DUAL_TRAFFIC_DEFAULT = (2_986_232_832 + 47_951_616) + (357_686_528 + 63_106_304)
DUAL_TRAFFIC_WHAT = ("DRAM bytes per step of k_classify_dual + k_finish_dual (the kernels of kernel_ms but the "
                     "side tiers): a constant from one ncu capture of each on this workload "
                     "(dram__bytes_read.sum + dram__bytes_write.sum), not measured in this run")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class ClockSampler:
    """nvidia-smi samples (SM clock, throttle reasons) while the timed region runs."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def wait_first(self, timeout: float = 5.0) -> None:
        """Block until nvidia-smi has written its first sample (or the timeout passes)."""
        t = time.time()
        while self.proc and time.time() - t < timeout:
            try:
                if os.path.getsize(self.path) > 0:
                    return
            except OSError:
                pass
            time.sleep(0.05)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = max(mx, float(f[2]))
                except ValueError:
                    continue
                for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), f[5:9]):
                    if v.lower() == "active":
                        reasons.add(name)
        except OSError:
            pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def hash28_windows_2d(seqs: np.ndarray) -> np.ndarray:
    """CreateHash24 of equal-length windows (rows of a uint8 matrix)."""
    x = np.full(seqs.shape[0], 2166136261, dtype=np.uint64)
    for j in range(seqs.shape[1]):
        x = ((x * 16777619) & 0xFFFFFFFF) ^ seqs[:, j].astype(np.uint64)
    return (((x >> 28) ^ x) & 0x0FFFFFFF).astype(np.uint32)


_COMP = np.zeros(256, np.uint8)
for _a, _b in zip(b"ACGTN", b"TGCAN"):
    _COMP[_a] = _b


def seed_hashes(data: np.ndarray, offs: np.ndarray, k: int = 31, chunk_seeds: int = 1 << 21):
    """The hashes of every seed of both strands (Analyser.cpp:1453-1478: seeds at p = 0, step,
    2 step, ... while p < L - k; the reverse complement read from the forward bytes), yielded in
    chunks of about chunk_seeds."""
    step, h = k // 2, k - k // 2 + 1
    offs = offs.astype(np.int64)
    lens = np.diff(offs)
    ns = np.where(lens > k, (lens - k + step - 1) // step, 0)
    cum = np.concatenate([[0], np.cumsum(ns)])
    i0, n = 0, len(lens)
    while i0 < n:
        i1 = int(np.searchsorted(cum, cum[i0] + chunk_seeds, side="right"))
        i1 = min(n, max(i1, i0 + 1))
        cnt = ns[i0:i1]
        rid = np.repeat(np.arange(i0, i1), cnt)
        j = np.arange(int(cnt.sum())) - np.repeat(cum[i0:i1] - cum[i0], cnt)
        p = j * step
        o, L = offs[rid], lens[rid]
        yield hash28_windows_2d(data[(o + p)[:, None] + np.arange(h)[None, :]])
        yield hash28_windows_2d(_COMP[data[(o + L - 1 - p)[:, None] - np.arange(h)[None, :]]])
        i0 = i1


def algorithmic_bytes(ix, reads, n_cands: int, k: int = 31) -> dict:
    """Bytes the path must move per batch (each term one access a minimal implementation
    cannot avoid): the read bytes; per seed of both strands one 32-byte directory sector and the
    32-byte sectors holding its postings (8 bytes each); per scored candidate two 32-byte
    reference windows (head and tail of at least one run); 16 bytes of result per read and per
    candidate."""
    lens = reads.lengths().astype(np.int64)
    post_bytes = 0
    n_seeds = 0
    for hs in seed_hashes(reads.data, reads.offs, k):
        cnt = ix.bucket_sizes(hs).astype(np.int64)
        n_seeds += len(hs)
        post_bytes += int((((cnt * 8) + 31) // 32 * 32).sum())
    seed_bytes = 32 * n_seeds
    read_bytes = int(lens.sum())
    total = read_bytes + seed_bytes + post_bytes + 64 * n_cands + 16 * len(lens) + 16 * n_cands
    return {"bytes": total, "read": read_bytes, "directory": seed_bytes, "postings": post_bytes,
            "ref_windows": 64 * n_cands, "results": 16 * (len(lens) + n_cands), "seeds": n_seeds}


def h2d_link_gbs(h_bases, d_bases):
    """Bandwidth of a plain copy of the pinned host bases to the device (5 copies after 2 warm-up
    copies, CUDA events), the bound the end-to-end figure is read against; None if it fails."""
    try:
        import torch

        with torch.cuda.device(d_bases.device):
            dst = torch.empty_like(d_bases)
            stream = torch.cuda.current_stream(d_bases.device)
            for _ in range(2):
                dst.copy_(h_bases, non_blocking=True)
            torch.cuda.synchronize()
            c0 = torch.cuda.Event(enable_timing=True)
            c1 = torch.cuda.Event(enable_timing=True)
            c0.record(stream)
            for _ in range(5):
                dst.copy_(h_bases, non_blocking=True)
            c1.record(stream)
            torch.cuda.synchronize()
            gbs = 5 * h_bases.numel() / (c0.elapsed_time(c1) / 1000) / 1e9
            del dst
            return gbs
    except Exception:  # a diagnostic: never fails the benchmark
        return None


def mhm_word(img: np.ndarray) -> int:
    """The .mhm word width (4 or 8): the 32-bit field 12 bytes after the 73-byte magic text."""
    return int.from_bytes(img[85:89].tobytes(), "little")


def load_synth():
    """The seeded workload generator (mirage_b200/synth.py, numpy only), loaded from its file so
    that the reference arm's process never imports the mirage_b200 package or its library."""
    import importlib.util

    if "mg_synth" not in sys.modules:
        spec = importlib.util.spec_from_file_location("mg_synth", os.path.join(ROOT, "mirage_b200", "synth.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules["mg_synth"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["mg_synth"]


# The workloads (one per configuration quoted for this path); `uneven` is the default line.
WORKLOADS = {
    "uneven": {"synth": "uneven_fast", "reads": 1_000_000, "cpu_sample": 100_000,
               "what": "uneven: {refs} refs {bp} bp log-normal (median 50 kb, sigma 0.8, GC 0.3-0.7), {n} reads "
                       "75-300 bp per GPU (0.5% subs, 0.1% indels, 20% unrelated)"},
    "long": {"synth": "long_fast", "reads": 100_000, "cpu_sample": 2_000,
             "what": "long: {refs} refs {bp} bp log-normal (the uneven references), {n} reads per GPU, log-normal "
                     "length median 5 kb clipped to 1-20 kb, 3% subs + 2% indels, 10% chimeras"},
    "plain": {"synth": "plain", "reads": 11_000, "cpu_sample": 11_000,
              "what": "plain: {refs} refs x 5,000 bp uniform, {n} reads of 150 bp per GPU (1% subs, 1 in 11 unrelated)"},
    "large": {"synth": "repeats", "reads": 10_000_000, "cpu_sample": 50_000,
              "what": "large: {refs} refs {bp} bp log-normal (median 80 kb) with 5% shared repeat segments, {n} reads "
                      "of 250 bp per GPU (1% subs)"},
}


def make_workload(scale: float, n_reads: int, rank: int, workload: str = "uneven"):
    synth = load_synth()
    w = WORKLOADS[workload]
    if w["synth"] in ("uneven_fast", "long_fast"):
        # one reference set (seed SEED) for every rank, one read set per rank
        refs, reads, _ = synth.workload(w["synth"], scale, seed=SEED, n_reads=n_reads, reads_seed=SEED + 1 + rank)
    else:
        refs, reads, _ = synth.workload(w["synth"], scale, seed=SEED + rank, n_reads=n_reads)
    return refs, reads


def workload_text(workload: str, refs, n: int) -> str:
    return WORKLOADS[workload]["what"].format(refs=len(refs), bp=int(refs.offs[-1]), n=n)


def cpu_baseline_and_parity(img: np.ndarray, reads, word: int, sample: int, gpu_reads: np.ndarray,
                            gpu_cands: np.ndarray) -> tuple[dict, dict | None]:
    """The reference CPU path (oracle harness) on the first `sample` reads of the batch with all
    host threads, one strand per job (per-read semantics); its dump of those reads is then
    compared bit for bit with the GPU's results for the same reads (from the e2e run). The CPU
    restatement is timed instead when the reference harness is not built (no parity then)."""
    from oracle import oracle as O
    from oracle import parity as P

    threads = os.cpu_count() or 1
    sub = reads.subset(min(sample, len(reads)))
    with tempfile.TemporaryDirectory(prefix="mg_cpu_") as tmp:
        mhm = os.path.join(tmp, "index.mhm")
        img.tofile(mhm)
        harness = O.HARNESS if word == 4 else O.HARNESS + "64"
        if os.path.exists(harness):
            fa = os.path.join(tmp, "reads.fasta")
            dump = os.path.join(tmp, "ref.dump")
            sub.write_fasta(fa)
            js = json.loads(O.run_harness(mhm, fa, out=dump, job=1, threads=threads, word=word))
            cpu = {"value": len(sub) / js["hot_s"], "unit": "reads/s", "cores": threads, "kind": "reference",
                   "sample": f"the first {len(sub)} reads of the batch; reference TPrepareGPUAnalysis + "
                             f"CPUGetHighestScore + strand merge, one strand per job on {threads} threads "
                             f"(index load excluded)"}
            t = time.perf_counter()
            want = P.canon_from_dump(O.parse_dump(dump))
            got = P.canon_from_arrays(gpu_reads, gpu_cands, len(sub))
            par = P.count_mismatches(want, got)
            par["examples"] = P.diff(want, got, limit=3)
            par["against"] = ("reference CPU path (oracle/_ref harness: TPrepareGPUAnalysis -> CPUGetHighestScore "
                              "-> strand merge, one strand per job) on the same reads and the same index")
            par["fields"] = ("per strand: scored candidates (refID, Score, percentageMatch, relative score bits) "
                             "and HighestScore bits; per read: kept strand, merged HighestScore bits, top group")
            par["gpu_results_from"] = "the last timed e2e step (mg_classify, host buffers)"
            par["compare_s"] = time.perf_counter() - t
            return cpu, par
        oix = O.Index(mhm)
        oix.count(sub.data[: int(sub.offs[min(1000, len(sub))])], sub.offs[: min(1000, len(sub)) + 1], threads)
        t = time.perf_counter()
        oix.count(sub.data, sub.offs, threads)
        dt = time.perf_counter() - t
        return {"value": len(sub) / dt, "unit": "reads/s", "cores": threads, "kind": "port",
                "sample": f"{len(sub)} reads of the same workload through the CPU restatement"}, None


def run_reference_arm(args, rank: int, world: int) -> None:
    """--impl reference: the reference's own CPU path on the host cores, on this arm's workload
    (the full batch per step). The index is built by the reference's own stock program from the
    references' FASTA, and the timed region is the reference harness's hot path under the stock
    program's thread scheme; this process never loads the mirage_b200 library."""
    if rank != 0:
        return
    from oracle import oracle as O

    refs, reads = make_workload(args.scale, args.reads, 0, args.workload)
    total_bp = int(refs.offs[-1])
    word = 8 if total_bp > 150_000_000 else 4  # the 32-bit layout stops at 4 GB of .mhm
    harness = O.HARNESS if word == 4 else O.HARNESS + "64"
    threads = os.cpu_count() or 1
    line = {"impl": "reference", "metric": "reads/s", "unit": "reads/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic"}
    if not os.path.exists(harness) or not os.path.exists(O.MIRAGE_REF + ("64" if word == 8 else "")):
        line["unavailable"] = "the reference CPU path (oracle/_ref) is not built on this machine"
        print(json.dumps(line), flush=True)
        return
    n = len(reads)
    with tempfile.TemporaryDirectory(prefix="mg_ref_") as tmp:
        rf = os.path.join(tmp, "refs.fasta")
        fa = os.path.join(tmp, "reads.fasta")
        refs.write_fasta(rf)
        reads.write_fasta(fa)
        t0 = time.time()
        mhm = O.build_mhm_with_reference(rf, os.path.join(tmp, "build"), word=word)
        t_build = time.time() - t0
        reps = O.run_harness(mhm, fa, word=word, scheme="stock", time_only=True, repeat=args.warmup + args.steps,
                             all_lines=True)
    timed = [r["hot_s"] for r in reps[args.warmup:]]
    ms = 1000 * float(np.mean(timed))
    value = n / (ms / 1000)
    r0 = reps[-1]
    line.update({
        "value": value, "ms_per_step": ms,
        "config": {"workload": workload_text(args.workload, refs, n), "k": 31, "mhm_word": word,
                   "reads_per_step": n},
        "scheme": {"prepare_workers": r0["threads"], "strands_per_job": r0["job"],
                   "what": "the stock program's scheduling: numCores x 4 TPrepareGPUAnalysis workers over jobs of "
                           "2 x max(1, reads / (numCores x 40 + 1)) strands (Analyser.cpp:3500-3503, 3712-3724), "
                           "then MatrixCPU::CPUGetHighestScore's own tasks, strand merge and top group; the whole "
                           "batch as one block"},
        "index": {"built_by": "the reference's stock program (oracle/_ref/mirage_ref%s) from the references' FASTA"
                              % ("64" if word == 8 else ""), "build_s": t_build, "load_s": r0["load_s"]},
        "cpu_baseline": {"value": value, "unit": "reads/s", "cores": threads, "kind": "reference",
                         "sample": f"all {n} reads of the batch per step (index build and load excluded)"},
        "e2e": {"value": value, "unit": "reads/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(line), flush=True)


def served_bench(M, ix, bases: np.ndarray, offs: np.ndarray, seed: int, level_s: float, clients: int = 8,
                 fracs=(0.25, 0.5, 0.75, 0.9, 1.0, 1.1)):
    """Served form (mg_server_*): saturated throughput, then latency under Poisson arrivals at
    fractions of it. Native client threads (mirage_b200/libmg_loadgen.so) drive the server
    through the public C ABI: requests are contiguous slices of the host reads with log-uniform
    sizes in [1, 50000] reads, whose pool is registered with the server (mg_server_register_host),
    so each submit copies the request's offsets and the server copies its bases to the device
    straight from the pool; the server writes the results into the client's own buffers
    (mg_server_submit_into), inside the measurement."""
    import ctypes as C

    class Report(C.Structure):
        _fields_ = [("reads_per_s", C.c_double), ("requests", C.c_uint64), ("reads", C.c_uint64),
                    ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("error", C.c_int)]

    LG = C.CDLL(os.path.join(ROOT, "mirage_b200", "libmg_loadgen.so"))
    LG.mg_loadgen_run.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_double, C.c_uint32,
                                  C.c_double, C.c_int, C.c_uint64, C.POINTER(Report)]
    bases = np.ascontiguousarray(bases, np.uint8)
    offs = np.ascontiguousarray(offs, np.uint64)
    n = len(offs) - 1
    sv = M.Server(ix)
    sv.register_host(bases)  # the reads' pool: requests' bases go to the device straight from it

    def run(rate: float, secs: float, depth: int, k: int) -> Report:
        rep = Report()
        rc = LG.mg_loadgen_run(sv.h, offs.ctypes.data, bases.ctypes.data, n, clients, secs, 50000, rate, depth,
                               seed + 1000 * k, C.byref(rep))
        if rc:
            raise RuntimeError(f"mg_loadgen_run: {rc} {M.lib().mg_last_error()}")
        return rep

    try:
        run(0.0, 0.5, 32, 0)  # warm-up
        sat = run(0.0, min(level_s, 5.0), 32, 1)
        levels = []
        for i, f in enumerate(fracs):
            r = run(f * sat.reads_per_s, level_s, 1, 2 + i)
            levels.append({"offered_frac": f, "offered_reads_s": f * sat.reads_per_s, "achieved_reads_s": r.reads_per_s,
                           "requests": int(r.requests), "p50_ms": r.p50_ms, "p99_ms": r.p99_ms, "mean_ms": r.mean_ms})
        return {"saturated": {"value": sat.reads_per_s, "unit": "reads/s", "p50_ms": sat.p50_ms, "p99_ms": sat.p99_ms},
                "requests": "log-uniform 1..50000 reads, contiguous slices of the batch",
                "clients": f"{clients} native threads (libmg_loadgen.so), closed loop 32 deep when saturated",
                "results": "written by the server into each client's buffers (mg_server_submit_into)",
                "bases": "the pool of reads registered with the server (mg_server_register_host): each request's "
                         "bases copied to the device from it, its offsets through the request ring",
                "arrivals": "Poisson (one process per client thread)", "seconds_per_level": level_s, "load": levels}
    finally:
        sv.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mirage", choices=["mirage", "reference"])
    ap.add_argument("--workload", default="uneven", choices=sorted(WORKLOADS),
                    help="uneven (default): 5,000 refs, 1M reads of 75-300 bp; long: the same refs, 100k reads "
                         "of 1-20 kb; plain: 200 x 5 kb refs, 11k reads of 150 bp; large: 20,000 refs ~2 Gbp "
                         "with shared repeats, 10M reads of 250 bp")
    ap.add_argument("--scale", type=float, default=1.0, help="shrink the reference set (tests)")
    ap.add_argument("--reads", type=int, default=None, help="reads per GPU per step (default: the workload's)")
    ap.add_argument("--cpu-sample", type=int, default=None, help="reads of the CPU baseline and parity sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--served-seconds", type=float, default=10.0, help="seconds per served-form load level (0: skip)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.reads is None:
        args.reads = WORKLOADS[args.workload]["reads"]
    if args.cpu_sample is None:
        args.cpu_sample = WORKLOADS[args.workload]["cpu_sample"]
    if args.workload not in ("uneven", "large"):
        # the served form runs on the index of configuration 2 (its request stream) and of the large
        # index stress; the plain and long workloads measure the batched and plain forms only
        args.served_seconds = 0.0

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    import mirage_b200 as M

    t0 = time.time()
    refs, reads = make_workload(args.scale, args.reads, rank, args.workload)
    t_gen = time.time() - t0
    t0 = time.time()
    img = M.build_image(refs.data, refs.offs, refs.headers, k=31, device=local)  # same bytes as the host build
    t_build = time.time() - t0
    word = mhm_word(img)
    t0 = time.time()
    ix = M.Index(img, k=31, device=local)
    t_open = time.time() - t0
    info = ix.info()
    log(f"[rank {rank}] gen {t_gen:.1f}s build {t_build:.1f}s open {t_open:.1f}s index {info}")
    n = len(reads)
    n_bases = int(reads.offs[-1])
    cap = 8 * n + 1024

    # pinned host buffers (the e2e inputs and outputs)
    h_bases = torch.from_numpy(reads.data).pin_memory()
    h_offs = torch.from_numpy(reads.offs.view(np.int64)).pin_memory()
    h_reads = torch.empty(n * 16, dtype=torch.uint8).pin_memory()
    h_cands = torch.empty(cap * 16, dtype=torch.uint8).pin_memory()
    # device-resident copies (the `value` inputs)
    d_bases = h_bases.to(f"cuda:{local}")
    d_offs = h_offs.to(f"cuda:{local}")
    d_reads = torch.empty(n * 16, dtype=torch.uint8, device=f"cuda:{local}")
    d_cands = torch.empty(cap * 16, dtype=torch.uint8, device=f"cuda:{local}")
    d_nc = torch.zeros(1, dtype=torch.int64, device=f"cuda:{local}")
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream

    def device_step():
        ix.classify_device(n, d_offs.data_ptr(), d_bases.data_ptr(), d_reads.data_ptr(), d_cands.data_ptr(), cap,
                           d_nc.data_ptr(), sp)

    def e2e_step(form="batched"):
        return ix.classify_ptrs(n, h_offs.data_ptr(), h_bases.data_ptr(), h_reads.data_ptr(), h_cands.data_ptr(), cap,
                                form)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    ix.set_timing(True)
    kernel_ms = np.zeros(5)
    step_ms = []
    # the clock sampler runs from before the warm-up to the end of the e2e timed region
    with ClockSampler(local) as clk:
        clk.wait_first()
        for _ in range(args.warmup):
            device_step()
            ix.device_sync(sp)
        barrier()
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        barrier()
        start.record(stream)
        for _ in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            device_step()
            e1.record(stream)
            n_cands = ix.device_sync(sp)  # per-step error check, as a caller would
            kernel_ms += ix.last_kernel_times()
            step_ms.append(e0.elapsed_time(e1))
        end.record(stream)
        barrier()
        total_ms = start.elapsed_time(end)
        total_ms = max_over_ranks(total_ms)
        ms_per_step = total_ms / args.steps
        value = world * n / (ms_per_step / 1000)
        # the launch shapes in effect (the tuning file's, for this GPU model and index class),
        # and the same device step under the library's defaults, untimed by the line's value
        shapes, density = ix.get_tuning()
        ix.set_tuning()
        defaults = ix.get_tuning()[0]
        default_ms = None
        if defaults != shapes:
            ts = []
            for i in range(3 + min(args.steps, 10)):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                device_step()
                e1.record(stream)
                ix.device_sync(sp)
                if i >= 3:
                    ts.append(e0.elapsed_time(e1))
            default_ms = float(np.mean(ts))
        ix.set_tuning(**shapes)
        tuning = {"density_class": density, "shapes": shapes, "source": os.environ.get("MG_TUNING_FILE") or
                  "tuning file of this GPU model beside the library (defaults where it has no entry)",
                  "ms_per_step": ms_per_step, "defaults": defaults, "default_ms_per_step": default_ms or ms_per_step}

        # end to end through the C ABI with pinned host buffers
        for _ in range(args.warmup):
            e2e_step()
        barrier()
        t = time.perf_counter()
        for _ in range(args.steps):
            n_c = e2e_step()
        torch.cuda.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t) / args.steps
        e2e = world * n / e2e_s
        # the same e2e measurement with the other upload of the bases (packed 2 bits per base on
        # host threads and unpacked on the device, or copied as given)
        upload = shapes["pack_bases"]
        ix.set_tuning(**{**shapes, "pack_bases": 3 - upload})
        for _ in range(2):
            e2e_step()
        barrier()
        k2 = max(1, min(args.steps, 10))
        t = time.perf_counter()
        for _ in range(k2):
            e2e_step()
        torch.cuda.synchronize()
        other_s = max_over_ranks(time.perf_counter() - t) / k2
        ix.set_tuning(**shapes)
    acgt = np.zeros(256, bool)
    acgt[list(b"ACGTacgt")] = True
    n_exc = int((~acgt[reads.data]).sum())
    h2d_given = n_bases + 8 * (n + 1)
    h2d_packed = (n_bases + 3) // 4 + 8 * n_exc + 8 * (n + 1)
    h2d = h2d_packed if upload == 2 else h2d_given
    d2h = 16 * n + 16 * n_c + 64
    link_gbs = h2d_link_gbs(h_bases, d_bases)

    # plain form (one block per read), same e2e measurement
    for _ in range(2):
        e2e_step("plain")
    barrier()
    t = time.perf_counter()
    plain_steps = max(1, min(args.steps, 3))
    for _ in range(plain_steps):
        e2e_step("plain")
    torch.cuda.synchronize()
    plain_s = max_over_ranks(time.perf_counter() - t) / plain_steps
    plain = world * n / plain_s

    served = None
    if args.served_seconds > 0:
        served = served_bench(M, ix, reads.data, reads.offs, SEED + 100 + rank, args.served_seconds)
        if dist:  # replicas: throughput adds up, latency is the worst rank's
            t = torch.tensor([served["saturated"]["value"]] + [x for l in served["load"] for x in
                              (l["achieved_reads_s"], l["p50_ms"], l["p99_ms"])], dtype=torch.float64,
                             device=f"cuda:{local}")
            s = t.clone()
            dist.all_reduce(s, op=dist.ReduceOp.SUM)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            served["saturated"]["value"] = float(s[0])
            for i, l in enumerate(served["load"]):
                l["achieved_reads_s"] = float(s[1 + 3 * i])
                l["p50_ms"], l["p99_ms"] = float(t[2 + 3 * i]), float(t[3 + 3 * i])
        served["served_over_plain"] = served["saturated"]["value"] / plain

    line = None
    if rank == 0:
        peaks = measured_peaks()
        hbm = peaks.get("hbm_gbs")
        ab = algorithmic_bytes(ix, reads, n_cands)
        # classification wall time per step: every tier, from the dual-strand tier's start to the
        # join of its finishing pass with the tiers beside it (the device step less the compaction);
        # the tiers take every read exactly once between them
        warp_ms = float(np.mean(step_ms)) - kernel_ms[4] / args.steps
        achieved = ab["bytes"] / (warp_ms / 1000) / 1e9
        gather = M.gather_bandwidth(local, 4 << 30)
        default_run = args.workload == "uneven" and args.scale == 1.0 and args.reads == N_READS
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm or 6650.0, "unit": "GB/s",
                "frac": achieved / (hbm or 6650.0),
                "traffic": DUAL_TRAFFIC_DEFAULT if default_run else None,
                "traffic_what": DUAL_TRAFFIC_WHAT if default_run else None,
                "gather_peak": gather, "frac_of_gather": achieved / gather,
                # the probe's own bytes (directory sectors + posting sectors) over the same time
                "probe_frac_of_gather": (ab["directory"] + ab["postings"]) / (warp_ms / 1000) / 1e9 / gather,
                "gather_peak_what": "random 32-byte sector gathers, 8 lanes per sector, over a 4 GiB buffer "
                                    "(mg_gather_bandwidth), measured in this run",
                "kernel": "classification: k_classify_dual + k_finish_dual, beside them the general, block "
                          "and global tiers (device step less compaction)",
                "kernel_ms": warp_ms,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if hbm else "fallback 6650 GB/s",
                "algorithmic_bytes_per_launch": ab}
        # an index and batch that fit the 126 MB L2 (configuration 1) are bound by L2 gathers, not HBM
        l2_resident = info["device_bytes"] + n_bases < 100e6
        if l2_resident:
            l2g = M.gather_bandwidth(local, 32 << 20)
            roof.update({"l2_gather_peak": l2g, "frac_of_l2_gather": achieved / l2g,
                         "l2_gather_peak_what": "the same gathers over a 32 MiB buffer, which L2 holds "
                                                "(mg_gather_bandwidth), measured in this run: the bound of an "
                                                "L2-resident index"})
        cpu, parity = None, None
        if not args.no_cpu_baseline and world == 1:
            try:
                cpu, parity = cpu_baseline_and_parity(img, reads, word, args.cpu_sample, h_reads.numpy(),
                                                      h_cands.numpy()[: 16 * n_c])
            except Exception as e:  # reported, not fatal
                cpu = {"value": None, "error": str(e)[:200]}
        line = {"metric": "reads/s", "value": value, "unit": "reads/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u8", "data": "synthetic",
                "config": {"workload": workload_text(args.workload, refs, n),
                           "index_bytes": len(img), "mhm_word": word, "k": 31,
                           "l2": ("index and reads fit the 126 MB L2: no flush, the bound is L2 gathers"
                                  if l2_resident else "inputs larger than L2 (index + reads), no flush"),
                           "parallelism": f"replicas x{world}, reads sharded"},
                "e2e": {"value": e2e, "unit": "reads/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "ms_per_step": 1000 * e2e_s, "host_buffers": "pinned",
                        "upload": "bases packed 2 bits each on host threads, unpacked on the device" if upload == 2
                                  else "bases copied as given",
                        "other_upload": {"upload": "bases copied as given" if upload == 2 else
                                         "bases packed 2 bits each on host threads, unpacked on the device",
                                         "value": world * n / other_s, "ms_per_step": 1000 * other_s,
                                         "h2d_bytes_per_step": h2d_given if upload == 2 else h2d_packed},
                        "link_h2d_gbs": link_gbs,
                        "link_what": "plain pinned-host-to-device copy of the step's bases on this machine, "
                                     "outside the timed regions"},
                "plain": {"value": plain, "unit": "reads/s", "ms_per_step": 1000 * plain_s,
                          "what": "mg_score_batch e2e (one block per read, one launch per batch)"},
                "batched_over_plain_e2e": e2e / plain,
                "served": served,
                "kernel_ms_per_step": {"what": "dual tier with its finishing pass on the call's stream; the "
                                               "general, block and global tiers on a second stream from the dual "
                                               "kernel's end, beside the finishing pass",
                                       "dual_warp_tier": kernel_ms[0] / args.steps,
                                       "general_warp_tier": kernel_ms[1] / args.steps,
                                       "block_tier": kernel_ms[2] / args.steps,
                                       "global_tier": kernel_ms[3] / args.steps,
                                       "compaction": kernel_ms[4] / args.steps},
                "roofline": roof, "cpu_baseline": cpu, "parity": parity, "clocks": clk.summary(),
                "gpu_launches": args.steps * LAUNCHES_PER_BATCH,
                "tuning": tuning,
                "setup_s": {"generate": t_gen, "index_build_device": t_build, "open": t_open}}
        print(json.dumps(line), flush=True)
    ix.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
