"""Launch-shape tuner of the batched form (the project's replacement for the reference's run-time
work balancing, Hardware::TryAutoIncreaseBlocksize / HardwareAutoConfigure, Hardware.cpp:
138-228).

It times the classification of a batch of reads already resident in the device (CUDA events on
the call's stream, the median of a few steps) under candidate launch shapes (mg_tuning), one
field at a time from the current best (coordinate descent over small grids), then the chunking
of a host-buffer batch end to end, within a time budget. Results never depend on the shapes
(each candidate's output is checked bitwise against the defaults'); only the times do. The best
shapes go to the tuning file of the GPU model under the index's density class, which mg_open
reads:

    python -m mirage_b200.tune --workload uneven --seconds 90

Workloads are the seeded synthetic sets of mirage_b200.synth: uneven (1M reads of 75-300 bp on
5,000 references, a dense index), long (reads of 1-20 kb on the same references: only the
long-read tier's shape is tuned), plain (a sparse index), large (a saturated index).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

import mirage_b200 as M

HERE = os.path.dirname(os.path.abspath(__file__))

# fields and candidate values, in the order they are swept
SHORT_GRID = {
    "first_tier": [1, 2, 3],
    "dual_blocks_per_sm": [3, 4, 5],
    "steal_chunk": [1, 2, 4, 8, 16],
    "second_blocks_per_sm": [1, 2, 4, 6],
    "third_blocks_per_sm": [2, 4, 6],
    "finish_blocks_per_sm": [2, 4, 8],
}
LONG_GRID = {"long_blocks_per_sm": [1, 2]}
E2E_GRID = {"chunks": [4, 6, 8], "weighted_chunks": [1, 2], "pack_bases": [1, 2]}


def tuning_path(device: int = 0) -> str:
    """tuning/<device name>.txt beside the library (the file mg_open reads)."""
    import torch

    name = torch.cuda.get_device_name(device).replace(" ", "_").replace("/", "_")
    return os.path.join(HERE, "tuning", name + ".txt")


def read_tuning_file(path: str, notes: dict | None = None) -> dict[str, dict[str, int]]:
    """Entries of a tuning file: class -> fields (and, into `notes`, each line's comment)."""
    out: dict[str, dict[str, int]] = {}
    if not os.path.exists(path):
        return out
    with open(path) as f:
        for raw in f:
            body, _, note = raw.partition("#")
            words = body.split()
            if not words:
                continue
            out[words[0]] = {k: int(v) for k, v in (kv.split("=", 1) for kv in words[1:] if "=" in kv)}
            if notes is not None:
                notes[words[0]] = note.strip()
    return out


def write_tuning_file(path: str, cls: str, fields: dict[str, int], note: str = "") -> None:
    """Set the entry of density class `cls` (the other classes' lines are kept)."""
    notes: dict[str, str] = {}
    entries = read_tuning_file(path, notes)
    entries[cls] = {**entries.get(cls, {}), **{k: int(v) for k, v in fields.items() if k in M.TUNING_FIELDS}}
    if note:
        notes[cls] = note.replace("\n", " ").replace("#", "")
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write("# mirage_b200 launch shapes per index density class (postings per 28-bit hash: sparse\n"
                "# < 0.25 <= dense < 4 <= saturated), written by python -m mirage_b200.tune; read by mg_open.\n")
        for c in sorted(entries):
            line = c + " " + " ".join(f"{k}={v}" for k, v in sorted(entries[c].items()))
            f.write(line + (f"  # {notes[c]}" if notes.get(c) else "") + "\n")


class _Resident:
    """A batch resident in device memory and the device step over it."""

    def __init__(self, ix: M.Index, reads, device: int = 0):
        import torch

        self.torch = torch
        self.ix = ix
        self.n = len(reads)
        dev = f"cuda:{device}"
        self.cap = 16 * self.n + 1024
        self.bases = torch.from_numpy(reads.data).to(dev)
        self.offs = torch.from_numpy(reads.offs.view(np.int64)).to(dev)
        self.reads = torch.empty(self.n * 16, dtype=torch.uint8, device=dev)
        self.cands = torch.empty(self.cap * 16, dtype=torch.uint8, device=dev)
        self.nc = torch.zeros(1, dtype=torch.int64, device=dev)
        self.stream = torch.cuda.Stream(device=dev)

    def step(self) -> float:
        t = self.torch
        e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        self.ix.classify_device(self.n, self.offs.data_ptr(), self.bases.data_ptr(), self.reads.data_ptr(),
                                self.cands.data_ptr(), self.cap, self.nc.data_ptr(), self.stream.cuda_stream)
        e1.record(self.stream)
        self.n_cands = self.ix.device_sync(self.stream.cuda_stream)
        return e0.elapsed_time(e1)

    def time(self, reps: int = 5) -> float:
        self.step()
        return float(np.median([self.step() for _ in range(reps)]))

    def output(self) -> tuple[bytes, bytes]:
        return self.reads.cpu().numpy().tobytes(), self.cands[: 16 * self.n_cands].cpu().numpy().tobytes()


def tune(ix: M.Index, reads, grid: dict, seconds: float = 60.0, reps: int = 5, e2e: bool = True,
         device: int = 0, start: dict | None = None) -> dict:
    """Coordinate descent over `grid` from `start` (default: the library's defaults), within about
    `seconds`. Returns the best fields, their device step time, the defaults' time and the trials."""
    t_end = time.time() + seconds
    res = _Resident(ix, reads, device)
    ix.set_tuning()
    default_ms = res.time(reps)
    want = res.output()
    best = dict(start or {})
    ix.set_tuning(**best)
    best_ms = res.time(reps)
    trials = [{"fields": dict(best), "ms": best_ms}]
    for field, values in grid.items():
        for v in values:
            if time.time() > t_end:
                break
            cand = {**best, field: v}
            if cand == best:
                continue
            ix.set_tuning(**cand)
            ms = res.time(reps)
            if res.output() != want:
                raise RuntimeError(f"launch shapes {cand} changed the results")
            trials.append({"fields": cand, "ms": ms})
            if ms < best_ms:
                best, best_ms = cand, ms
    out = {"fields": best, "ms_per_step": best_ms, "default_ms_per_step": default_ms, "trials": trials}
    if e2e and time.time() < t_end:
        # chunking of a host-buffer batch, timed end to end from pinned memory
        import torch

        h_bases = torch.from_numpy(reads.data).pin_memory()
        h_offs = torch.from_numpy(reads.offs.view(np.int64)).pin_memory()
        h_reads = torch.empty(len(reads) * 16, dtype=torch.uint8).pin_memory()
        h_cands = torch.empty(res.cap * 16, dtype=torch.uint8).pin_memory()

        def e2e_ms() -> float:
            ts = []
            for _ in range(reps + 1):
                t0 = time.perf_counter()
                ix.classify_ptrs(len(reads), h_offs.data_ptr(), h_bases.data_ptr(), h_reads.data_ptr(),
                                 h_cands.data_ptr(), res.cap)
                ts.append(1000 * (time.perf_counter() - t0))
            return float(np.median(ts[1:]))

        ix.set_tuning(**best)
        e2e_best = e2e_ms()
        e2e_want = h_reads.numpy().tobytes()
        out["e2e_trials"] = [{"fields": dict(best), "ms": e2e_best}]
        for field, values in E2E_GRID.items():
            for v in values:
                if time.time() > t_end:
                    break
                cand = {**best, field: v}
                if cand == best:
                    continue
                ix.set_tuning(**cand)
                ms = e2e_ms()
                if h_reads.numpy().tobytes() != e2e_want:
                    raise RuntimeError(f"launch shapes {cand} changed the results end to end")
                out["e2e_trials"].append({"fields": cand, "ms": ms})
                if ms < e2e_best:
                    best, e2e_best = cand, ms
        out["fields"] = best
        out["e2e_ms"] = e2e_best
    ix.set_tuning(**best)
    return out


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--workload", default="uneven", choices=["uneven", "long", "plain", "large"])
    ap.add_argument("--reads", type=int, default=None)
    ap.add_argument("--seconds", type=float, default=90.0)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=None, help="tuning file (default: the GPU model's, beside the library)")
    args = ap.parse_args()
    from mirage_b200 import synth

    import torch

    torch.cuda.set_device(args.device)
    name, n_def = {"uneven": ("uneven_fast", 1_000_000), "long": ("long_fast", 20_000), "plain": ("plain", 11_000),
                   "large": ("repeats", 2_000_000)}[args.workload]
    kw = {"reads_seed": 7} if name.endswith("_fast") else {}
    refs, reads, _ = synth.workload(name, 1.0, seed=2024, n_reads=args.reads or n_def, **kw)
    img = M.build_image(refs.data, refs.offs, refs.headers, k=31, device=args.device)
    ix = M.Index(img, k=31, device=args.device)
    _, cls = ix.get_tuning()
    path = args.out or tuning_path(args.device)
    start = read_tuning_file(path).get(cls, {})
    grid = LONG_GRID if args.workload == "long" else SHORT_GRID
    res = tune(ix, reads, grid, args.seconds, e2e=args.workload != "long", device=args.device,
               start={k: v for k, v in start.items() if k not in grid})
    fields = res["fields"] if args.workload != "long" else {k: res["fields"][k] for k in LONG_GRID}
    write_tuning_file(path, cls, fields,
                      note=f"{cls}: {args.workload} workload, {len(reads)} reads; device step {res['ms_per_step']:.3f} ms "
                           f"(defaults {res['default_ms_per_step']:.3f} ms)"
                           + (f"; end to end {res['e2e_ms']:.3f} ms (first setting {res['e2e_trials'][0]['ms']:.3f} ms)"
                              if res.get("e2e_trials") else ""))
    print(json.dumps({"class": cls, "file": path, **{k: v for k, v in res.items() if k != "trials"},
                      "n_trials": len(res["trials"])}))
    ix.close()


if __name__ == "__main__":
    main()
