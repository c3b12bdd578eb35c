"""A profiling case: one seeded workload classified a few times and nothing else (no host copies
in the timed steps, no other measurement), so that an ncu capture of a classification kernel,
which runs the program once per pass, stays short:

    python -m mirage_b200.profile --workload uneven --scale 0.25 --reads 200000 --steps 4
    ncu --replay-mode application --clock-control none -k regex:"^k_classify_dual$" -s 3 -c 1 ... \\
        python -m mirage_b200.profile --workload uneven --scale 0.25 --reads 200000 --steps 4

Workloads are mirage_b200.synth's (uneven_fast, long_fast, plain, repeats). --form plain runs the
plain form (one block per read) instead of the batched one; --first-tier starts the dual-strand
tiers at the 64-, 128- or 256-posting tier (mg_tuning.first_tier). Prints the time of each step
(CUDA events; wall time for the plain form, whose copies it includes).
"""
from __future__ import annotations

import argparse
import json

import numpy as np

import mirage_b200 as M

SYNTH = {"uneven": "uneven_fast", "long": "long_fast", "plain": "plain", "large": "repeats"}


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--workload", default="uneven", choices=sorted(SYNTH))
    ap.add_argument("--scale", type=float, default=0.25)
    ap.add_argument("--reads", type=int, default=200_000)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--form", default="batched", choices=["batched", "plain"])
    ap.add_argument("--first-tier", type=int, default=0)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    import torch

    from mirage_b200 import synth

    torch.cuda.set_device(args.device)
    name = SYNTH[args.workload]
    kw = {"reads_seed": 2025} if name.endswith("_fast") else {}
    refs, reads, _ = synth.workload(name, args.scale, seed=2024, n_reads=args.reads, **kw)
    img = M.build_image(refs.data, refs.offs, refs.headers, k=31, device=args.device)
    ix = M.Index(img, k=31, device=args.device)
    if args.first_tier:
        ix.set_tuning(first_tier=args.first_tier)
    n = len(reads)
    dev = f"cuda:{args.device}"
    cap = 16 * n + 1024
    d_bases = torch.from_numpy(reads.data).to(dev)
    d_offs = torch.from_numpy(reads.offs.view(np.int64)).to(dev)
    d_reads = torch.empty(n * 16, dtype=torch.uint8, device=dev)
    d_cands = torch.empty(cap * 16, dtype=torch.uint8, device=dev)
    d_nc = torch.zeros(1, dtype=torch.int64, device=dev)
    st = torch.cuda.Stream(device=dev)
    ix.set_timing(True)
    ms = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        if args.form == "plain":  # host buffers and the index's own stream: wall time
            import time

            t0 = time.perf_counter()
            ix.classify(reads.data, reads.offs, form="plain", cand_cap=cap)
            ms.append(1000 * (time.perf_counter() - t0))
            continue
        else:
            ix.classify_device(n, d_offs.data_ptr(), d_bases.data_ptr(), d_reads.data_ptr(), d_cands.data_ptr(), cap,
                               d_nc.data_ptr(), st.cuda_stream)
            ix.device_sync(st.cuda_stream)
        e1.record(st)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    extra = {}
    if args.form == "batched":  # the last step's tier times and the reads each tier handed on
        extra = {"kernel_ms": [round(float(x), 4) for x in ix.last_kernel_times()], "handed_on": ix.last_tier_counts()}
    print(json.dumps({"workload": args.workload, "scale": args.scale, "reads": n, "bases": int(reads.offs[-1]),
                      "form": args.form, "index": ix.info(), "shapes": ix.get_tuning()[0], "step_ms": ms, **extra}))
    ix.close()


if __name__ == "__main__":
    main()
