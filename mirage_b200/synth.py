"""Seeded synthetic references and reads with the shapes of the MirAge benchmark workloads.

No public read set is named for this path, so every test and benchmark runs on data made here
from a fixed seed (numpy PCG64: identical bytes on every machine with the same numpy).

Workloads (``scale`` shrinks counts, never per-sequence shapes):

* ``plain``   200 references x 5,000 bp, uniform ACGT; 10,000 reads of 150 bp from uniform
              random references, positions and strands with 1% substitutions, plus 1,000
              unrelated uniform reads.
* ``uneven``  5,000 references, log-normal lengths (median 50 kb, sigma 0.8, total regenerated
              into 300 Mbp +- 10%), GC fraction per reference uniform in [0.3, 0.7];
              1,000,000 reads of uniform length in [75, 300] bp with 0.5% substitutions and
              0.1% single-base indels, 20% unrelated (GC 0.5).
* ``uneven_fast`` the same shapes with a vectorised read generator and a separate read seed
              (the benchmark's form: one reference set, one read set per GPU).
* ``long``    the same references; 100,000 reads, log-normal length (median 5 kb, clipped to
              1-20 kb), 3% substitutions + 2% indels, 10% chimeras of two references.
* ``long_fast`` the same shapes with a vectorised read generator and a separate read seed
              (the benchmark's form of ``long``).
* ``repeats`` 20,000 references, log-normal (median 80 kb, sigma 0.67), 5% of every reference
              overwritten by segments of 500-5,000 bp from a pool of 1,000 shared segments;
              10,000,000 reads of 250 bp with 1% substitutions.
"""
from __future__ import annotations

import numpy as np

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)
_COMP = np.zeros(256, dtype=np.uint8)
for _a, _b in zip(b"ACGTN", b"TGCAN"):
    _COMP[_a] = _b


def revcomp(seq: np.ndarray) -> np.ndarray:
    return _COMP[seq[::-1]]


class SeqSet:
    """Sequences as one uint8 buffer plus CSR offsets, with headers."""

    def __init__(self, data: np.ndarray, offs: np.ndarray, headers: list[bytes]):
        self.data = np.ascontiguousarray(data, dtype=np.uint8)
        self.offs = np.ascontiguousarray(offs, dtype=np.uint64)
        self.headers = headers

    def __len__(self) -> int:
        return len(self.offs) - 1

    def seq(self, i: int) -> np.ndarray:
        return self.data[int(self.offs[i]) : int(self.offs[i + 1])]

    def lengths(self) -> np.ndarray:
        return np.diff(self.offs)

    def subset(self, n: int) -> "SeqSet":
        end = int(self.offs[n])
        return SeqSet(self.data[:end], self.offs[: n + 1].copy(), self.headers[:n])

    def write_fasta(self, path: str, width: int = 0) -> None:
        with open(path, "wb") as f:
            for i in range(len(self)):
                f.write(b">" + self.headers[i] + b"\n")
                s = self.seq(i).tobytes()
                if width:
                    for j in range(0, len(s), width):
                        f.write(s[j : j + width] + b"\n")
                else:
                    f.write(s + b"\n")


def read_fasta(path: str) -> SeqSet:
    """Plain FASTA/FASTQ reader (sequence bytes kept as written, header without '>')."""
    headers: list[bytes] = []
    chunks: list[bytes] = []
    offs = [0]
    cur: list[bytes] = []
    fastq = False
    qline = 0
    with open(path, "rb") as f:
        for line in f:
            line = line.rstrip(b"\n").rstrip(b"\r")
            if line[:1] in (b">", b"@") and not (fastq and qline > 0):
                if headers:
                    s = b"".join(cur)
                    chunks.append(s)
                    offs.append(offs[-1] + len(s))
                headers.append(line[1:])
                fastq = line[:1] == b"@"
                qline = 0
                cur = []
            elif fastq:
                if qline == 0:
                    cur.append(line)
                qline += 1
            else:
                cur.append(line)
    if headers:
        s = b"".join(cur)
        chunks.append(s)
        offs.append(offs[-1] + len(s))
    data = np.frombuffer(b"".join(chunks), dtype=np.uint8).copy()
    return SeqSet(data, np.array(offs, dtype=np.uint64), headers)


def _bases(rng: np.random.Generator, n: int, gc: float = 0.5) -> np.ndarray:
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    return ACGT[rng.choice(4, size=n, p=p).astype(np.uint8)]


def _lognormal_lengths(rng, n, median, sigma, lo=None, hi=None, total=None, tol=0.1):
    for _ in range(1000):
        lens = np.round(np.exp(rng.normal(np.log(median), sigma, size=n))).astype(np.int64)
        if lo is not None or hi is not None:
            lens = np.clip(lens, lo if lo is not None else 1, hi if hi is not None else None)
        if total is None or abs(lens.sum() - total) <= tol * total:
            return lens
    raise RuntimeError("could not hit the requested total length")


def make_references(n_refs: int, lengths: np.ndarray, gc: np.ndarray, rng) -> SeqSet:
    offs = np.zeros(n_refs + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(lengths)
    data = np.empty(int(offs[-1]), dtype=np.uint8)
    # one categorical draw per reference keeps per-reference GC exact in expectation
    for i in range(n_refs):
        a, b = int(offs[i]), int(offs[i + 1])
        g = float(gc[i])
        data[a:b] = ACGT[np.searchsorted(np.cumsum([(1 - g) / 2, g / 2, g / 2]), rng.random(b - a)).astype(np.uint8)]
    return SeqSet(data, offs, [b"ref%d" % i for i in range(n_refs)])


def _substitute(rng, seq: np.ndarray, rate: float, chunk: int = 1 << 26) -> None:
    if rate <= 0 or len(seq) == 0:
        return
    # uniform draws in chunks (the same stream as one draw of len(seq))
    m = np.concatenate([np.flatnonzero(rng.random(min(chunk, len(seq) - a)) < rate) + a
                        for a in range(0, len(seq), chunk)])
    if len(m):
        code = np.searchsorted(ACGT, seq[m])
        code = np.where(code < 4, code, 0)
        seq[m] = ACGT[(code + rng.integers(1, 4, size=len(m))) % 4]


def _indels(rng, seq: np.ndarray, rate: float) -> np.ndarray:
    if rate <= 0:
        return seq
    n = rng.binomial(len(seq), rate)
    if n == 0:
        return seq
    pos = np.sort(rng.integers(0, len(seq), size=n))
    ins = rng.random(n) < 0.5
    out = seq
    # apply from the right so earlier positions stay valid
    for p, is_ins in zip(pos[::-1], ins[::-1]):
        if is_ins:
            out = np.concatenate([out[:p], ACGT[rng.integers(0, 4, size=1)], out[p:]])
        else:
            out = np.concatenate([out[:p], out[p + 1 :]])
    return out


def make_reads(refs: SeqSet, n_related: int, n_unrelated: int, length_fn, rng, sub=0.0,
               indel=0.0, chimera_frac=0.0, unrelated_gc=0.5) -> tuple[SeqSet, np.ndarray]:
    """Reads drawn from the references (random ref, position and strand) with errors, then
    unrelated random reads. Returns the reads and the true reference per read (-1 unrelated,
    first part's reference for chimeras)."""
    rlen = refs.lengths().astype(np.int64)
    n = n_related + n_unrelated
    lens = np.asarray(length_fn(n), dtype=np.int64)
    truth = np.full(n, -1, dtype=np.int64)
    seqs: list[np.ndarray] = []
    for i in range(n_related):
        L = int(lens[i])
        chim = chimera_frac > 0 and rng.random() < chimera_frac
        parts = []
        if chim:
            cut = int(rng.integers(1, L))
            plen = [cut, L - cut]
        else:
            plen = [L]
        for j, pl in enumerate(plen):
            while True:
                r = int(rng.integers(0, len(refs)))
                if rlen[r] >= pl + 2:
                    break
            p = int(rng.integers(0, rlen[r] - pl + 1))
            parts.append(refs.seq(r)[p : p + pl].copy())
            if j == 0:
                truth[i] = r
        s = np.concatenate(parts)
        if rng.random() < 0.5:
            s = revcomp(s)
        _substitute(rng, s, sub)
        s = _indels(rng, s, indel)
        seqs.append(s)
    for i in range(n_unrelated):
        seqs.append(_bases(rng, int(lens[n_related + i]), unrelated_gc))
    order = np.arange(n)
    offs = np.zeros(n + 1, dtype=np.uint64)
    offs[1:] = np.cumsum([len(s) for s in seqs])
    data = np.concatenate(seqs) if seqs else np.zeros(0, np.uint8)
    return SeqSet(data, offs, [b"read%d" % i for i in order]), truth


def _fast_fixed_reads(refs: SeqSet, n_related: int, n_unrelated: int, L: int, rng, sub: float):
    """Vectorised fixed-length reads with substitutions only (plain and repeats workloads)."""
    rlen = refs.lengths().astype(np.int64)
    ok = np.flatnonzero(rlen >= L + 2)
    r = ok[rng.integers(0, len(ok), size=n_related)]
    p = (rng.random(n_related) * (rlen[r] - L + 1)).astype(np.int64)
    start = refs.offs[r].astype(np.int64) + p
    rel = np.empty((n_related, L), np.uint8)
    for c in range(0, n_related, 1 << 20):  # gathered in row blocks (no n x L index matrix)
        rel[c : c + (1 << 20)] = refs.data[start[c : c + (1 << 20), None] + np.arange(L)[None, :]]
    flip = rng.random(n_related) < 0.5
    fi = np.flatnonzero(flip)
    for c in range(0, len(fi), 1 << 20):
        rows = fi[c : c + (1 << 20)]
        rel[rows] = _COMP[rel[rows][:, ::-1]]
    flat = rel.reshape(-1)
    _substitute(rng, flat, sub)
    unrel = ACGT[rng.integers(0, 4, size=n_unrelated * L).astype(np.uint8)]
    data = np.concatenate([flat, unrel])
    n = n_related + n_unrelated
    offs = np.arange(n + 1, dtype=np.uint64) * np.uint64(L)
    truth = np.concatenate([r, np.full(n_unrelated, -1)])
    return SeqSet(data, offs, [b"read%d" % i for i in range(n)]), truth


def _fast_variable_reads(refs: SeqSet, n_related: int, n_unrelated: int, lo: int, hi: int, rng, sub: float,
                         indel: float):
    """Vectorised reads of uniform length in [lo, hi] with substitutions and single-base
    indels (half insertions of a uniform base, half deletions), random reference, position and
    strand; then uniform unrelated reads."""
    n = n_related + n_unrelated
    lens = rng.integers(lo, hi + 1, size=n).astype(np.int64)
    W = hi + 4
    rlen = refs.lengths().astype(np.int64)
    ok = np.flatnonzero(rlen >= W + 2)
    r = ok[rng.integers(0, len(ok), size=n_related)]
    p = (rng.random(n_related) * (rlen[r] - W + 1)).astype(np.int64)
    start = refs.offs[r].astype(np.int64) + p
    mat = refs.data[start[:, None] + np.arange(W)[None, :]]
    # substitutions over the whole source window (what falls past the read end is dropped)
    flat = mat.reshape(-1)
    _substitute(rng, flat, sub)
    # indels: per read a binomial count; applied row by row only where there are any
    n_ev = rng.binomial(lens[:n_related], indel)
    for i in np.flatnonzero(n_ev):
        row = mat[i]
        L = int(lens[i])
        pos = np.sort(rng.integers(0, L, size=int(n_ev[i])))
        ins = rng.random(len(pos)) < 0.5
        s = row
        for q, is_ins in zip(pos[::-1], ins[::-1]):
            if is_ins:
                s = np.concatenate([s[:q], ACGT[rng.integers(0, 4, size=1)], s[q:]])
            else:
                s = np.concatenate([s[:q], s[q + 1 :]])
        mat[i] = s[:W] if len(s) >= W else np.concatenate([s, row[len(s) - W :]])[:W]
    # strand: reverse-complement the read part of half the rows
    flip = rng.random(n_related) < 0.5
    fi = np.flatnonzero(flip)
    if len(fi):
        Lf = lens[fi]
        idx = np.clip(Lf[:, None] - 1 - np.arange(W)[None, :], 0, W - 1)
        mat[fi] = _COMP[np.take_along_axis(mat[fi], idx, axis=1)]
    valid = np.arange(W)[None, :] < lens[:n_related, None]
    rel = mat[valid]
    unrel = ACGT[rng.integers(0, 4, size=int(lens[n_related:].sum())).astype(np.uint8)]
    data = np.concatenate([rel, unrel])
    offs = np.zeros(n + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(lens)
    truth = np.concatenate([r, np.full(n_unrelated, -1)])
    return SeqSet(data, offs, [b"read%d" % i for i in range(n)]), truth


def _fast_long_reads(refs: SeqSet, n: int, rng, sub: float, indel: float, chimera_frac: float,
                     median: int = 5000, sigma: float = 0.8, lo: int = 1000, hi: int = 20000, chunk: int = 4096):
    """Vectorised long reads: log-normal lengths clipped to [lo, hi]; a chimera fraction joins
    two references at a uniform breakpoint; single-base indels at rate `indel` (half
    insertions of a uniform base, half deletions), then substitutions at rate `sub` of the
    read's bases, then the reverse complement of half the reads. Returns the reads and the
    reference of each read's first part."""
    lens = _lognormal_lengths(rng, n, median, sigma, lo=lo, hi=hi)
    rlen = refs.lengths().astype(np.int64)
    roffs = refs.offs.astype(np.int64)
    truth = np.empty(n, np.int64)
    out_offs = np.zeros(n + 1, np.uint64)
    out_offs[1:] = np.cumsum(lens)
    data = np.empty(int(out_offs[-1]), np.uint8)
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        m = c1 - c0
        L = lens[c0:c1]
        W = int(L.max()) + int(4 * indel * L.max()) + 64  # source window: the read plus its deletions
        chim = rng.random(m) < chimera_frac
        cut = np.where(chim, (rng.random(m) * (L - 1)).astype(np.int64) + 1, L)  # bases from the first part
        need_a = np.where(chim, cut + 64, W)
        ra = np.empty(m, np.int64)
        rb = np.empty(m, np.int64)
        for dst, need in ((ra, need_a), (rb, np.where(chim, W, 0))):
            pick = rng.integers(0, len(refs), size=m)
            bad = rlen[pick] < need + 2
            while bad.any():
                pick[bad] = rng.integers(0, len(refs), size=int(bad.sum()))
                bad = rlen[pick] < need + 2
            dst[:] = pick
        pa = (rng.random(m) * (rlen[ra] - need_a - 1)).astype(np.int64)
        pb = (rng.random(m) * np.maximum(rlen[rb] - W - 1, 1)).astype(np.int64)
        q = np.arange(W)[None, :]
        src = np.where(q < cut[:, None], roffs[ra][:, None] + pa[:, None] + q,
                       roffs[rb][:, None] + pb[:, None] + (q - cut[:, None]))
        srcb = refs.data[src]
        # indel events per output position: insertion or deletion, each at rate indel / 2
        ev = rng.random((m, W))
        valid = q < L[:, None]
        ins = (ev < indel / 2) & valid
        dele = (ev >= indel / 2) & (ev < indel) & valid
        # source index of output j: j - insertions before j + deletions up to and including j
        sidx = np.clip(q - (np.cumsum(ins, axis=1) - ins) + np.cumsum(dele, axis=1), 0, W - 1)
        read = np.take_along_axis(srcb, sidx, axis=1)
        read[ins] = ACGT[rng.integers(0, 4, size=int(ins.sum())).astype(np.uint8)]
        flat = read[valid]
        _substitute(rng, flat, sub)
        starts = out_offs[c0:c1].astype(np.int64) - int(out_offs[c0])
        for i in np.flatnonzero(rng.random(m) < 0.5):  # reverse complement of half the reads
            a, b = int(starts[i]), int(starts[i] + L[i])
            flat[a:b] = _COMP[flat[a:b][::-1]]
        data[int(out_offs[c0]) : int(out_offs[c1])] = flat
        truth[c0:c1] = ra
    return SeqSet(data, out_offs, [b"read%d" % i for i in range(n)]), truth


def workload(name: str, scale: float = 1.0, seed: int = 1, n_reads: int | None = None,
             reads_seed: int | None = None, refs: SeqSet | None = None):
    """Return (references, reads, truth) for a named workload. With reads_seed the reads come
    from their own generator (so several read sets can share one reference set, which `refs`
    may pass in already generated)."""
    rng = np.random.default_rng(seed)
    if name == "long_fast":
        n_refs = max(4, int(round(5000 * scale)))
        if refs is None:
            total = 344e6 * n_refs / 5000
            lens = _lognormal_lengths(rng, n_refs, 50_000, 0.8, lo=1000, total=total, tol=0.1)
            refs = make_references(n_refs, lens, rng.uniform(0.3, 0.7, size=n_refs), rng)
        rr = np.random.default_rng(reads_seed if reads_seed is not None else seed + 1_000_003)
        nr = n_reads if n_reads is not None else int(round(100_000 * scale))
        reads, truth = _fast_long_reads(refs, nr, rr, 0.03, 0.02, 0.1)
        return refs, reads, truth
    if name == "uneven_fast":
        n_refs = max(4, int(round(5000 * scale)))
        if refs is None:
            total = 344e6 * n_refs / 5000
            lens = _lognormal_lengths(rng, n_refs, 50_000, 0.8, lo=1000, total=total, tol=0.1)
            refs = make_references(n_refs, lens, rng.uniform(0.3, 0.7, size=n_refs), rng)
        rr = np.random.default_rng(reads_seed if reads_seed is not None else seed + 1_000_003)
        nr = n_reads if n_reads is not None else int(round(1_000_000 * scale))
        n_unrel = nr // 5
        reads, truth = _fast_variable_reads(refs, nr - n_unrel, n_unrel, 75, 300, rr, 0.005, 0.001)
        return refs, reads, truth
    if name == "plain":
        n_refs = max(2, int(round(200 * min(1.0, scale * 4))))
        refs = make_references(n_refs, np.full(n_refs, 5000), np.full(n_refs, 0.5), rng)
        nr = n_reads if n_reads is not None else int(round(11000 * scale))
        n_unrel = nr // 11
        reads, truth = _fast_fixed_reads(refs, nr - n_unrel, n_unrel, 150, rng, 0.01)
        return refs, reads, truth
    if name in ("uneven", "long"):
        n_refs = max(4, int(round(5000 * scale)))
        total = 344e6 * n_refs / 5000
        lens = _lognormal_lengths(rng, n_refs, 50_000, 0.8, lo=1000, total=total, tol=0.1)
        refs = make_references(n_refs, lens, rng.uniform(0.3, 0.7, size=n_refs), rng)
        if name == "uneven":
            nr = n_reads if n_reads is not None else int(round(1_000_000 * scale))
            n_unrel = nr // 5
            reads, truth = make_reads(refs, nr - n_unrel, n_unrel,
                                      lambda n: rng.integers(75, 301, size=n), rng,
                                      sub=0.005, indel=0.001)
        else:
            nr = n_reads if n_reads is not None else int(round(100_000 * scale))
            reads, truth = make_reads(refs, nr, 0,
                                      lambda n: _lognormal_lengths(rng, n, 5000, 0.8, lo=1000, hi=20000),
                                      rng, sub=0.03, indel=0.02, chimera_frac=0.1)
        return refs, reads, truth
    if name == "ultralong":
        # reads past 65,535 bases (the oversize tier): references of 270 kb and more, reads of
        # 66-250 kb with 3% substitutions, 2% indels and chimeras, one unrelated read, and a few
        # short reads beside them in the batch
        n_refs = max(4, int(round(16 * scale)))
        lens = _lognormal_lengths(rng, n_refs, 400_000, 0.3, lo=270_000)
        refs = make_references(n_refs, lens, rng.uniform(0.35, 0.65, size=n_refs), rng)
        nr = n_reads if n_reads is not None else int(round(12 * scale))
        n_short = nr // 4
        n_unrel = 1 if nr >= 4 else 0
        long_reads, truth = make_reads(refs, nr - n_short - n_unrel, n_unrel,
                                       lambda n: rng.integers(66_000, 250_001, size=n), rng,
                                       sub=0.03, indel=0.02, chimera_frac=0.25)
        short_reads, t2 = make_reads(refs, n_short, 0, lambda n: rng.integers(150, 20_001, size=n), rng,
                                     sub=0.01, indel=0.005)
        seqs = [long_reads.seq(i) for i in range(len(long_reads))] + [short_reads.seq(i) for i in range(len(short_reads))]
        offs = np.zeros(len(seqs) + 1, dtype=np.uint64)
        offs[1:] = np.cumsum([len(x) for x in seqs])
        reads = SeqSet(np.concatenate(seqs), offs, [b"read%d" % i for i in range(len(seqs))])
        return refs, reads, np.concatenate([truth, t2])
    if name == "repeats":
        n_refs = max(4, int(round(20_000 * scale)))
        lens = _lognormal_lengths(rng, n_refs, 80_000, 0.67, lo=6000)
        refs = make_references(n_refs, lens, np.full(n_refs, 0.5), rng)
        pool_n = max(4, int(round(1000 * min(1.0, scale * 10))))
        pool_len = rng.integers(500, 5001, size=pool_n)
        pool = [_bases(rng, int(x)) for x in pool_len]
        for i in range(n_refs):
            want = int(0.05 * lens[i])
            done = 0
            while done < want:
                seg = pool[int(rng.integers(0, pool_n))]
                if len(seg) >= lens[i]:
                    break
                p = int(rng.integers(0, lens[i] - len(seg) + 1))
                a = int(refs.offs[i]) + p
                refs.data[a : a + len(seg)] = seg
                done += len(seg)
        nr = n_reads if n_reads is not None else int(round(10_000_000 * scale))
        reads, truth = _fast_fixed_reads(refs, nr, 0, 250, rng, 0.01)
        return refs, reads, truth
    raise ValueError(f"unknown workload {name!r}")
