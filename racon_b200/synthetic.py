"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No public dataset is named for racon's throughput, so every workload is
generated here from a fixed seed (numpy PCG64, seed = configuration index
unless given):

  contig(...)   polishing job: uniform-ACGT truth genome, draft = truth with
                errors, reads sampled from the truth with errors, half reverse
                complemented, PAF overlaps written from the known sampling
                coordinates mapped onto the draft (optional end jitter).
                config 0: 50 kb, 30x, log-normal(5 kb, 2 kb) in [500, 20k],
                          5% sub + 4% ins + 4% del, FASTA reads.
                config 1: 1 Mb, 50x, log-normal(8 kb, 4 kb) in [1k, 50k],
                          6% sub + 3% ins + 3% del, FASTQ Phred U[5, 30],
                          PAF ends jittered by +-50 bp.
  pairs(...)    overlap-alignment batch (config 2): target spans U[lo, hi],
                query = span mutated at 7% sub + 4% ins + 4% del, half reverse
                complemented (the query is given in the orientation racon
                aligns, so the pair itself is forward).
  serving_jobs(...) config 4 job stream: config-0-like jobs with log-uniform
                contig length, uniform coverage and error.
  fragment(...) read correction (config 3 shape, scaled): contigs, reads at a
                sinusoidal local depth, all-vs-all PAF overlaps (dual
                directions) from the known coordinates.
"""
import os

import numpy as np

BASES = np.frombuffer(b"ACGT", dtype=np.uint8)
_COMP = np.zeros(256, dtype=np.uint8)
for a, b in zip(b"ACGTN", b"TGCAN"):
    _COMP[a] = b


def revcomp(s):
    return _COMP[np.frombuffer(s, dtype=np.uint8)[::-1]].tobytes()


def mutate(rng, seq, p_sub, p_ins, p_del):
    """seq: uint8 codes 0..3. Returns (mutated codes, map) where map[i] is the
    output position of input base i (or of its successor when deleted),
    map[len(seq)] = output length."""
    n = len(seq)
    u = rng.random(n)
    dele = u < p_del
    sub = (u >= p_del) & (u < p_del + p_sub)
    ins = rng.random(n) < p_ins
    keep = ~dele
    k = keep.astype(np.int64) + ins.astype(np.int64)
    ends = np.cumsum(k)
    starts = ends - k
    total = int(ends[-1]) if n else 0
    out = np.empty(total, dtype=np.uint8)
    base = seq.copy()
    base[sub] = (seq[sub] + rng.integers(1, 4, int(sub.sum()), dtype=np.uint8)) % 4
    out[starts[keep]] = base[keep]
    ins_pos = starts[ins] + keep[ins]
    out[ins_pos] = rng.integers(0, 4, len(ins_pos), dtype=np.uint8)
    mp = np.empty(n + 1, dtype=np.int64)
    mp[:n] = starts
    mp[n] = total
    return out, mp


def _lognormal_lengths(rng, count, mean, sd, lo, hi):
    s2 = np.log(1 + (sd / mean) ** 2)
    mu = np.log(mean) - s2 / 2
    return np.clip(rng.lognormal(mu, np.sqrt(s2), count), lo, hi).astype(np.int64)


CONFIGS = {
    0: dict(genome=50_000, coverage=30, mean=5_000, sd=2_000, lo=500, hi=20_000,
            read_err=(0.05, 0.04, 0.04), fastq=False, jitter=0),
    1: dict(genome=1_000_000, coverage=50, mean=8_000, sd=4_000, lo=1_000, hi=50_000,
            read_err=(0.06, 0.03, 0.03), fastq=True, jitter=50),
}


def contig(out_dir, config=1, seed=None, scale=1.0, qual_range=(5, 30), params=None):
    """Writes reads (FASTA/FASTQ), overlaps (PAF) and the draft (FASTA) of a
    contig-polishing job; returns the three paths and a summary dict.
    params (optional) replaces the configuration's shape dict."""
    c = dict(CONFIGS[config] if params is None else params)
    rng = np.random.default_rng(config if seed is None else seed)
    g = max(2_000, int(c["genome"] * scale))
    truth = rng.integers(0, 4, g, dtype=np.uint8)
    draft, dmap = mutate(rng, truth, 0.01 / 3, 0.01 / 3, 0.01 / 3)
    n_reads = max(4, int(round(c["coverage"] * g / c["mean"])))
    lens = np.minimum(_lognormal_lengths(rng, n_reads, c["mean"], c["sd"], c["lo"], c["hi"]), g)
    starts = rng.integers(0, np.maximum(1, g - lens + 1))
    strands = rng.random(n_reads) < 0.5
    os.makedirs(out_dir, exist_ok=True)
    ext = "fastq" if c["fastq"] else "fasta"
    rpath = os.path.join(out_dir, "reads.%s" % ext)
    opath = os.path.join(out_dir, "overlaps.paf")
    tpath = os.path.join(out_dir, "draft.fasta")
    dlen = len(draft)
    sub, ins, dele = c["read_err"]
    with open(rpath, "wb") as rf, open(opath, "w") as of:
        for i in range(n_reads):
            s, e = int(starts[i]), int(starts[i] + lens[i])
            r, _ = mutate(rng, truth[s:e], sub, ins, dele)
            if len(r) == 0:
                continue
            rb = BASES[r].tobytes()
            if strands[i]:
                rb = revcomp(rb)
            name = "read%d" % i
            if c["fastq"]:
                q = (rng.integers(qual_range[0], qual_range[1] + 1, len(rb)) + 33).astype(np.uint8).tobytes()
                rf.write(b"@" + name.encode() + b"\n" + rb + b"\n+\n" + q + b"\n")
            else:
                rf.write(b">" + name.encode() + b"\n" + rb + b"\n")
            tb, te = int(dmap[s]), int(dmap[e])
            qb, qe = 0, len(rb)
            if c["jitter"]:
                j = c["jitter"]
                tb = int(np.clip(tb + rng.integers(-j, j + 1), 0, dlen - 1))
                te = int(np.clip(te + rng.integers(-j, j + 1), tb + 1, dlen))
                qb = int(np.clip(qb + rng.integers(0, j + 1), 0, len(rb) - 1))
                qe = int(np.clip(qe - rng.integers(0, j + 1), qb + 1, len(rb)))
            span = max(qe - qb, te - tb)
            of.write("%s\t%d\t%d\t%d\t%s\tdraft\t%d\t%d\t%d\t%d\t%d\t60\n" % (
                name, len(rb), qb, qe, "-" if strands[i] else "+", dlen, tb, te, min(qe - qb, te - tb), span))
    with open(tpath, "wb") as tf:
        tf.write(b">draft\n" + BASES[draft].tobytes() + b"\n")
    info = {"config": config, "genome": g, "reads": int(n_reads), "draft_length": dlen}
    return rpath, opath, tpath, info


def serving_jobs(out_dir, count, seed=4, length=(20_000, 2_000_000), coverage=(20, 80), error=(0.08, 0.15)):
    """Config 4 job stream: `count` config-0-like jobs with contig length
    log-uniform in `length`, coverage uniform in `coverage` and read error
    uniform in `error` (split 5:4:4 over sub/ins/del as in config 0). Returns
    a list of (reads, overlaps, draft, info), job i generated from seed
    (seed, i)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(count):
        g = int(np.exp(rng.uniform(np.log(length[0]), np.log(length[1]))))
        cov = float(rng.uniform(*coverage))
        err = float(rng.uniform(*error))
        params = dict(CONFIGS[0])
        params.update(genome=g, coverage=cov, read_err=(err * 5 / 13, err * 4 / 13, err * 4 / 13))
        d = os.path.join(out_dir, "job%03d" % i)
        r, o, t, info = contig(d, 0, seed=int(rng.integers(1 << 31)), params=params)
        info.update(coverage=cov, error=err)
        jobs.append((r, o, t, info))
    return jobs


def pairs(count, lo=1_000, hi=50_000, seed=2, err=(0.07, 0.04, 0.04)):
    """Overlap-alignment pairs (config 2 shape): list of dicts for
    racon_b200.Context.align (query already in the aligned orientation)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(lo, hi + 1))
        t = rng.integers(0, 4, n, dtype=np.uint8)
        q, _ = mutate(rng, t, *err)
        if len(q) == 0:
            q = t[:1]
        # a read sampled from the reverse strand is aligned as its reverse
        # complement, i.e. as a mutated copy of the forward span: both halves
        # give pairs of this form
        qb = BASES[q].tobytes()
        out.append({"query": qb, "target": BASES[t].tobytes(), "q_offset": int(rng.integers(0, 1000)),
                    "t_begin": int(rng.integers(0, 100_000))})
    return out


def fragment(out_dir, genome=200_000, contigs=3, depth=(10, 60), mean=6_000, sd=2_000, err=0.15, seed=3,
             qual_range=(3, 40)):
    """Read-correction job (-f): reads as targets, all-vs-all dual PAF overlaps
    from the known coordinates. Local depth follows a sinusoid in depth."""
    rng = np.random.default_rng(seed)
    os.makedirs(out_dir, exist_ok=True)
    rpath = os.path.join(out_dir, "reads.fastq")
    opath = os.path.join(out_dir, "overlaps.paf")
    sizes = np.full(contigs, genome // contigs)
    reads = []  # (name, contig, start, end, strand, bytes)
    idx = 0
    with open(rpath, "wb") as rf:
        for ci, gs in enumerate(sizes):
            truth = rng.integers(0, 4, int(gs), dtype=np.uint8)
            phase = rng.random() * 2 * np.pi
            pos = 0
            while pos < gs:
                d = depth[0] + (depth[1] - depth[0]) * 0.5 * (1 + np.sin(phase + 2 * np.pi * pos / gs * 3))
                step = max(1, int(mean / d))
                ln = int(np.clip(_lognormal_lengths(rng, 1, mean, sd, 500, 4 * mean)[0], 1, gs))
                s = min(pos, max(0, int(gs) - ln))
                r, _ = mutate(rng, truth[s:s + ln], err / 2, err / 4, err / 4)
                if len(r) >= 2:
                    rb = BASES[r].tobytes()
                    strand = rng.random() < 0.5
                    if strand:
                        rb = revcomp(rb)
                    name = "r%d" % idx
                    idx += 1
                    q = (rng.integers(qual_range[0], qual_range[1] + 1, len(rb)) + 33).astype(np.uint8).tobytes()
                    rf.write(b"@" + name.encode() + b"\n" + rb + b"\n+\n" + q + b"\n")
                    reads.append((name, ci, s, s + ln, strand, len(rb)))
                pos += step
    # all-vs-all overlaps from true coordinates (both directions, no self)
    with open(opath, "w") as of:
        by_contig = {}
        for r in reads:
            by_contig.setdefault(r[1], []).append(r)
        for rs in by_contig.values():
            rs.sort(key=lambda x: x[2])
            for i, a in enumerate(rs):
                for b in rs[i + 1:]:
                    if b[2] >= a[3]:
                        break
                    ov_s, ov_e = max(a[2], b[2]), min(a[3], b[3])
                    if ov_e - ov_s < 500:
                        continue
                    for x, y in ((a, b), (b, a)):
                        # approximate read coordinates by proportional scaling
                        def span(r):
                            f0 = (ov_s - r[2]) / (r[3] - r[2])
                            f1 = (ov_e - r[2]) / (r[3] - r[2])
                            lo_, hi_ = int(f0 * r[5]), max(int(f0 * r[5]) + 1, int(f1 * r[5]))
                            if r[4]:
                                lo_, hi_ = r[5] - hi_, r[5] - lo_
                            return lo_, min(hi_, r[5])
                        qb, qe = span(x)
                        tb, te = span(y)
                        strand = "-" if x[4] != y[4] else "+"
                        of.write("%s\t%d\t%d\t%d\t%s\t%s\t%d\t%d\t%d\t%d\t%d\t60\n" % (
                            x[0], x[5], qb, qe, strand, y[0], y[5], tb, te, min(qe - qb, te - tb),
                            max(qe - qb, te - tb)))
    return rpath, opath, rpath, {"reads": len(reads)}
