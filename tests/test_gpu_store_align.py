"""Overlap alignment from the device sequence table (rb_align_stage_overlaps)
and the fused alignment + layer staging (rb_poa_stage_alignments) against
the host-buffer forms they replace.

rb_align_batch is pinned to the oracle's edlib restatement by the alignment
parity tests; here the same spans cut on the device (forward and reverse
complement, as src/overlap.cpp:193-197 cuts them) must give the same edit
distances, CIGARs and breaking points, and the fused call must stage the same
windows as aligning first and assembling from the host breaking points.
"""
import random

import pytest

from racon_b200 import RaconB200Error

pytestmark = pytest.mark.gpu

COMP = {"A": "T", "T": "A", "C": "G", "G": "C"}


def _revcomp(s):
    return "".join(COMP.get(c, c) for c in reversed(s))


def _mutate(rng, s, err):
    out = []
    for c in s:
        u = rng.random()
        if u < err / 3:
            continue
        out.append(rng.choice("ACGT") if u < 2 * err / 3 else c)
        if rng.random() < err / 3:
            out.append(rng.choice("ACGT"))
    return "".join(out)


def _world(seed, n_reads=40, tlen=6000, alphabet="ACGT"):
    """Targets, reads sampled from them (both strands, FASTQ-like
    qualities), and racon-style overlap records."""
    rng = random.Random(seed)
    targets = ["".join(rng.choice(alphabet) for _ in range(tlen)), "".join(rng.choice(alphabet) for _ in range(2500))]
    seqs = [{"data": t, "quality": bytes(33 + rng.randint(5, 30) for _ in t), "forward": 1, "reverse": 0}
            for t in targets]
    pairs = []
    for k in range(n_reads):
        t_id = k % 2
        T = targets[t_id]
        tb = rng.randint(0, len(T) - 300)
        te = min(len(T), tb + rng.randint(200, 3000))
        core = _mutate(rng, T[tb:te], 0.12)
        pre = "".join(rng.choice("ACGT") for _ in range(rng.randint(0, 40)))
        post = "".join(rng.choice("ACGT") for _ in range(rng.randint(0, 40)))
        oriented = pre + core + post
        strand = k % 3 == 1
        data = _revcomp(oriented) if strand else oriented
        L = len(data)
        # forward read coordinates of the aligned core
        qb, qe = (len(post), L - len(pre)) if strand else (len(pre), len(pre) + len(core))
        seqs.append({"data": data, "quality": bytes(33 + rng.randint(5, 30) for _ in data),
                     "forward": 0 if strand else 1, "reverse": 1 if strand else 0})
        pairs.append({"q_id": len(seqs) - 1, "q_begin": qb, "q_end": qe, "t_id": t_id, "t_begin": tb,
                      "t_end": te, "strand": int(strand)})
    return seqs, pairs


def _host_pairs(seqs, pairs):
    out = []
    for p in pairs:
        d = seqs[p["q_id"]]["data"]
        L = len(d)
        if p["strand"]:
            q = _revcomp(d)[L - p["q_end"]:L - p["q_begin"]]
            q_offset = L - p["q_end"]
        else:
            q = d[p["q_begin"]:p["q_end"]]
            q_offset = p["q_begin"]
        t = seqs[p["t_id"]]["data"][p["t_begin"]:p["t_end"]]
        out.append({"query": q, "target": t, "q_offset": q_offset, "t_begin": p["t_begin"]})
    return out


@pytest.mark.parametrize("seed", [1, 2])
def test_store_alignment_matches_host_pairs(native_lib, seed):
    seqs, pairs = _world(seed)
    # edge spans: empty query, empty target, bytes beyond ACGT
    seqs.append({"data": "NNACGTNNRYACGT" * 20, "quality": None, "forward": 1, "reverse": 1})
    n_id = len(seqs) - 1
    pairs += [
        {"q_id": 2, "q_begin": 5, "q_end": 5, "t_id": 0, "t_begin": 100, "t_end": 180, "strand": 0},
        {"q_id": 2, "q_begin": 0, "q_end": 30, "t_id": 0, "t_begin": 700, "t_end": 700, "strand": 0},
        {"q_id": n_id, "q_begin": 3, "q_end": 250, "t_id": 1, "t_begin": 10, "t_end": 260, "strand": 1},
        {"q_id": n_id, "q_begin": 0, "q_end": 280, "t_id": n_id, "t_begin": 0, "t_end": 280, "strand": 0},
    ]
    with native_lib.Context(0, 3, -5, -4, 500) as ctx:
        want = ctx.align(_host_pairs(seqs, pairs), want_cigar=True)
        ctx.sequences_stage(seqs)
        got = ctx.align_overlaps(pairs, want_cigar=True)
        assert got == want
        got = ctx.align_overlaps(pairs, want_cigar=False)
        assert [g["edit_distance"] for g in got] == [w["edit_distance"] for w in want]
        assert [g["breakpoints"] for g in got] == [w["breakpoints"] for w in want]


def test_store_alignment_errors(native_lib):
    seqs, pairs = _world(3, n_reads=4)
    rng = random.Random(5)
    seqs.append({"data": "".join(chr(rng.randint(65, 120)) for _ in range(300)), "quality": None, "forward": 1,
                 "reverse": 0})
    many = len(seqs) - 1
    with native_lib.Context(0, 3, -5, -4, 500) as ctx:
        ctx.sequences_stage(seqs)
        cases = [
            ({"q_id": 99, "q_begin": 0, "q_end": 1, "t_id": 0, "t_begin": 0, "t_end": 1, "strand": 0}, "id"),
            ({"q_id": 2, "q_begin": 0, "q_end": 10**6, "t_id": 0, "t_begin": 0, "t_end": 1, "strand": 0}, "outside"),
            # pair 0's read is staged for its own strand only
            (dict(pairs[0], strand=1 - pairs[0]["strand"]), "strand"),
        ]
        for bad, word in cases:
            with pytest.raises(RaconB200Error) as e:
                ctx.align_overlaps(pairs[:2] + [bad])
            assert word in str(e.value)
        assert ctx.align_overlaps(pairs) == ctx.align(_host_pairs(seqs, pairs))
        # a pair of more than 32 distinct bytes is aligned, not refused (the
        # device codes any byte alphabet), the same as from host buffers
        wide = pairs[:2] + [{"q_id": many, "q_begin": 0, "q_end": 300, "t_id": 0, "t_begin": 0, "t_end": 300,
                             "strand": 0}]
        assert ctx.align_overlaps(wide) == ctx.align(_host_pairs(seqs, wide))


@pytest.mark.parametrize("seed", [4, 6])
def test_fused_staging_matches_two_steps(native_lib, seed):
    seqs, pairs = _world(seed, n_reads=60)
    with native_lib.Context(0, 3, -5, -4, 500) as ctx:
        ctx.sequences_stage(seqs)
        aln = ctx.align_overlaps(pairs, want_cigar=False)
        overlaps = [{"q_id": p["q_id"], "t_id": p["t_id"], "strand": p["strand"], "breakpoints": a["breakpoints"]}
                    for p, a in zip(pairs, aln)]
        ctx.poa_stage_overlaps(2, overlaps, quality_threshold=10.0, tgs=True)
        ctx.poa_run()
        want = ctx.poa_fetch()
        got_aln = ctx.poa_stage_alignments(2, pairs, quality_threshold=10.0, tgs=True)
        assert got_aln == [(a["edit_distance"], a["breakpoints"]) for a in aln]
        ctx.poa_run()
        assert ctx.poa_fetch() == want
        assert any(c != "" for c, _ in want)


def test_fused_staging_in_many_alignment_batches(native_lib, monkeypatch):
    # the aligner runs in batches bounded by bases; every batch's breaking
    # points go to the layer candidates in overlap order
    seqs, pairs = _world(8, n_reads=50)
    with native_lib.Context(0, 3, -5, -4, 500) as ctx:
        ctx.sequences_stage(seqs)
        want_aln = ctx.poa_stage_alignments(2, pairs, quality_threshold=10.0, tgs=True)
        ctx.poa_run()
        want = ctx.poa_fetch()
        monkeypatch.setenv("RB_ALIGN_BATCH_BASES", "6000")
        got_aln = ctx.poa_stage_alignments(2, pairs, quality_threshold=10.0, tgs=True)
        ctx.poa_run()
        got = ctx.poa_fetch()
        assert ctx.layer_stats().launches > 20  # one candidates launch per batch
    assert got_aln == want_aln
    assert got == want
