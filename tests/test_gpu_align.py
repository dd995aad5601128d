"""Device overlap alignment vs the oracle: edit distance, standard CIGAR and
racon's window breaking points must be identical (integer work: bit-exact)."""
import random

import pytest

from conftest import lambda_path
from seqio import paf_pairs, read_fastx, read_paf

pytestmark = pytest.mark.gpu


def _mutate(rng, s, sub, ins, dele, alpha="ACGT"):
    out = []
    for c in s:
        u = rng.random()
        if u < dele:
            continue
        out.append(rng.choice(alpha) if u < dele + sub else c)
        while rng.random() < ins:
            out.append(rng.choice(alpha))
    return "".join(out)


def _random_pairs(seed, count, lo, hi, err):
    rng = random.Random(seed)
    pairs = []
    for i in range(count):
        n = rng.randint(lo, hi)
        alpha = "ACGTN" if i % 7 == 0 else "ACGT"
        t = "".join(rng.choice(alpha) for _ in range(n))
        q = _mutate(rng, t, err / 2, err / 4, err / 4, alpha)
        if not q:
            q = "A"
        pairs.append({"query": q, "target": t, "q_offset": rng.randint(0, 1000), "t_begin": rng.randint(0, 3000)})
    return pairs


def _check(ctx, oracle_lib, pairs, window_length):
    got = ctx.align(pairs, want_cigar=True)
    bad = 0
    for p, g in zip(pairs, got):
        d, cig = oracle_lib.nw_cigar(p["query"], p["target"])
        exp_bp = oracle_lib.breakpoints(cig, p["q_offset"], p["q_offset"] + len(p["query"]),
                                        p["q_offset"] + len(p["query"]), p["t_begin"],
                                        p["t_begin"] + len(p["target"]), 0, window_length)
        if (g["edit_distance"], g["cigar"], g["breakpoints"]) != (d, cig, exp_bp):
            bad += 1
    assert bad == 0, "%d of %d pairs differ" % (bad, len(pairs))


@pytest.fixture(scope="module")
def ctx(native_lib):
    c = native_lib.Context(0, 3, -5, -4, 500)
    yield c
    c.close()


def test_edge_cases(ctx, oracle_lib):
    pairs = [
        {"query": "A", "target": "A"}, {"query": "A", "target": "C"}, {"query": "AC", "target": "A"},
        {"query": "A", "target": "ACGTACGTAC"}, {"query": "ACGTACGTAC", "target": "G"},
        {"query": "ACGT" * 40, "target": "ACGT" * 40}, {"query": "A" * 70, "target": "C" * 70},
        {"query": "ACGT" * 16, "target": "ACGT" * 16 + "A"}, {"query": "T" * 129, "target": "T" * 64},
        {"query": "GATTACA" * 100, "target": "GATTACA" * 95},
    ]
    for p in pairs:
        p.setdefault("q_offset", 0)
        p.setdefault("t_begin", 0)
    _check(ctx, oracle_lib, pairs, 500)


def test_random_small(ctx, oracle_lib):
    _check(ctx, oracle_lib, _random_pairs(1, 300, 1, 300, 0.15), 500)


def test_random_medium(ctx, oracle_lib):
    _check(ctx, oracle_lib, _random_pairs(2, 120, 300, 4000, 0.15), 500)


def test_random_hirschberg(ctx, oracle_lib):
    # spans above edlib's 1 MiB traceback threshold take the Hirschberg split
    _check(ctx, oracle_lib, _random_pairs(3, 24, 6000, 14000, 0.15), 500)


def test_random_high_divergence(ctx, oracle_lib):
    _check(ctx, oracle_lib, _random_pairs(4, 60, 50, 3000, 0.45), 500)


def test_lambda_paf_overlaps(ctx, oracle_lib):
    reads = read_fastx(lambda_path("sample_reads.fasta.gz"))
    layout = read_fastx(lambda_path("sample_layout.fasta.gz"))
    pairs = paf_pairs(reads, layout, read_paf(lambda_path("sample_overlaps.paf.gz")))
    _check(ctx, oracle_lib, pairs, 500)


def test_lambda_ava_overlaps_sample(ctx, oracle_lib):
    reads = read_fastx(lambda_path("sample_reads.fasta.gz"))
    rows = read_paf(lambda_path("sample_ava_overlaps.paf.gz"))[::16]
    pairs = paf_pairs(reads, reads, rows)
    _check(ctx, oracle_lib, pairs, 500)


def _check_parallel(ctx, oracle_lib, pairs, window_length):
    """_check with the oracle's alignments computed on every host thread."""
    import concurrent.futures
    import os
    got = ctx.align(pairs, want_cigar=True)
    with concurrent.futures.ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        want = list(ex.map(lambda p: oracle_lib.nw_cigar(p["query"], p["target"]), pairs))
    bad = 0
    for p, g, (d, cig) in zip(pairs, got, want):
        exp_bp = oracle_lib.breakpoints(cig, p["q_offset"], p["q_offset"] + len(p["query"]),
                                        p["q_offset"] + len(p["query"]), p["t_begin"],
                                        p["t_begin"] + len(p["target"]), 0, window_length)
        if (g["edit_distance"], g["cigar"], g["breakpoints"]) != (d, cig, exp_bp):
            bad += 1
    assert bad == 0, "%d of %d pairs differ" % (bad, len(pairs))


def test_config2_long_pairs(ctx, oracle_lib):
    # the overlap-alignment batch's longest spans: 30-50 kb targets, query at
    # 7% sub + 4% ins + 4% del (Hirschberg splits many levels deep)
    from racon_b200 import synthetic
    _check_parallel(ctx, oracle_lib, synthetic.pairs(48, 30_000, 50_000, seed=21), 500)


def test_config2_batch_sample(ctx, oracle_lib):
    # 1000 pairs with the batch's full span range, 1-50 kb
    from racon_b200 import synthetic
    _check_parallel(ctx, oracle_lib, synthetic.pairs(1000, 1_000, 50_000, seed=22), 500)


def test_wide_alphabet(ctx, oracle_lib):
    # more than 32 distinct bytes in a pair (IUPAC codes, lowercase, other
    # printable bytes): edlib aligns any byte alphabet, and so must the device
    # (its query masks then live in global scratch instead of shared memory)
    rng = random.Random(11)
    iupac = "ACGTURYKMSWBDHVN"
    wide = iupac + "acgturykmswbdhvn" + "0123456789!#$%&*+-.:;<=>?@"
    pairs = []
    for i, (lo, hi) in enumerate([(1, 80), (200, 2000), (6000, 9000)] * 4):
        alpha = wide if i % 3 else iupac + "xyz*-"
        n = rng.randint(lo, hi)
        t = "".join(rng.choice(alpha) for _ in range(n))
        q = _mutate(rng, t, 0.06, 0.03, 0.03, alpha) or "A"
        pairs.append({"query": q, "target": t, "q_offset": rng.randint(0, 500), "t_begin": rng.randint(0, 2000)})
    assert any(len(set(p["query"] + p["target"])) > 32 for p in pairs)
    _check(ctx, oracle_lib, pairs, 500)


def test_stage_run_fetch_matches_batch(ctx, oracle_lib):
    pairs = _random_pairs(5, 50, 100, 2000, 0.12)
    a = ctx.align(pairs, want_cigar=True)
    ctx.align_stage(pairs, want_cigar=True)
    ctx.align_run()
    ctx.align_run()
    b = ctx.align_fetch()
    assert a == b


def test_sam_cigar_breakpoints(ctx, oracle_lib):
    rng = random.Random(7)
    ovs = []
    for _ in range(200):
        ops = []
        tl = 0
        ql = 0
        if rng.random() < 0.5:
            ops.append("%dS" % rng.randint(1, 50))
        for _ in range(rng.randint(1, 60)):
            k = rng.choice("MMMMID=X")
            n = rng.randint(1, 60)
            ops.append("%d%s" % (n, k))
            if k in "M=XD":
                tl += n
        if rng.random() < 0.5:
            ops.append("%dH" % rng.randint(1, 50))
        cig = "".join(ops)
        tb = rng.randint(0, 5000)
        ovs.append({"cigar": cig, "q_offset": rng.randint(0, 100), "t_begin": tb, "t_end": tb + tl})
    got = ctx.cigar_breakpoints(ovs)
    for o, g in zip(ovs, got):
        # the oracle walks the CIGAR from q_begin (forward strand)
        exp = oracle_lib.breakpoints(o["cigar"], o["q_offset"], o["q_offset"], o["q_offset"], o["t_begin"],
                                     o["t_end"], 0, 500)
        assert g == exp
