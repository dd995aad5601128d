"""Device window consensus vs the oracle, window by window (byte-identical)."""
import random

import pytest

from conftest import lambda_path

pytestmark = pytest.mark.gpu


def _compare(ctx, oracle_lib, wins, match, mismatch, gap, trim=True):
    got = ctx.poa(wins, trim=trim)
    bad = []
    for i, (w, g) in enumerate(zip(wins, got)):
        cons, pol, _ = oracle_lib.window_consensus(w, match, mismatch, gap, trim)
        if (cons, pol) != g:
            bad.append(i)
    assert not bad, "%d of %d windows differ, first %s" % (len(bad), len(wins), bad[:10])


@pytest.mark.parametrize("reads,overlaps,w,m,x,g", [
    ("sample_reads.fastq.gz", "sample_overlaps.paf.gz", 500, 5, -4, -8),
    ("sample_reads.fasta.gz", "sample_overlaps.paf.gz", 500, 5, -4, -8),
    ("sample_reads.fastq.gz", "sample_overlaps.sam.gz", 500, 5, -4, -8),
    ("sample_reads.fastq.gz", "sample_overlaps.paf.gz", 1000, 5, -4, -8),
    ("sample_reads.fastq.gz", "sample_overlaps.paf.gz", 500, 1, -1, -1),
])
def test_lambda_contig_windows(native_lib, oracle_lib, reads, overlaps, w, m, x, g):
    wins = oracle_lib.dump_windows(lambda_path(reads), lambda_path(overlaps), lambda_path("sample_layout.fasta.gz"),
                                   window_length=w)
    with native_lib.Context(0, m, x, g, w) as ctx:
        _compare(ctx, oracle_lib, wins, m, x, g)


def test_lambda_fragment_windows_sample(native_lib, oracle_lib):
    wins = oracle_lib.dump_windows(lambda_path("sample_reads.fasta.gz"), lambda_path("sample_ava_overlaps.paf.gz"),
                                   lambda_path("sample_reads.fasta.gz"), fragment=True)
    wins = wins[::7]
    with native_lib.Context(0, 1, -1, -1, 500) as ctx:
        _compare(ctx, oracle_lib, wins, 1, -1, -1)


def test_small_windows_and_untrimmed(native_lib, oracle_lib):
    rng = random.Random(11)
    wins = []
    for k in range(40):
        bl = rng.randint(2, 60)
        bb = "".join(rng.choice("ACGT") for _ in range(bl))
        nl = rng.randint(0, 6)
        layers, quals, begins, ends = [], [], [], []
        for _ in range(nl):
            b = rng.randint(0, bl - 2)
            e = rng.randint(b + 1, bl - 1)
            s = "".join(rng.choice("ACGT") for _ in range(rng.randint(1, 80)))
            layers.append(s)
            quals.append("".join(chr(33 + rng.randint(0, 40)) for _ in s) if k % 2 else None)
            begins.append(b)
            ends.append(e)
        wins.append({"backbone": bb, "backbone_quality": None if k % 3 else "".join(chr(40 + rng.randint(0, 20)) for _ in bb),
                     "layers": layers, "qualities": quals, "begins": begins, "ends": ends, "tgs": k % 2})
    with native_lib.Context(0, 3, -5, -4, 500) as ctx:
        _compare(ctx, oracle_lib, wins, 3, -5, -4, trim=True)
        _compare(ctx, oracle_lib, wins, 3, -5, -4, trim=False)


def test_stage_run_fetch(native_lib, oracle_lib):
    wins = oracle_lib.dump_windows(lambda_path("sample_reads.fastq.gz"), lambda_path("sample_overlaps.paf.gz"),
                                   lambda_path("sample_layout.fasta.gz"))
    with native_lib.Context(0, 3, -5, -4, 500) as ctx:
        a = ctx.poa(wins)
        ctx.poa_stage(wins)
        ctx.poa_run()
        ctx.poa_run()
        assert ctx.poa_fetch() == a
        # plain comparison form: same results
        ctx.poa_run(plain=True)
        assert ctx.poa_fetch() == a
        assert ctx.poa_stats().launches >= 1
