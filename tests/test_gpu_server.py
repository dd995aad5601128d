"""Serving loop (rb_server_*): every job's FASTA is the same alone and in the
mix (with the shared consensus and alignment kernels, jobs admitted while
they run; with per-job kernels; and with jobs whose spans exceed the shared
alignment kernel's scratch), admission by footprint serialises jobs under a
small budget, and a bad job fails alone without stopping the server."""
import time

import pytest

from conftest import lambda_path

pytestmark = pytest.mark.gpu

# four of racon's golden jobs that share -m 5 -x -4 -g -8 -w 500
JOBS = [
    ("sample_reads.fastq.gz", "sample_overlaps.paf.gz"),
    ("sample_reads.fasta.gz", "sample_overlaps.paf.gz"),
    ("sample_reads.fastq.gz", "sample_overlaps.sam.gz"),
    ("sample_reads.fasta.gz", "sample_overlaps.sam.gz"),
]
TARGET = "sample_layout.fasta.gz"


def _alone(native_lib):
    return [native_lib.polish_files(lambda_path(r), lambda_path(o), lambda_path(TARGET), match=5, mismatch=-4,
                                    gap=-8) for r, o in JOBS]


def test_server_mix_matches_alone(native_lib):
    want = _alone(native_lib)
    with native_lib.Server(0, workers=3, match=5, mismatch=-4, gap=-8, window_length=500) as srv:
        tickets = [srv.submit(lambda_path(r), lambda_path(o), lambda_path(TARGET)) for r, o in JOBS * 2]
        got = [srv.wait(t) for t in tickets]
    for i, (fasta, times) in enumerate(got):
        assert fasta == want[i % len(JOBS)], "job %d differs in the mix" % i
        assert times["submitted"] <= times["admitted"] <= times["finished"]
    # with 3 workers, some jobs overlapped in time
    spans = sorted((t["admitted"], t["finished"]) for _, t in got)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))


def test_server_budget_serialises(native_lib):
    want = _alone(native_lib)[:2]
    # a 1-byte budget admits one job at a time (a job alone always starts)
    with native_lib.Server(0, workers=2, hbm_budget=1, match=5, mismatch=-4, gap=-8) as srv:
        tickets = [srv.submit(lambda_path(r), lambda_path(o), lambda_path(TARGET)) for r, o in JOBS[:2] * 2]
        got = [srv.wait(t) for t in tickets]
    for i, (fasta, _) in enumerate(got):
        assert fasta == want[i % 2]
    spans = sorted((t["admitted"], t["finished"]) for _, t in got)
    assert all(spans[i + 1][0] >= spans[i][1] for i in range(len(spans) - 1))


def test_server_bad_job_fails_alone(native_lib):
    want = _alone(native_lib)[0]
    with native_lib.Server(0, workers=2, match=5, mismatch=-4, gap=-8) as srv:
        bad = srv.submit(lambda_path("sample_reads.fastq.gz"), "/nonexistent/overlaps.txt", lambda_path(TARGET))
        good = srv.submit(lambda_path(JOBS[0][0]), lambda_path(JOBS[0][1]), lambda_path(TARGET))
        with pytest.raises(native_lib.RaconB200Error, match="unsupported format extension"):
            srv.wait(bad)
        assert srv.wait(good)[0] == want


def test_server_jobs_join_running_kernel(native_lib, tmp_path):
    """Continuous batching: a long job keeps the shared consensus kernel busy
    while small jobs arrive one by one; each small job's windows join the
    running kernel (through the first, smallest-jobs ring) and every output
    equals the job run alone, including the long one."""
    from racon_b200 import synthetic
    r, o, t, _ = synthetic.contig(str(tmp_path / "big"), 1, scale=0.08)
    big_alone = native_lib.polish_files(r, o, t, match=5, mismatch=-4, gap=-8)
    want = _alone(native_lib)
    with native_lib.Server(0, workers=4, match=5, mismatch=-4, gap=-8, window_length=500,
                           priority_windows=120) as srv:
        tb = srv.submit(r, o, t)
        small = []
        for i, (rr, oo) in enumerate(JOBS * 2):
            time.sleep(0.05)
            small.append(srv.submit(lambda_path(rr), lambda_path(oo), lambda_path(TARGET)))
        got_small = [srv.wait(x) for x in small]
        got_big = srv.wait(tb)
    assert got_big[0] == big_alone
    for i, (fasta, _) in enumerate(got_small):
        assert fasta == want[i % len(JOBS)], "small job %d differs in the mix" % i


def test_server_private_kernels_match(native_lib):
    """shared_consensus=False: each job launches its own consensus kernel;
    same outputs."""
    want = _alone(native_lib)
    with native_lib.Server(0, workers=2, match=5, mismatch=-4, gap=-8, shared_consensus=False) as srv:
        tickets = [srv.submit(lambda_path(r), lambda_path(o), lambda_path(TARGET)) for r, o in JOBS]
        got = [srv.wait(x)[0] for x in tickets]
    assert got == want


def test_server_private_alignment_match(native_lib):
    """shared_alignment=False: each job aligns on its own kernels; same
    outputs."""
    want = _alone(native_lib)
    with native_lib.Server(0, workers=3, match=5, mismatch=-4, gap=-8, shared_alignment=False) as srv:
        tickets = [srv.submit(lambda_path(r), lambda_path(o), lambda_path(TARGET)) for r, o in JOBS]
        got = [srv.wait(x)[0] for x in tickets]
    assert got == want


def test_server_alignment_span_fallback(native_lib, tmp_path):
    """A shared alignment kernel sized for 13 kb spans: the lambda jobs'
    overlaps (up to 12016 bases) align through the shared queue, several
    levels of the path recursion deep, and a job with reads up to 30 kb
    aligns on its own kernels; all outputs unchanged."""
    from racon_b200 import synthetic
    shape = dict(synthetic.CONFIGS[0], mean=9_000, sd=5_000, hi=30_000)
    r, o, t, _ = synthetic.contig(str(tmp_path / "long"), 0, scale=0.5, params=shape)
    long_alone = native_lib.polish_files(r, o, t, match=5, mismatch=-4, gap=-8)
    want = _alone(native_lib)
    with native_lib.Server(0, workers=3, match=5, mismatch=-4, gap=-8, alignment_max_span=13_000,
                           priority_pairs=16, alignment_ctas_per_sm=2) as srv:
        tickets = [srv.submit(r, o, t)] + [srv.submit(lambda_path(rr), lambda_path(oo), lambda_path(TARGET))
                                           for rr, oo in JOBS]
        got = [srv.wait(x)[0] for x in tickets]
    assert got[0] == long_alone
    assert got[1:] == want
