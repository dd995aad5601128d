"""Scheduling knobs of a context (rb_set_yield, rb_set_priority,
rb_set_sm_share) leave every result unchanged: bounded work per warp and
launch, with as many launches back to back as the queue needs, the
high-priority stream, and persistent kernels on part of the SMs."""
import pytest

from racon_b200 import synthetic

pytestmark = pytest.mark.gpu


def test_yield_and_priority_keep_results(native_lib, tmp_path, monkeypatch):
    r, o, t, _ = synthetic.contig(str(tmp_path), 0)
    job = native_lib.Job(r, o, t, window_length=500, match=3, mismatch=-5, gap=-4)
    # more pairs than resident alignment warps (148 SMs x 16), so a cap of 1
    # needs several launches of the distance and level kernels
    pairs = synthetic.pairs(3000, 300, 1500, seed=5)
    # 16 resident consensus warps for the job's windows: several launches
    monkeypatch.setenv("RB_POA_SLOTS", "16")
    try:
        with native_lib.Context(0, 3, -5, -4, 500) as ctx:
            want_aln = ctx.align(pairs, want_cigar=True)
            base_aln_launches = ctx.align_stats().launches
            ctx.poa_stage_job(job)
            ctx.poa_run()
            want = ctx.poa_fetch()
            assert ctx.poa_stats().launches == 1

            ctx.set_yield(1, 1)
            assert ctx.align(pairs, want_cigar=True) == want_aln
            assert ctx.align_stats().launches > base_aln_launches
            ctx.poa_run()
            assert ctx.poa_fetch() == want
            assert ctx.poa_stats().launches == -(-job.n // 16)

            ctx.set_priority(True)
            ctx.poa_stage_job_device(job)
            ctx.poa_run()
            assert ctx.poa_fetch() == want
            assert ctx.align(pairs, want_cigar=False)[7]["breakpoints"] == want_aln[7]["breakpoints"]

            ctx.set_sm_share(40)
            assert ctx.align(pairs, want_cigar=True) == want_aln
            ctx.poa_run()
            assert ctx.poa_fetch() == want

            ctx.set_sm_share(100)
            ctx.set_priority(False)
            ctx.set_yield(0, 0)
            ctx.poa_run()
            assert ctx.poa_fetch() == want
            assert ctx.poa_stats().launches == 1
    finally:
        job.close()
