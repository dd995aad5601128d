"""Autotuner (rb_autotune / rb_tuning_*): the launch choices it sweeps
(consensus CTAs per SM, queue order, alignment warps per SM) never change a
result, and the sweep keeps the fastest for the device."""
import pytest

from conftest import lambda_path
from seqio import paf_pairs, read_fastx, read_paf

pytestmark = pytest.mark.gpu


@pytest.fixture
def ctx(native_lib):
    before = native_lib.tuning_get(0)
    c = native_lib.Context(0, 5, -4, -8, 500)
    yield c
    c.close()
    native_lib.tuning_set(0, **before)


def _windows(oracle_lib):
    return oracle_lib.dump_windows(lambda_path("sample_reads.fastq.gz"), lambda_path("sample_overlaps.paf.gz"),
                                   lambda_path("sample_layout.fasta.gz"))


def _pairs():
    reads = read_fastx(lambda_path("sample_reads.fasta.gz"))
    rows = read_paf(lambda_path("sample_ava_overlaps.paf.gz"))[::8]
    return paf_pairs(reads, reads, rows)


def test_pinned_settings_give_identical_results(native_lib, oracle_lib, ctx):
    wins = _windows(oracle_lib)
    pairs = _pairs()
    outs = []
    for cps, order, warps in [(3, 0, 16), (1, 1, 8), (2, 1, 32)]:
        native_lib.tuning_set(0, consensus_ctas_per_sm=cps, consensus_order=order, alignment_warps_per_sm=warps)
        t = native_lib.tuning_get(0)
        assert (t["consensus_ctas_per_sm"], t["consensus_order"], t["alignment_warps_per_sm"]) == (cps, order, warps)
        outs.append((ctx.poa(wins), ctx.align(pairs, want_cigar=True)))
    assert all(o == outs[0] for o in outs[1:])


def test_autotune_keeps_results_and_records_choice(native_lib, oracle_lib, ctx):
    wins = _windows(oracle_lib)
    want = ctx.poa(wins)
    ctx.poa_stage(wins)
    pairs = _pairs()
    want_aln = ctx.align(pairs, want_cigar=True)
    ctx.align_stage(pairs, want_cigar=True)
    t = ctx.autotune(consensus=True, alignment=True)
    assert t["tuned"] == 3
    assert 1 <= t["consensus_ctas_per_sm"] <= 3 and t["consensus_order"] in (0, 1)
    assert t["alignment_warps_per_sm"] in (8, 12, 16, 24, 32)
    assert t["consensus_ms"] > 0 and t["alignment_ms"] > 0
    assert ctx.poa_fetch() == want
    assert ctx.align_fetch() == want_aln
    # the tuned choices apply to later runs on the device
    assert ctx.poa(wins) == want


def test_autotune_needs_a_staged_batch(native_lib, ctx):
    with pytest.raises(native_lib.RaconB200Error, match="no windows staged"):
        ctx.autotune(consensus=True)
