"""End-to-end parity on the benchmark shapes: the polished FASTA from the
device path (rb_polish_files) is byte-identical to the CPU oracle's on a
seeded config-0 job (contig polishing, 50 kb), on the full-size config-1 job
that bench.py times (1 Mb genome, 50x FASTQ), and on small jobs with the
config-3 shape (fragment correction -f, uneven depth up to 200x, all-vs-all
dual PAF, FASTQ Phred 3-40)."""
import os

import pytest

from racon_b200 import synthetic

pytestmark = pytest.mark.gpu


def _both(native_lib, oracle_lib, paths, fragment, drop):
    got = native_lib.polish_files(*paths, fragment=fragment, window_length=500, quality_threshold=10.0,
                                  error_threshold=0.3, match=3, mismatch=-5, gap=-4, drop_unpolished=drop)
    want, _, _ = oracle_lib.polish(*paths, fragment=fragment, window_length=500, quality_threshold=10.0,
                                   error_threshold=0.3, match=3, mismatch=-5, gap=-4, drop_unpolished=drop,
                                   threads=os.cpu_count() or 8)
    return got, want


def test_config0_contig(native_lib, oracle_lib, tmp_path):
    r, o, t, _ = synthetic.contig(str(tmp_path), 0)
    got, want = _both(native_lib, oracle_lib, (r, o, t), False, True)
    assert got.count(">") == 1
    assert got == want


def test_config3_shape_fragment(native_lib, oracle_lib, tmp_path):
    r, o, t, info = synthetic.fragment(str(tmp_path), genome=12_000, contigs=2, depth=(10, 60), mean=2_000,
                                       sd=800, err=0.15, seed=3, qual_range=(3, 40))
    got, want = _both(native_lib, oracle_lib, (r, o, t), True, False)
    assert got.count(">") == info["reads"]
    assert got == want


def test_config1_full(native_lib, oracle_lib, tmp_path):
    # the timed workload itself: 1 Mb draft, 2001 windows of ~50 layers
    r, o, t, info = synthetic.contig(str(tmp_path), 1)
    got, want = _both(native_lib, oracle_lib, (r, o, t), False, True)
    assert got.count(">") == 1
    assert got == want


def test_config3_depth_to_200(native_lib, oracle_lib, tmp_path):
    # local depth 10-200x: windows of up to ~210 layers
    r, o, t, info = synthetic.fragment(str(tmp_path), genome=4_000, contigs=1, depth=(10, 200), mean=1_500,
                                       sd=500, err=0.15, seed=5, qual_range=(3, 40))
    got, want = _both(native_lib, oracle_lib, (r, o, t), True, False)
    assert got.count(">") == info["reads"]
    assert got == want
