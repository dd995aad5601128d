"""racon_wrapper on the device path: the output of a split (and subsampled)
run equals the CPU oracle's racon output on each chunk, concatenated in chunk
order, byte for byte; sequentially and through the serving loop."""
import contextlib
import io
import os

import pytest

from conftest import lambda_path
from racon_b200 import wrapper

pytestmark = pytest.mark.gpu

READS = lambda_path("sample_reads.fastq.gz")
AVA = lambda_path("sample_ava_overlaps.paf.gz")


def _run(args, cwd):
    out = io.StringIO()
    old = os.getcwd()
    os.chdir(cwd)
    try:
        with contextlib.redirect_stdout(out):
            assert wrapper.main(args) == 0
    finally:
        os.chdir(old)
    return out.getvalue()


def _oracle_chunks(oracle_lib, reads, targets_recs, chunk, tmp_path, **kw):
    text = ""
    for i, c in enumerate(wrapper.split_targets(targets_recs, chunk)):
        p = str(tmp_path / ("part%d.fastq" % i))
        wrapper.write_records(p, c)
        text += oracle_lib.polish(reads, AVA, p, **kw)[0]
    return text


@pytest.mark.parametrize("parallel", [0, 2])
def test_wrapper_split_fragment(native_lib, oracle_lib, tmp_path, parallel):
    chunk = 600000
    got = _run([READS, AVA, READS, "--split", str(chunk), "-f", "-u", "-m", "1", "-x", "-1", "-g", "-1",
                "--parallel", str(parallel)], str(tmp_path))
    want = _oracle_chunks(oracle_lib, READS, wrapper.read_records(READS), chunk, tmp_path, fragment=True,
                          match=1, mismatch=-1, gap=-1, drop_unpolished=False)
    assert got.count(">") == 236
    assert got == want


def test_wrapper_subsample_and_split(native_lib, oracle_lib, tmp_path):
    got = _run([READS, AVA, READS, "--subsample", "48502", "20", "--split", "800000", "-f", "-m", "1", "-x", "-1",
                "-g", "-1"], str(tmp_path))
    sub = wrapper.subsample_reads(wrapper.read_records(READS), 48502, 20)
    reads = str(tmp_path / "sub.fastq")
    wrapper.write_records(reads, sub)
    want = _oracle_chunks(oracle_lib, reads, wrapper.read_records(READS), 800000, tmp_path, fragment=True,
                          match=1, mismatch=-1, gap=-1)
    assert got == want
