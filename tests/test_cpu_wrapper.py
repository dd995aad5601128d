"""racon_wrapper's preprocessing (split of the targets, subsampling of the
reads) on the CPU: chunks keep every target, in order, within the chunk size;
subsampling reaches the coverage, keeps input order and is deterministic."""
import gzip

from conftest import lambda_path
from racon_b200 import wrapper


def test_read_records_fasta_fastq_gz():
    fa = wrapper.read_records(lambda_path("sample_reads.fasta.gz"))
    fq = wrapper.read_records(lambda_path("sample_reads.fastq.gz"))
    assert len(fa) == len(fq) == 236
    assert [r[1] for r in fa] == [r[1] for r in fq]
    assert all(q is not None and len(q) == len(s) for _, s, q in fq)


def test_split_targets(tmp_path):
    recs = [("t%d" % i, "A" * n, None) for i, n in enumerate([10, 30, 5, 100, 1, 1, 50])]
    chunks = wrapper.split_targets(recs, 40)
    assert [r for c in chunks for r in c] == recs
    assert [[r[0] for r in c] for c in chunks] == [["t0", "t1"], ["t2"], ["t3"], ["t4", "t5"], ["t6"]]
    assert all(sum(len(r[1]) for r in c) <= 40 or len(c) == 1 for c in chunks)
    path = tmp_path / "x.fasta"
    wrapper.write_records(str(path), recs)
    assert wrapper.read_records(str(path)) == recs


def test_subsample_reads():
    recs = wrapper.read_records(lambda_path("sample_reads.fastq.gz"))
    total = sum(len(r[1]) for r in recs)
    sub = wrapper.subsample_reads(recs, 48502, 10)
    got = sum(len(r[1]) for r in sub)
    assert got >= 485020 and got - max(len(r[1]) for r in sub) < 485020
    idx = [recs.index(r) for r in sub]
    assert idx == sorted(idx)
    assert sub == wrapper.subsample_reads(recs, 48502, 10)
    assert wrapper.subsample_reads(recs, 1, total * 2) == recs
