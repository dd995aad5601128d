"""The restatement of racon's layer loop that the device layer-assembly tests
compare against (tests/layer_loop.py) rebuilds the oracle's own windows
exactly, from the oracle's sequence table and breaking points, on the
reference's lambda inputs: contig polishing with and without qualities, PAF,
SAM and MHAP overlaps, fragment correction, and a stricter -q."""
import pytest

from conftest import lambda_path
from layer_loop import host_windows

CASES = [
    ("sample_reads.fastq.gz", "sample_overlaps.paf.gz", "sample_layout.fasta.gz", False, 10.0),
    ("sample_reads.fasta.gz", "sample_overlaps.paf.gz", "sample_layout.fasta.gz", False, 10.0),
    ("sample_reads.fastq.gz", "sample_overlaps.sam.gz", "sample_layout.fasta.gz", False, 10.0),
    ("sample_reads.fastq.gz", "sample_ava_overlaps.mhap.gz", "sample_reads.fastq.gz", True, 10.0),
    ("sample_reads.fasta.gz", "sample_ava_overlaps.paf.gz", "sample_reads.fasta.gz", True, 10.0),
    # -q 13 keeps about a quarter of the layers -q 10 keeps
    ("sample_reads.fastq.gz", "sample_overlaps.paf.gz", "sample_layout.fasta.gz", False, 13.0),
]


@pytest.mark.parametrize("reads,overlaps,targets,fragment,q", CASES)
def test_restatement_rebuilds_the_oracle_windows(oracle_lib, reads, overlaps, targets, fragment, q):
    paths = [lambda_path(x) for x in (reads, overlaps, targets)]
    inp = oracle_lib.dump_layer_input(*paths, fragment=fragment, quality_threshold=q)
    want = oracle_lib.dump_windows(*paths, fragment=fragment, quality_threshold=q)
    got = host_windows(inp["sequences"], inp["n_targets"], inp["overlaps"], 500, q, inp["tgs"])
    assert len(got) == len(want)
    layers = 0
    for g, w in zip(got, want):
        assert (g["id"], g["rank"], bool(g["tgs"])) == (w["id"], w["rank"], bool(w["tgs"]))
        assert g["backbone"] == w["backbone"]
        # a target without qualities has racon's dummy '!' quality (weight 0)
        assert (g["backbone_quality"] or b"!" * len(g["backbone"])) == w["backbone_quality"]
        assert g["layers"] == w["layers"]
        assert g["qualities"] == w["qualities"]
        assert g["begins"] == w["begins"] and g["ends"] == w["ends"]
        layers += len(g["layers"])
    assert layers > 0
