"""racon's whole pipeline with the device hot path (createPolisher +
initialize + polish through the C ABI) vs the oracle pipeline: the polished
FASTA must be byte-identical, and racon's golden numbers must hold."""
import gzip
import json
import os

import pytest

from conftest import GOLDEN, lambda_path
from seqio import revcomp

pytestmark = pytest.mark.gpu

GOLDENS = json.load(open(os.path.join(GOLDEN, "goldens.json")))


@pytest.mark.parametrize("g", GOLDENS, ids=[g["name"] for g in GOLDENS])
def test_pipeline_matches_oracle(native_lib, oracle_lib, g):
    kw = dict(fragment=bool(g["fragment"]), window_length=g["window_length"], match=g["match"],
              mismatch=g["mismatch"], gap=g["gap"], drop_unpolished=bool(g["drop_unpolished"]))
    paths = (lambda_path(g["reads"]), lambda_path(g["overlaps"]), lambda_path(g["targets"]))
    dev = native_lib.polish_files(*paths, **kw)
    ref, _, _ = oracle_lib.polish(*paths, threads=8, **kw)
    assert dev == ref
    exp = g["expected"]
    lines = dev.split("\n")
    recs = [lines[i + 1] for i in range(0, len(lines) - 1, 2)]
    if "edit_distance" in exp:
        with gzip.open(lambda_path("sample_reference.fasta.gz"), "rt") as fh:
            truth = "".join(l.strip() for l in fh if not l.startswith(">"))
        assert oracle_lib.nw_distance(revcomp(recs[0]), truth) == exp["edit_distance"]
    else:
        assert len(recs) == exp["sequences"]
