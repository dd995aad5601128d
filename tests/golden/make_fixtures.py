"""Builds the committed parity fixtures under tests/golden/.

lambda/  the reference's own test inputs (racon test/data/*.gz: lambda phage
         draft, truth, 236 reads, PAF/SAM/MHAP overlaps), copied unmodified so
         the device tests can run where the reference tree is absent. They are
         the inputs of the ten end-to-end goldens in racon's
         test/racon_test.cpp:88-290.
goldens.json  those ten expected values, transcribed from
         test/racon_test.cpp:107,129,151,173,195,217,229-235,247-253,265-271,
         283-289 (configuration and expected edit distance / sequence count /
         total length).

Usage: python tests/golden/make_fixtures.py [/path/to/racon/test/data]
"""
import json
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = ["sample_layout.fasta.gz", "sample_reference.fasta.gz", "sample_reads.fasta.gz",
         "sample_reads.fastq.gz", "sample_overlaps.paf.gz", "sample_overlaps.sam.gz",
         "sample_ava_overlaps.paf.gz", "sample_ava_overlaps.mhap.gz"]

# (name, reads, overlaps, targets, fragment, window, match, mismatch, gap, drop_unpolished, expected)
GOLDENS = [
    ("ConsensusWithQualities", "sample_reads.fastq.gz", "sample_overlaps.paf.gz", "sample_layout.fasta.gz",
     0, 500, 5, -4, -8, 1, {"edit_distance": 1312}),
    ("ConsensusWithoutQualities", "sample_reads.fasta.gz", "sample_overlaps.paf.gz", "sample_layout.fasta.gz",
     0, 500, 5, -4, -8, 1, {"edit_distance": 1566}),
    ("ConsensusWithQualitiesAndAlignments", "sample_reads.fastq.gz", "sample_overlaps.sam.gz",
     "sample_layout.fasta.gz", 0, 500, 5, -4, -8, 1, {"edit_distance": 1317}),
    ("ConsensusWithoutQualitiesAndWithAlignments", "sample_reads.fasta.gz", "sample_overlaps.sam.gz",
     "sample_layout.fasta.gz", 0, 500, 5, -4, -8, 1, {"edit_distance": 1770}),
    ("ConsensusWithQualitiesLargerWindow", "sample_reads.fastq.gz", "sample_overlaps.paf.gz",
     "sample_layout.fasta.gz", 0, 1000, 5, -4, -8, 1, {"edit_distance": 1289}),
    ("ConsensusWithQualitiesEditDistance", "sample_reads.fastq.gz", "sample_overlaps.paf.gz",
     "sample_layout.fasta.gz", 0, 500, 1, -1, -1, 1, {"edit_distance": 1321}),
    ("FragmentCorrectionWithQualities", "sample_reads.fastq.gz", "sample_ava_overlaps.paf.gz",
     "sample_reads.fastq.gz", 0, 500, 1, -1, -1, 1, {"sequences": 39, "total_length": 389394}),
    ("FragmentCorrectionWithQualitiesFull", "sample_reads.fastq.gz", "sample_ava_overlaps.paf.gz",
     "sample_reads.fastq.gz", 1, 500, 1, -1, -1, 0, {"sequences": 236, "total_length": 1658216}),
    ("FragmentCorrectionWithoutQualitiesFull", "sample_reads.fasta.gz", "sample_ava_overlaps.paf.gz",
     "sample_reads.fasta.gz", 1, 500, 1, -1, -1, 0, {"sequences": 236, "total_length": 1663982}),
    ("FragmentCorrectionWithQualitiesFullMhap", "sample_reads.fastq.gz", "sample_ava_overlaps.mhap.gz",
     "sample_reads.fastq.gz", 1, 500, 1, -1, -1, 0, {"sequences": 236, "total_length": 1658216}),
]


def main(src):
    dst = os.path.join(HERE, "lambda")
    os.makedirs(dst, exist_ok=True)
    for f in FILES:
        shutil.copyfile(os.path.join(src, f), os.path.join(dst, f))
    keys = ["name", "reads", "overlaps", "targets", "fragment", "window_length", "match", "mismatch", "gap",
            "drop_unpolished", "expected"]
    with open(os.path.join(HERE, "goldens.json"), "w") as fh:
        json.dump([dict(zip(keys, g)) for g in GOLDENS], fh, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py <racon checkout>/test/data")
    main(sys.argv[1])
