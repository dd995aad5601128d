#!/usr/bin/env python
"""racon_wrapper on the B200 path: split targets into chunks and/or subsample
reads, then polish every chunk with racon_b200's pipeline.

Same command line and behaviour as racon's scripts/racon_wrapper.py
(RaconWrapper.run, scripts/racon_wrapper.py:56-146): an optional subsampling
of the reads to a coverage of a given reference length, an optional split of
the target sequences into chunks of at most --split bytes, then one racon run
per chunk, in order, each printing its polished FASTA to stdout. The
reference delegates both preprocessing steps to the external `rampler` tool,
which is not part of its tree; they are defined here:

  split      targets are taken in file order and packed into consecutive
             chunks; a chunk takes the next target while its sequence bytes
             stay within the chunk size (a target larger than the chunk size
             forms a chunk of its own).
  subsample  reads are drawn in a seeded random order (numpy PCG64, seed 0
             unless --seed) until their total length reaches coverage x
             reference length, and written in their input order.

Chunks run one after another through rb_polish_files (as the reference runs
racon sequentially), or, with --parallel N, concurrently through the serving
loop (rb_server) on N workers with outputs still printed in chunk order. The
CUDA flags of the reference are accepted and ignored.
"""
import argparse
import gzip
import os
import shutil
import sys
import tempfile
import time

import numpy as np

from . import RaconB200Error, Server, polish_files


def _open(path):
    return gzip.open(path, "rt") if path.endswith(".gz") else open(path)


def read_records(path):
    """(name line without the marker, sequence, quality or None) per record of
    a FASTA/FASTQ file (plain or gzip); FASTA sequences may span lines."""
    recs = []
    with _open(path) as fh:
        lines = fh.read().split("\n")
    if not lines or not lines[0]:
        return recs
    if lines[0].startswith("@"):
        # multi-line FASTQ: sequence lines up to '+', then quality lines until
        # the quality is as long as the sequence
        k, n = 0, len(lines)
        while k < n:
            if not lines[k]:
                k += 1
                continue
            name = lines[k][1:]
            k += 1
            seq = []
            while k < n and not lines[k].startswith("+"):
                seq.append(lines[k])
                k += 1
            k += 1
            s = "".join(seq)
            qual, ql = [], 0
            while k < n and ql < len(s):
                qual.append(lines[k])
                ql += len(lines[k])
                k += 1
            recs.append((name, s, "".join(qual)))
        return recs
    name, parts = None, []
    for line in lines:
        if line.startswith(">"):
            if name is not None:
                recs.append((name, "".join(parts), None))
            name, parts = line[1:], []
        elif line:
            parts.append(line)
    if name is not None:
        recs.append((name, "".join(parts), None))
    return recs


def write_records(path, recs):
    with open(path, "w") as fh:
        for name, seq, qual in recs:
            if qual is None:
                fh.write(">%s\n%s\n" % (name, seq))
            else:
                fh.write("@%s\n%s\n+\n%s\n" % (name, seq, qual))


def _ext(path, recs):
    return ".fastq" if recs and recs[0][2] is not None else ".fasta"


def split_targets(recs, chunk_size):
    """Consecutive chunks of whole targets with at most chunk_size sequence
    bytes each (a longer target alone)."""
    chunks, cur, size = [], [], 0
    for r in recs:
        n = len(r[1])
        if cur and size + n > chunk_size:
            chunks.append(cur)
            cur, size = [], 0
        cur.append(r)
        size += n
    if cur:
        chunks.append(cur)
    return chunks


def subsample_reads(recs, reference_length, coverage, seed=0):
    """Reads in input order whose total length first reaches coverage x
    reference_length when drawn in a seeded random order (all reads when
    they are fewer)."""
    goal = int(reference_length) * float(coverage)
    order = np.random.default_rng(seed).permutation(len(recs))
    keep, total = [], 0
    for i in order:
        if total >= goal:
            break
        keep.append(int(i))
        total += len(recs[i][1])
    keep.sort()
    return [recs[i] for i in keep]


def main(argv=None):
    p = argparse.ArgumentParser(description="racon_wrapper on the B200 path: optional subsampling of the reads and "
                                            "splitting of the targets, then racon_b200 on every chunk.")
    p.add_argument("sequences")
    p.add_argument("overlaps")
    p.add_argument("target_sequences")
    p.add_argument("--split", type=int, help="split target sequences into chunks of at most this many bytes")
    p.add_argument("--subsample", nargs=2, metavar=("REFERENCE_LENGTH", "COVERAGE"),
                   help="subsample the sequences to COVERAGE x REFERENCE_LENGTH bases")
    p.add_argument("--seed", type=int, default=0, help="seed of the subsampling draw")
    p.add_argument("-u", "--include-unpolished", action="store_true")
    p.add_argument("-f", "--fragment-correction", action="store_true")
    p.add_argument("-w", "--window-length", type=int, default=500)
    p.add_argument("-q", "--quality-threshold", type=float, default=10.0)
    p.add_argument("-e", "--error-threshold", type=float, default=0.3)
    p.add_argument("-m", "--match", type=int, default=5)
    p.add_argument("-x", "--mismatch", type=int, default=-4)
    p.add_argument("-g", "--gap", type=int, default=-8)
    p.add_argument("-t", "--threads", type=int, default=1)
    p.add_argument("--cudaaligner-batches", default=0, help="accepted for compatibility; ignored")
    p.add_argument("-c", "--cudapoa-batches", default=0, help="accepted for compatibility; ignored")
    p.add_argument("-b", "--cuda-banded-alignment", action="store_true", help="accepted for compatibility; ignored")
    p.add_argument("--parallel", type=int, default=0, help="run the chunks concurrently on this many serving workers")
    p.add_argument("--device", type=int, default=int(os.environ.get("RACON_B200_DEVICE", "0")))
    a = p.parse_args(argv)

    work = os.path.join(os.getcwd(), "racon_work_directory_" + str(time.time()))
    try:
        os.makedirs(work)
    except OSError:
        sys.stderr.write("[RaconWrapper::__enter__] error: unable to create work directory!\n")
        return 1
    try:
        reads = a.sequences
        if a.subsample:
            sys.stderr.write("[RaconWrapper::run] preparing data: subsampling\n")
            recs = read_records(a.sequences)
            sub = subsample_reads(recs, a.subsample[0], a.subsample[1], a.seed)
            reads = os.path.join(work, "sequences_%sx%s" % (a.subsample[1], _ext(a.sequences, recs)))
            write_records(reads, sub)
        parts = [a.target_sequences]
        if a.split:
            recs = read_records(a.target_sequences)
            chunks = split_targets(recs, a.split)
            parts = []
            for i, c in enumerate(chunks):
                path = os.path.join(work, "targets_%d%s" % (i, _ext(a.target_sequences, recs)))
                write_records(path, c)
                parts.append(path)
            sys.stderr.write("[RaconWrapper::run] total number of splits: %d\n" % len(parts))
        if a.parallel > 0 and len(parts) > 1:
            with Server(a.device, workers=a.parallel, match=a.match, mismatch=a.mismatch, gap=a.gap,
                        window_length=a.window_length) as srv:
                tickets = [srv.submit(reads, a.overlaps, t, fragment=a.fragment_correction,
                                      quality_threshold=a.quality_threshold, error_threshold=a.error_threshold,
                                      drop_unpolished=not a.include_unpolished) for t in parts]
                for t in tickets:
                    sys.stdout.write(srv.wait(t)[0])
                    sys.stdout.flush()
        else:
            for t in parts:
                sys.stderr.write("[RaconWrapper::run] processing data with racon\n")
                sys.stdout.write(polish_files(reads, a.overlaps, t, fragment=a.fragment_correction,
                                              window_length=a.window_length, quality_threshold=a.quality_threshold,
                                              error_threshold=a.error_threshold, match=a.match,
                                              mismatch=a.mismatch, gap=a.gap, threads=a.threads,
                                              drop_unpolished=not a.include_unpolished, device=a.device))
                sys.stdout.flush()
    except RaconB200Error as e:
        sys.stderr.write("%s\n" % e)
        return 1
    finally:
        try:
            shutil.rmtree(work)
        except OSError:
            sys.stderr.write("[RaconWrapper::__exit__] warning: unable to clean work directory!\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
