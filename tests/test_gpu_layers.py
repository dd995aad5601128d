"""Device layer assembly (rb_sequences_stage + rb_poa_stage_overlaps) against
the host assembly of racon's initialize() (src/polisher.cpp:401-457).

Two kinds of cases:
* jobs: a prepared job's windows through the device assembly give the same
  consensus as its host-assembled rb_window views through rb_poa_batch (the
  path the oracle parity tests pin), for contig polishing, fragment
  correction and several quality thresholds;
* hand-built tables that hit every branch of racon's layer loop: the span
  filter (< 0.02 w), the mean-quality filter at its boundary, add_layer's
  begin == end skip, reverse-strand slicing, reads without qualities, and a
  window with many layers of equal begin (racon's unstable sort). The
  expected windows come from a restatement of racon's loop
  (tests/layer_loop.py, checked against the oracle's own windows by
  tests/test_cpu_layer_loop.py); the library's rb_poa_batch then computes
  both consensuses.
Quality bytes outside '!'..'~' are refused (RB_ERR_ARG) once they would
reach a window graph; the filter still reads them with racon's uint32
wrap-around, so such a layer is kept (and refused) where racon keeps it.
"""
import random

import pytest

from layer_loop import host_windows, revcomp
from racon_b200 import RaconB200Error, synthetic

pytestmark = pytest.mark.gpu

def _revcomp(s):
    return revcomp(s).decode()


def _host_windows(seqs, n_targets, overlaps, w, q_thr, tgs):
    return host_windows(seqs, n_targets, overlaps, w, q_thr, tgs)


def _mutate(rng, s, err):
    out = []
    for c in s:
        u = rng.random()
        if u < err / 3:
            continue
        out.append(rng.choice("ACGT") if u < 2 * err / 3 else c)
        if rng.random() < err / 3:
            out.append(rng.choice("ACGT"))
    return "".join(out)


def _quals(rng, n, lo=5, hi=30):
    return bytes(33 + rng.randint(lo, hi) for _ in range(n))


def _table(seed, wrap=False):
    """A target (FASTQ) and reads cut from it, with breaking points whose
    pairs cover every branch of the layer loop."""
    rng = random.Random(seed)
    w = 200
    T = "".join(rng.choice("ACGT") for _ in range(1234))
    seqs = [{"data": T, "quality": _quals(rng, len(T)), "forward": 1, "reverse": 0}]
    overlaps = []

    def add_read(qual_kind, strand, pieces):
        """pieces: list of (t0, t1, length of the read slice); the read is the
        concatenation of mutated target slices, breaking points at their
        ends (q in the orientation used)."""
        parts, bps, q = [], [], 0
        for t0, t1, _ in pieces:
            piece = _mutate(rng, T[t0:t1], 0.08) or "A"
            parts.append(piece)
            bps += [(t0, q), (t1, q + len(piece))]
            q += len(piece)
        oriented = "".join(parts)
        data = _revcomp(oriented) if strand else oriented
        if qual_kind == "none":
            qual = None
        elif qual_kind == "q10":
            qual = b"+" * len(data)  # exactly 10: kept at -q 10
        elif qual_kind == "q9":
            qual = b"*" * len(data)  # 9: dropped at -q 10
        elif qual_kind == "wrap":
            # bytes below '!' and above 127 wrap around in racon's uint32 sum
            qual = bytes(rng.choice([32, 5, 200, 35]) for _ in range(len(data)))
        else:
            qual = _quals(rng, len(data))
        seqs.append({"data": data, "quality": qual, "forward": 0 if strand else 1, "reverse": 1 if strand else 0})
        overlaps.append({"q_id": len(seqs) - 1, "t_id": 0, "strand": strand, "breakpoints": bps})

    # spanning reads, both strands, with and without qualities
    kinds = ["phred", "none", "q10", "q9", "phred"] if not wrap else ["wrap"]
    for k in range(14 if not wrap else 1):
        full = [(j, min(j + w, len(T)) - 1, 0) for j in range(0, len(T), w)]
        add_read(kinds[k % len(kinds)], k % 2, full)
    # many layers with equal begin in window 1 (ties for the unstable sort)
    for k in range(40):
        end = 200 + 60 + rng.randint(0, 120)
        add_read("phred", k % 2, [(200, end, 0)])
    # a query span below 0.02 * w (3 < 4 bases): dropped
    seqs.append({"data": T[400:403], "quality": b"555", "forward": 1, "reverse": 0})
    overlaps.append({"q_id": len(seqs) - 1, "t_id": 0, "strand": 0, "breakpoints": [(400, 0), (402, 3)]})
    # begin == end (one target base, t1 = t0 + 1): skipped by add_layer
    seqs.append({"data": T[610:622], "quality": b"5" * 12, "forward": 1, "reverse": 0})
    overlaps.append({"q_id": len(seqs) - 1, "t_id": 0, "strand": 0, "breakpoints": [(610, 0), (611, 12)]})
    # partial layers in the short last window
    add_read("phred", 1, [(1205, 1233, 0)])
    return seqs, overlaps, w


def _device(ctx, seqs, overlaps, n_targets, q_thr, tgs, trim=True):
    ctx.sequences_stage(seqs)
    ctx.poa_stage_overlaps(n_targets, overlaps, quality_threshold=q_thr, tgs=tgs, trim=trim)
    ctx.poa_run()
    return ctx.poa_fetch()


@pytest.mark.parametrize("seed", [1, 2])
@pytest.mark.parametrize("q_thr", [10.0, 0.0, 25.0])
def test_table_matches_host_assembly(native_lib, seed, q_thr):
    seqs, overlaps, w = _table(seed)
    want_windows = _host_windows(seqs, 1, overlaps, w, q_thr, 1)
    if q_thr <= 10.0:
        assert max(len(x["layers"]) for x in want_windows) > 16
    with native_lib.Context(0, 3, -5, -4, w) as ctx:
        want = ctx.poa(want_windows)
        got = _device(ctx, seqs, overlaps, 1, q_thr, 1)
        assert got == want
        st = ctx.layer_stats()
        assert st.items == sum(len(x["layers"]) for x in want_windows)
        # the plain form reads the same staged records
        ctx.poa_run(plain=True)
        assert ctx.poa_fetch() == want


def test_targets_without_layers_and_untrimmed(native_lib):
    seqs, overlaps, w = _table(5)
    rng = random.Random(9)
    # a second target (FASTA) that no overlap touches, and one with a layer
    T2 = "".join(rng.choice("ACGT") for _ in range(450))
    T3 = "".join(rng.choice("ACGT") for _ in range(77))
    seqs = seqs[:1] + [{"data": T2, "quality": None, "forward": 1, "reverse": 0},
                       {"data": T3, "quality": None, "forward": 1, "reverse": 0}] + seqs[1:]
    for o in overlaps:
        o["q_id"] += 2
    r3 = _mutate(rng, T3[5:70], 0.05)
    seqs.append({"data": r3, "quality": None, "forward": 1, "reverse": 0})
    overlaps.append({"q_id": len(seqs) - 1, "t_id": 2, "strand": 0, "breakpoints": [(5, 0), (70, len(r3))]})
    want_windows = _host_windows(seqs, 3, overlaps, w, 10.0, 0)
    with native_lib.Context(0, 3, -5, -4, w) as ctx:
        want = ctx.poa(want_windows, trim=False)
        got = _device(ctx, seqs, overlaps, 3, 10.0, 0, trim=False)
    assert got == want
    assert len(got) == len(want_windows)


@pytest.mark.parametrize("fragment", [False, True])
def test_job_device_matches_host_views(native_lib, tmp_path, fragment):
    if fragment:
        paths = synthetic.fragment(str(tmp_path), genome=9_000, contigs=2, depth=(10, 50), mean=1_800, sd=600,
                                   err=0.15, seed=4, qual_range=(3, 40))[:3]
    else:
        paths = synthetic.contig(str(tmp_path), 0)[:3]
    for q in (10.0, 20.0):
        job = native_lib.Job(*paths, fragment=fragment, window_length=500, quality_threshold=q, match=3,
                             mismatch=-5, gap=-4)
        try:
            with native_lib.Context(0, 3, -5, -4, 500) as ctx:
                want = ctx.poa_job(job)
                ctx.poa_stage_job_device(job)
                ctx.poa_run()
                got = ctx.poa_fetch()
                assert ctx.layer_stats().items == job.layer_stats()[1]
            assert got == want
        finally:
            job.close()


def test_out_of_range_quality_refused(native_lib):
    # one read whose quality bytes are ' ', 0x05, 0xc8 and '#': racon's
    # uint32 terms make its mean quality huge, so the layers are kept
    seqs, overlaps, w = _table(7, wrap=True)
    with native_lib.Context(0, 3, -5, -4, w) as ctx:
        ctx.sequences_stage(seqs)
        with pytest.raises(RaconB200Error) as e:
            ctx.poa_stage_overlaps(1, overlaps, quality_threshold=10.0)
        assert e.value.code == 1 and "quality" in str(e.value)
        with pytest.raises(RaconB200Error) as e:
            ctx.poa(_host_windows(seqs, 1, overlaps, w, 10.0, 1))
        assert e.value.code == 1 and "quality" in str(e.value)
        # a dropped layer (query span below 0.02 w) may carry them
        bad = {"data": "ACG", "quality": bytes([200, 5, 32]), "forward": 1, "reverse": 0}
        seqs2 = seqs[:1] + [bad]
        ovl = [{"q_id": 1, "t_id": 0, "strand": 0, "breakpoints": [(10, 0), (12, 3)]}]
        assert _device(ctx, seqs2, ovl, 1, 10.0, 1) == ctx.poa(_host_windows(seqs2, 1, ovl, w, 10.0, 1))
        # so may a backbone byte '~' (93), but not 0x7f
        seqs3 = [dict(seqs[0], quality=b"~" * len(seqs[0]["data"]))]
        assert _device(ctx, seqs3, [], 1, 10.0, 1) == ctx.poa(_host_windows(seqs3, 1, [], w, 10.0, 1))
        seqs3 = [dict(seqs[0], quality=b"\x7f" * len(seqs[0]["data"]))]
        ctx.sequences_stage(seqs3)
        with pytest.raises(RaconB200Error):
            ctx.poa_stage_overlaps(1, [], quality_threshold=10.0)


def test_rejects_bad_input_and_recovers(native_lib):
    seqs, overlaps, w = _table(3)
    with native_lib.Context(0, 3, -5, -4, w) as ctx:
        ctx.sequences_stage(seqs)
        bad_cases = [
            ({"q_id": len(seqs), "t_id": 0, "strand": 0, "breakpoints": [(0, 0), (10, 10)]}, "id"),
            ({"q_id": 1, "t_id": 0, "strand": 0, "breakpoints": [(0, 0), (10, 10**6)]}, "outside"),
            ({"q_id": 1, "t_id": 0, "strand": 0, "breakpoints": [(0, 0), (w + 1, 50)]}, "invalid"),
            ({"q_id": 1, "t_id": 0, "strand": 0, "breakpoints": [(0, 0), (w + 2, 50)]}, "add_layer"),
            # the read of overlap 0 is staged for the forward strand only
            ({"q_id": overlaps[0]["q_id"], "t_id": 0, "strand": 1, "breakpoints": [(0, 0), (50, 50)]},
             "strand"),
        ]
        for bad, word in bad_cases:
            with pytest.raises(RaconB200Error) as e:
                ctx.poa_stage_overlaps(1, overlaps[:3] + [bad], quality_threshold=10.0)
            assert word in str(e.value)
        # an odd number of points is refused before any kernel runs
        with pytest.raises(RaconB200Error):
            ctx.poa_stage_overlaps(1, [{"q_id": 1, "t_id": 0, "strand": 0, "breakpoints": [(0, 0)]}])
        # the context still works
        want = ctx.poa(_host_windows(seqs, 1, overlaps, w, 10.0, 1))
        got = _device(ctx, seqs, overlaps, 1, 10.0, 1)
        assert got == want
