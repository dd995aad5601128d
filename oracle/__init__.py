"""ORACLE — test infrastructure only.

ctypes loader of the CPU restatement (oracle/_build/liboracle.so, built by
oracle/Makefile) of racon's polishing path: edlib-semantics NW alignment,
spoa-semantics window POA and racon's host pipeline. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use it, and only as
the checker; the racon_b200 product never imports it.
"""
import ctypes
import os
import struct
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
BIN = os.path.join(HERE, "_build", "racon_oracle")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "-j8"], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = ctypes.CDLL(LIB)
    c = ctypes
    lib.oracle_nw_distance.argtypes = [c.c_char_p, c.c_int, c.c_char_p, c.c_int]
    lib.oracle_nw_cigar.argtypes = [c.c_char_p, c.c_int, c.c_char_p, c.c_int, c.c_char_p, c.c_int,
                                    c.POINTER(c.c_int)]
    lib.oracle_breakpoints.argtypes = [c.c_char_p] + [c.c_uint32] * 7 + [c.POINTER(c.c_uint32), c.c_int]
    lib.oracle_window_consensus.argtypes = [c.c_char_p, c.c_char_p, c.c_uint32, c.c_uint32,
                                            c.POINTER(c.c_char_p), c.POINTER(c.c_char_p),
                                            c.POINTER(c.c_uint32), c.POINTER(c.c_uint32),
                                            c.POINTER(c.c_uint32), c.c_int, c.c_int, c.c_int, c.c_int, c.c_int,
                                            c.c_char_p, c.c_int, c.POINTER(c.c_int), c.POINTER(c.c_uint64),
                                            c.POINTER(c.c_uint32)]
    lib.oracle_polish.restype = c.c_void_p
    lib.oracle_polish.argtypes = [c.c_char_p] * 3 + [c.c_int, c.c_uint32, c.c_double, c.c_double, c.c_int,
                                                     c.c_int, c.c_int, c.c_int, c.c_uint32, c.c_int,
                                                     c.POINTER(c.c_double), c.POINTER(c.c_uint64)]
    lib.oracle_dump_windows.restype = c.c_void_p
    lib.oracle_dump_windows.argtypes = [c.c_char_p] * 3 + [c.c_int, c.c_uint32, c.c_double, c.c_double,
                                                           c.c_uint32, c.POINTER(c.c_uint64)]
    lib.oracle_dump_layer_input.restype = c.c_void_p
    lib.oracle_dump_layer_input.argtypes = [c.c_char_p] * 3 + [c.c_int, c.c_uint32, c.c_double, c.c_double,
                                                               c.c_uint32, c.POINTER(c.c_uint64)]
    lib.oracle_free.argtypes = [c.c_void_p]
    lib.oracle_consensus_blob.restype = c.c_int64
    lib.oracle_consensus_blob.argtypes = [c.c_char_p, c.c_uint64, c.c_int64, c.c_uint32, c.c_int, c.c_int, c.c_int,
                                          c.c_int, c.POINTER(c.c_double), c.POINTER(c.c_uint64)]
    lib.oracle_consensus_blob_out.restype = c.c_int64
    lib.oracle_consensus_blob_out.argtypes = [c.c_char_p, c.c_uint64, c.c_int64, c.c_uint32, c.c_int, c.c_int,
                                              c.c_int, c.c_int, c.POINTER(c.c_double), c.POINTER(c.c_uint64),
                                              c.POINTER(c.c_uint64), c.c_char_p, c.c_uint64,
                                              c.POINTER(c.c_uint64), c.POINTER(c.c_uint8)]
    _lib = lib
    return lib


def _b(s):
    return s.encode() if isinstance(s, str) else s


def nw_distance(q, t):
    q, t = _b(q), _b(t)
    return load().oracle_nw_distance(q, len(q), t, len(t))


def nw_cigar(q, t):
    """(edit distance, standard CIGAR) as edlib NW + PATH + STANDARD CIGAR."""
    q, t = _b(q), _b(t)
    lib = load()
    cap = 16 * (len(q) + len(t)) + 64
    buf = ctypes.create_string_buffer(cap)
    n = ctypes.c_int()
    d = lib.oracle_nw_cigar(q, len(q), t, len(t), buf, cap, ctypes.byref(n))
    return d, buf.value.decode()


def breakpoints(cigar, q_begin, q_end, q_length, t_begin, t_end, strand, window_length):
    lib = load()
    cap = 4 * ((t_end - t_begin) // max(1, window_length) + 4)
    out = (ctypes.c_uint32 * cap)()
    n = lib.oracle_breakpoints(_b(cigar), q_begin, q_end, q_length, t_begin, t_end, strand, window_length, out, cap)
    assert n >= 0
    return [(out[i], out[i + 1]) for i in range(0, n, 2)]


def window_consensus(w, match, mismatch, gap, trim=True):
    """w: dict like racon_b200.Context.poa windows. Returns (consensus, polished, cells)."""
    lib = load()
    layers = [_b(s) for s in w["layers"]]
    quals = [_b(q) if q is not None else None for q in w.get("qualities", [None] * len(layers))]
    n = len(layers)
    bb = _b(w["backbone"])
    bq = _b(w.get("backbone_quality")) or b"!" * len(bb)
    la = (ctypes.c_char_p * max(1, n))(*layers)
    qa = (ctypes.c_char_p * max(1, n))(*quals)
    ll = (ctypes.c_uint32 * max(1, n))(*[len(s) for s in layers])
    bg = (ctypes.c_uint32 * max(1, n))(*w["begins"])
    en = (ctypes.c_uint32 * max(1, n))(*w["ends"])
    cap = 4 * len(bb) + sum(len(s) for s in layers) + 1024
    out = ctypes.create_string_buffer(cap)
    olen = ctypes.c_int()
    cells = ctypes.c_uint64()
    nodes = ctypes.c_uint32()
    r = lib.oracle_window_consensus(bb, bq, len(bb), n, la, qa, ll, bg, en, int(w.get("tgs", 1)), int(trim), match,
                                    mismatch, gap, out, cap, ctypes.byref(olen), ctypes.byref(cells),
                                    ctypes.byref(nodes))
    assert r >= 0
    return out.raw[:olen.value].decode(), bool(r), cells.value


def polish(sequences, overlaps, targets, fragment=False, window_length=500, quality_threshold=10.0,
           error_threshold=0.3, trim=True, match=3, mismatch=-5, gap=-4, threads=8, drop_unpolished=True):
    """racon's pipeline on the CPU; returns (fasta text, stage seconds, counts)."""
    lib = load()
    tm = (ctypes.c_double * 4)()
    cn = (ctypes.c_uint64 * 3)()
    p = lib.oracle_polish(_b(sequences), _b(overlaps), _b(targets), int(fragment), window_length,
                          quality_threshold, error_threshold, int(trim), match, mismatch, gap, threads,
                          int(drop_unpolished), tm, cn)
    if not p:
        raise RuntimeError("oracle pipeline failed")
    try:
        text = ctypes.string_at(p).decode()
    finally:
        lib.oracle_free(p)
    return text, list(tm), list(cn)


def dump_layer_input(sequences, overlaps, targets, fragment=False, window_length=500, quality_threshold=10.0,
                     error_threshold=0.3, threads=8):
    """The inputs of racon's layer loop after the breaking points: the
    sequence table (dicts with data, quality, rc, rquality as bytes or None),
    the target count, tgs, and the overlaps (q_id, t_id, strand,
    breakpoints as (t, q) points) in racon's order."""
    lib = load()
    nb = ctypes.c_uint64()
    p = lib.oracle_dump_layer_input(_b(sequences), _b(overlaps), _b(targets), int(fragment), window_length,
                                    quality_threshold, error_threshold, threads, ctypes.byref(nb))
    if not p:
        raise RuntimeError("oracle layer-input dump failed")
    try:
        blob = ctypes.string_at(p, nb.value)
    finally:
        lib.oracle_free(p)
    ns, nt, tgs = struct.unpack_from("<QQB", blob, 0)
    off = 17
    seqs = []
    for _ in range(ns):
        parts = []
        for _ in range(4):
            (n,) = struct.unpack_from("<I", blob, off)
            off += 4
            parts.append(blob[off:off + n] if n else None)
            off += n
        seqs.append({"data": parts[0], "quality": parts[1], "rc": parts[2], "rquality": parts[3]})
    (no,) = struct.unpack_from("<Q", blob, off)
    off += 8
    ovl = []
    for _ in range(no):
        q_id, t_id, strand, npts = struct.unpack_from("<IIII", blob, off)
        off += 16
        pts = list(struct.iter_unpack("<II", blob[off:off + 8 * npts]))
        off += 8 * npts
        ovl.append({"q_id": q_id, "t_id": t_id, "strand": strand, "breakpoints": pts})
    return {"sequences": seqs, "n_targets": nt, "tgs": bool(tgs), "overlaps": ovl}


def dump_windows(sequences, overlaps, targets, fragment=False, window_length=500, quality_threshold=10.0,
                 error_threshold=0.3, threads=8):
    """Every window after racon's initialize(), as dicts for Context.poa."""
    lib = load()
    nb = ctypes.c_uint64()
    p = lib.oracle_dump_windows(_b(sequences), _b(overlaps), _b(targets), int(fragment), window_length,
                                quality_threshold, error_threshold, threads, ctypes.byref(nb))
    if not p:
        raise RuntimeError("oracle window dump failed")
    try:
        blob = ctypes.string_at(p, nb.value)
    finally:
        lib.oracle_free(p)
    (nw,) = struct.unpack_from("<Q", blob, 0)
    off = 8
    wins = []
    for _ in range(nw):
        tid, rank, tgs, bl, nl = struct.unpack_from("<QIBII", blob, off)
        off += 21
        bb = blob[off:off + bl]
        off += bl
        bq = blob[off:off + bl]
        off += bl
        layers, quals, begins, ends = [], [], [], []
        for _ in range(nl):
            ln, b, e, hq = struct.unpack_from("<IIIB", blob, off)
            off += 13
            layers.append(blob[off:off + ln])
            off += ln
            if hq:
                quals.append(blob[off:off + ln])
                off += ln
            else:
                quals.append(None)
            begins.append(b)
            ends.append(e)
        wins.append({"id": tid, "rank": rank, "tgs": tgs, "backbone": bb, "backbone_quality": bq,
                     "layers": layers, "qualities": quals, "begins": begins, "ends": ends})
    return wins


def windows_blob(windows):
    """Windows (dicts) in the oracle_dump_windows layout."""
    parts = [struct.pack("<Q", len(windows))]
    for w in windows:
        bb = _b(w["backbone"])
        bq = _b(w.get("backbone_quality")) or b"!" * len(bb)
        parts.append(struct.pack("<QIBII", w.get("id", 0), w.get("rank", 0), int(w.get("tgs", 1)), len(bb),
                                 len(w["layers"])))
        parts += [bb, bq]
        quals = w.get("qualities") or [None] * len(w["layers"])
        for s_, q, b, e in zip(w["layers"], quals, w["begins"], w["ends"]):
            s_ = _b(s_)
            parts.append(struct.pack("<IIIB", len(s_), b, e, 1 if q else 0))
            parts.append(s_)
            if q:
                parts.append(_b(q))
    return b"".join(parts)


def consensus_blob(blob, max_windows, threads, match, mismatch, gap, trim=True):
    """CPU window consensus of up to max_windows windows on `threads` threads:
    (windows done, seconds, DP cells)."""
    sec = ctypes.c_double()
    cells = ctypes.c_uint64()
    n = load().oracle_consensus_blob(blob, len(blob), max_windows, threads, match, mismatch, gap, int(trim),
                                     ctypes.byref(sec), ctypes.byref(cells))
    if n < 0:
        raise RuntimeError("bad window blob")
    return n, sec.value, cells.value


def consensus_blob_out(blob, max_windows, threads, match, mismatch, gap, trim=True, out_cap=None):
    """As consensus_blob, and also the results: (windows done, seconds, DP
    cells, edge-cells, [(consensus, polished)] per window). Edge-cells count
    the DP work as sum |layer| x sum_v (1 + indeg v) over every alignment."""
    lib = load()
    (nw,) = struct.unpack_from("<Q", blob, 0)
    n = min(nw, max_windows)
    cap = out_cap or 4 * len(blob) + 1024
    out = ctypes.create_string_buffer(cap)
    offs = (ctypes.c_uint64 * (n + 1))()
    pol = (ctypes.c_uint8 * max(1, n))()
    sec = ctypes.c_double()
    cells = ctypes.c_uint64()
    ecells = ctypes.c_uint64()
    r = lib.oracle_consensus_blob_out(blob, len(blob), max_windows, threads, match, mismatch, gap, int(trim),
                                      ctypes.byref(sec), ctypes.byref(cells), ctypes.byref(ecells), out, cap,
                                      offs, pol)
    if r < 0:
        raise RuntimeError("bad window blob or output too small")
    raw = out.raw
    res = [(raw[offs[i]:offs[i + 1]].decode(), bool(pol[i])) for i in range(r)]
    return r, sec.value, cells.value, ecells.value, res
