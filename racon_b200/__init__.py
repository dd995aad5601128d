"""racon_b200: racon's polishing hot path (overlap alignment + window POA
consensus) on the NVIDIA B200.

This module is the Python mirror of the C ABI in include/racon_b200.h,
loaded with ctypes from the in-tree library racon_b200/lib/libracon_b200.so
(built by racon_b200/build.py). It exposes:

  Context(device, match, mismatch, gap, window_length)
      .align(pairs, want_cigar)      -> device edit distance / CIGAR / breaking
                                        points (racon src/overlap.cpp:179-292)
      .cigar_breakpoints(overlaps)   -> breaking points from SAM CIGARs
      .poa(windows, trim)            -> window consensus (src/window.cpp:65-142)
      .poa_stage / poa_run / poa_fetch, align_stage / align_run / align_fetch
  polish_files(...)                  -> racon's whole pipeline (createPolisher +
                                        initialize + polish, src/main.cpp:152-166)

There is no CPU fallback: if the library is missing or no B200 is present,
the calls raise.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libracon_b200.so")
CLI_PATH = os.path.join(_HERE, "bin", "racon_b200")

RB_OK = 0
_ERRORS = {1: "RB_ERR_ARG", 2: "RB_ERR_CUDA", 3: "RB_ERR_NOMEM", 4: "RB_ERR_DEVICE", 5: "RB_ERR_NODEV"}


class RaconB200Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (_ERRORS.get(code, str(code)), msg))
        self.code = code


class _Params(ctypes.Structure):
    _fields_ = [("match", ctypes.c_int8), ("mismatch", ctypes.c_int8), ("gap", ctypes.c_int8),
                ("window_length", ctypes.c_uint32)]


class _Pair(ctypes.Structure):
    _fields_ = [("query", ctypes.c_char_p), ("query_length", ctypes.c_uint32),
                ("target", ctypes.c_char_p), ("target_length", ctypes.c_uint32),
                ("q_offset", ctypes.c_uint32), ("t_begin", ctypes.c_uint32)]


class _AlnResult(ctypes.Structure):
    _fields_ = [("edit_distance", ctypes.POINTER(ctypes.c_int32)),
                ("breakpoints", ctypes.POINTER(ctypes.c_uint32)),
                ("bp_offsets", ctypes.POINTER(ctypes.c_uint64)),
                ("cigars", ctypes.POINTER(ctypes.c_char)),
                ("cigar_offsets", ctypes.POINTER(ctypes.c_uint64))]


class _CigarOverlap(ctypes.Structure):
    _fields_ = [("cigar", ctypes.c_char_p), ("cigar_length", ctypes.c_uint32),
                ("q_offset", ctypes.c_uint32), ("t_begin", ctypes.c_uint32), ("t_end", ctypes.c_uint32)]


class _Window(ctypes.Structure):
    _fields_ = [("backbone", ctypes.c_char_p), ("backbone_quality", ctypes.c_char_p),
                ("backbone_length", ctypes.c_uint32), ("n_layers", ctypes.c_uint32),
                ("layers", ctypes.POINTER(ctypes.c_char_p)),
                ("layer_qualities", ctypes.POINTER(ctypes.c_char_p)),
                ("layer_lengths", ctypes.POINTER(ctypes.c_uint32)),
                ("begins", ctypes.POINTER(ctypes.c_uint32)), ("ends", ctypes.POINTER(ctypes.c_uint32)),
                ("tgs", ctypes.c_uint8), ("id", ctypes.c_uint64), ("rank", ctypes.c_uint32)]


class _Sequence(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("quality", ctypes.c_void_p), ("length", ctypes.c_uint32),
                ("forward", ctypes.c_uint8), ("reverse", ctypes.c_uint8)]


class _LayerOverlap(ctypes.Structure):
    _fields_ = [("q_id", ctypes.c_uint32), ("t_id", ctypes.c_uint32), ("strand", ctypes.c_uint32)]


class _StorePair(ctypes.Structure):
    _fields_ = [("q_id", ctypes.c_uint32), ("q_begin", ctypes.c_uint32), ("q_end", ctypes.c_uint32),
                ("t_id", ctypes.c_uint32), ("t_begin", ctypes.c_uint32), ("t_end", ctypes.c_uint32),
                ("strand", ctypes.c_uint32)]


class _PoaResult(ctypes.Structure):
    _fields_ = [("consensus", ctypes.POINTER(ctypes.c_char)), ("offsets", ctypes.POINTER(ctypes.c_uint64)),
                ("polished", ctypes.POINTER(ctypes.c_uint8))]


class _ServerParams(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("workers", ctypes.c_uint32), ("hbm_budget", ctypes.c_uint64),
                ("match", ctypes.c_int8), ("mismatch", ctypes.c_int8), ("gap", ctypes.c_int8),
                ("window_length", ctypes.c_uint32), ("shared_consensus", ctypes.c_int),
                ("consensus_ctas_per_sm", ctypes.c_uint32), ("priority_windows", ctypes.c_uint32),
                ("alignment_yield", ctypes.c_uint32), ("alignment_share", ctypes.c_uint32),
                ("shared_alignment", ctypes.c_int), ("alignment_ctas_per_sm", ctypes.c_uint32),
                ("alignment_max_span", ctypes.c_uint32), ("priority_pairs", ctypes.c_uint32),
                ("large_first_every", ctypes.c_uint32)]


class _ServerJob(ctypes.Structure):
    _fields_ = [("sequences_path", ctypes.c_char_p), ("overlaps_path", ctypes.c_char_p),
                ("target_path", ctypes.c_char_p), ("fragment", ctypes.c_int),
                ("quality_threshold", ctypes.c_double), ("error_threshold", ctypes.c_double),
                ("trim", ctypes.c_int), ("drop_unpolished", ctypes.c_int)]


class ServerTimes(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_double), ("admitted", ctypes.c_double), ("finished", ctypes.c_double),
                ("stage_seconds", ctypes.c_double * 4), ("footprint", ctypes.c_uint64), ("worker", ctypes.c_uint32)]


class Tuning(ctypes.Structure):
    """rb_tuning: a device's launch choices (none changes a result)."""
    _fields_ = [("consensus_ctas_per_sm", ctypes.c_uint32), ("consensus_order", ctypes.c_uint32),
                ("alignment_warps_per_sm", ctypes.c_uint32), ("tuned", ctypes.c_uint32),
                ("consensus_ms", ctypes.c_double), ("alignment_ms", ctypes.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Stats(ctypes.Structure):
    _fields_ = [("kernel_ms", ctypes.c_double), ("h2d_ms", ctypes.c_double), ("d2h_ms", ctypes.c_double),
                ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64), ("launches", ctypes.c_uint64),
                ("cells", ctypes.c_uint64), ("items", ctypes.c_uint64), ("max_nodes", ctypes.c_uint32),
                ("top_kernel_ms", ctypes.c_double), ("edge_cells", ctypes.c_uint64)]


_lib = None


def load():
    """Loads the in-tree native library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RaconB200Error(5, "native library missing: %s (run racon_b200/build.py)" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    lib.rb_create.restype = vp
    lib.rb_create.argtypes = [ctypes.c_int, ctypes.POINTER(_Params)]
    lib.rb_create_error.restype = ctypes.c_char_p
    lib.rb_destroy.argtypes = [vp]
    lib.rb_last_error.restype = ctypes.c_char_p
    lib.rb_last_error.argtypes = [vp]
    lib.rb_align_batch.argtypes = [vp, ctypes.POINTER(_Pair), ctypes.c_size_t, ctypes.c_int,
                                   ctypes.POINTER(_AlnResult)]
    lib.rb_align_stage.argtypes = [vp, ctypes.POINTER(_Pair), ctypes.c_size_t, ctypes.c_int]
    lib.rb_align_run.argtypes = [vp]
    lib.rb_align_fetch.argtypes = [vp, ctypes.POINTER(_AlnResult)]
    lib.rb_cigar_breakpoints.argtypes = [vp, ctypes.POINTER(_CigarOverlap), ctypes.c_size_t,
                                         ctypes.POINTER(_AlnResult)]
    lib.rb_poa_batch.argtypes = [vp, ctypes.POINTER(_Window), ctypes.c_size_t, ctypes.c_int,
                                 ctypes.POINTER(_PoaResult)]
    lib.rb_poa_stage.argtypes = [vp, ctypes.POINTER(_Window), ctypes.c_size_t, ctypes.c_int]
    lib.rb_poa_run.argtypes = [vp]
    lib.rb_poa_run_plain.argtypes = [vp]
    lib.rb_poa_fetch.argtypes = [vp, ctypes.POINTER(_PoaResult)]
    lib.rb_poa_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    lib.rb_sequences_stage.argtypes = [vp, ctypes.POINTER(_Sequence), ctypes.c_size_t]
    lib.rb_poa_stage_overlaps.argtypes = [vp, ctypes.c_size_t, ctypes.POINTER(_LayerOverlap), ctypes.c_size_t,
                                          ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64),
                                          ctypes.c_double, ctypes.c_int, ctypes.c_int]
    lib.rb_align_stage_overlaps.argtypes = [vp, ctypes.POINTER(_StorePair), ctypes.c_size_t, ctypes.c_int]
    lib.rb_poa_stage_alignments.argtypes = [vp, ctypes.c_size_t, ctypes.POINTER(_StorePair), ctypes.c_size_t,
                                            ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(_AlnResult)]
    lib.rb_layer_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    lib.rb_set_yield.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32]
    lib.rb_set_priority.argtypes = [vp, ctypes.c_int]
    lib.rb_set_sm_share.argtypes = [vp, ctypes.c_uint32]
    lib.rb_autotune.argtypes = [vp, ctypes.c_int]
    lib.rb_tuning_get.argtypes = [ctypes.c_int, ctypes.POINTER(Tuning)]
    lib.rb_tuning_set.argtypes = [ctypes.c_int, ctypes.POINTER(Tuning)]
    lib.rb_sequence_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    lib.rb_job_layer_input.argtypes = [vp, ctypes.POINTER(ctypes.POINTER(_Sequence)),
                                       ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t),
                                       ctypes.POINTER(ctypes.POINTER(_LayerOverlap)),
                                       ctypes.POINTER(ctypes.c_size_t),
                                       ctypes.POINTER(ctypes.POINTER(ctypes.c_uint32)),
                                       ctypes.POINTER(ctypes.POINTER(ctypes.c_uint64)),
                                       ctypes.POINTER(ctypes.c_int)]
    lib.rb_align_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    lib.rb_polish_files.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int,
                                    ctypes.c_uint32, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_int8, ctypes.c_int8, ctypes.c_int8, ctypes.c_uint32, ctypes.c_int,
                                    ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                    ctypes.POINTER(ctypes.c_double)]
    lib.rb_pipeline_error.restype = ctypes.c_char_p
    lib.rb_job_prepare.restype = vp
    lib.rb_job_prepare.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_uint32,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_int8, ctypes.c_int8, ctypes.c_int8,
                                   ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.rb_job_windows.restype = ctypes.c_size_t
    lib.rb_job_windows.argtypes = [vp, ctypes.POINTER(ctypes.POINTER(_Window))]
    lib.rb_job_free.argtypes = [vp]
    lib.rb_job_context.restype = vp
    lib.rb_job_context.argtypes = [vp]
    lib.rb_free.argtypes = [vp]
    lib.rb_server_create.restype = vp
    lib.rb_server_create.argtypes = [ctypes.POINTER(_ServerParams)]
    lib.rb_server_submit.argtypes = [vp, ctypes.POINTER(_ServerJob), ctypes.POINTER(ctypes.c_uint64)]
    lib.rb_server_wait.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ServerTimes)]
    lib.rb_server_error.restype = ctypes.c_char_p
    lib.rb_server_load.argtypes = [vp, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                                   ctypes.POINTER(ctypes.c_uint64)]
    lib.rb_server_destroy.argtypes = [vp]
    _lib = lib
    return lib


def _b(s):
    if s is None:
        return None
    return s.encode() if isinstance(s, str) else bytes(s)


class Context:
    """One device context (include/racon_b200.h rb_create)."""

    def __init__(self, device=0, match=3, mismatch=-5, gap=-4, window_length=500):
        self.lib = load()
        p = _Params(match, mismatch, gap, window_length)
        self.ptr = self.lib.rb_create(device, ctypes.byref(p))
        if not self.ptr:
            raise RaconB200Error(5, self.lib.rb_create_error().decode())
        self.device = device
        self.window_length = window_length
        self._keep = None

    def close(self):
        if self.ptr:
            self.lib.rb_destroy(self.ptr)
            self.ptr = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != RB_OK:
            raise RaconB200Error(rc, self.lib.rb_last_error(self.ptr).decode())

    # ---- overlap alignment ----
    def _pairs(self, pairs):
        arr = (_Pair * max(1, len(pairs)))()
        keep = []
        for i, p in enumerate(pairs):
            q, t = _b(p["query"]), _b(p["target"])
            keep += [q, t]
            arr[i] = _Pair(q, len(q), t, len(t), p.get("q_offset", 0), p.get("t_begin", 0))
        return arr, keep

    @staticmethod
    def _aln_out(r, n, want_cigar):
        out = []
        for i in range(n):
            b, e = r.bp_offsets[i], r.bp_offsets[i + 1]
            bp = [(r.breakpoints[k], r.breakpoints[k + 1]) for k in range(b, e, 2)]
            cig = None
            if want_cigar and r.cigar_offsets:
                cb, ce = r.cigar_offsets[i], r.cigar_offsets[i + 1]
                cig = ctypes.string_at(ctypes.addressof(r.cigars.contents) + cb, ce - cb).decode() if ce > cb else ""
            out.append({"edit_distance": r.edit_distance[i], "breakpoints": bp, "cigar": cig})
        return out

    def prepare_pairs(self, pairs):
        """The rb_pair array (host buffers) for pairs, to pass to
        align_prepared repeatedly."""
        arr, keep = self._pairs(pairs)
        return arr, keep, len(pairs)

    def align_prepared(self, prepared, want_cigar=True):
        """rb_align_batch on a prepare_pairs array; returns the raw result
        (library-owned arrays) without converting it to Python objects."""
        arr, _, n = prepared
        r = _AlnResult()
        self._check(self.lib.rb_align_batch(self.ptr, arr, n, int(want_cigar), ctypes.byref(r)))
        return r

    def aln_results(self, r, n, want_cigar=True):
        """Python view of a raw rb_aln_result of n pairs."""
        return self._aln_out(r, n, want_cigar)

    def align(self, pairs, want_cigar=True):
        """pairs: list of dicts with query, target, q_offset, t_begin."""
        arr, keep = self._pairs(pairs)
        r = _AlnResult()
        self._check(self.lib.rb_align_batch(self.ptr, arr, len(pairs), int(want_cigar), ctypes.byref(r)))
        return self._aln_out(r, len(pairs), want_cigar)

    def align_stage(self, pairs, want_cigar=False):
        arr, keep = self._pairs(pairs)
        self._check(self.lib.rb_align_stage(self.ptr, arr, len(pairs), int(want_cigar)))
        self._staged_pairs = len(pairs)
        self._staged_cigar = want_cigar

    def align_run(self):
        self._check(self.lib.rb_align_run(self.ptr))

    def align_fetch(self):
        r = _AlnResult()
        self._check(self.lib.rb_align_fetch(self.ptr, ctypes.byref(r)))
        return self._aln_out(r, self._staged_pairs, self._staged_cigar)

    def cigar_breakpoints(self, overlaps):
        """overlaps: list of dicts with cigar, q_offset, t_begin, t_end."""
        arr = (_CigarOverlap * max(1, len(overlaps)))()
        keep = []
        for i, o in enumerate(overlaps):
            c = _b(o["cigar"])
            keep.append(c)
            arr[i] = _CigarOverlap(c, len(c), o["q_offset"], o["t_begin"], o["t_end"])
        r = _AlnResult()
        self._check(self.lib.rb_cigar_breakpoints(self.ptr, arr, len(overlaps), ctypes.byref(r)))
        return [x["breakpoints"] for x in self._aln_out(r, len(overlaps), False)]

    # ---- window consensus ----
    def _windows(self, windows):
        arr = (_Window * max(1, len(windows)))()
        keep = []
        for i, w in enumerate(windows):
            bb = _b(w["backbone"])
            bq = _b(w.get("backbone_quality"))
            layers = [_b(s) for s in w["layers"]]
            quals = [_b(q) for q in w.get("qualities", [None] * len(layers))]
            n = len(layers)
            la = (ctypes.c_char_p * max(1, n))(*layers)
            qa = (ctypes.c_char_p * max(1, n))(*quals)
            ll = (ctypes.c_uint32 * max(1, n))(*[len(s) for s in layers])
            bg = (ctypes.c_uint32 * max(1, n))(*w["begins"])
            en = (ctypes.c_uint32 * max(1, n))(*w["ends"])
            keep += [bb, bq, layers, quals, la, qa, ll, bg, en]
            arr[i] = _Window(bb, bq, len(bb), n, la, qa, ll, bg, en, int(w.get("tgs", 1)), w.get("id", 0),
                             w.get("rank", 0))
        return arr, keep

    @staticmethod
    def _poa_out(r, n):
        out = []
        base = ctypes.addressof(r.consensus.contents) if n else 0
        for i in range(n):
            b, e = r.offsets[i], r.offsets[i + 1]
            out.append((ctypes.string_at(base + b, e - b).decode() if e > b else "", bool(r.polished[i])))
        return out

    def poa(self, windows, trim=True):
        """windows: list of dicts (backbone, backbone_quality, layers, qualities,
        begins, ends, tgs). Returns [(consensus, polished)]."""
        arr, keep = self._windows(windows)
        r = _PoaResult()
        self._check(self.lib.rb_poa_batch(self.ptr, arr, len(windows), int(trim), ctypes.byref(r)))
        return self._poa_out(r, len(windows))

    def poa_stage(self, windows, trim=True):
        arr, keep = self._windows(windows)
        self._check(self.lib.rb_poa_stage(self.ptr, arr, len(windows), int(trim)))
        self._staged_windows = len(windows)

    def poa_run(self, plain=False):
        """Runs the staged windows: the batched form (size-sorted work queue),
        or with plain=True the comparison form (one window per block, input
        order, no queue). Both give identical results."""
        self._check((self.lib.rb_poa_run_plain if plain else self.lib.rb_poa_run)(self.ptr))

    def poa_fetch(self):
        r = _PoaResult()
        self._check(self.lib.rb_poa_fetch(self.ptr, ctypes.byref(r)))
        return self._poa_out(r, self._staged_windows)

    def poa_job(self, job, trim=True):
        """Consensus of every window of a Job, passing its window views straight
        to rb_poa_batch (host buffers, copies included)."""
        r = _PoaResult()
        self._check(self.lib.rb_poa_batch(self.ptr, job.windows, job.n, int(trim), ctypes.byref(r)))
        return self._poa_out(r, job.n)

    def poa_stage_job(self, job, trim=True):
        self._check(self.lib.rb_poa_stage(self.ptr, job.windows, job.n, int(trim)))
        self._staged_windows = job.n

    # ---- device layer assembly ----
    def sequences_stage(self, sequences):
        """sequences: racon's sequence table (targets first) as dicts with
        data, quality (or None), forward, reverse (rb_sequences_stage)."""
        n = len(sequences)
        arr = (_Sequence * max(1, n))()
        keep = []
        for i, e in enumerate(sequences):
            d = _b(e["data"]) or b""
            q = _b(e.get("quality"))
            db = ctypes.create_string_buffer(d, max(1, len(d)))
            qb = ctypes.create_string_buffer(q, max(1, len(q))) if q is not None else None
            keep += [db, qb]
            arr[i] = _Sequence(ctypes.addressof(db), ctypes.addressof(qb) if qb is not None else None, len(d),
                               int(e.get("forward", 1)), int(e.get("reverse", 0)))
        self._check(self.lib.rb_sequences_stage(self.ptr, arr, n))
        self._seq_lengths = [len(_b(e["data"]) or b"") for e in sequences]

    def poa_stage_overlaps(self, n_targets, overlaps, quality_threshold=10.0, tgs=True, trim=True):
        """overlaps: dicts with q_id, t_id, strand and breakpoints, a list of
        (t, q) points (first match, last match + 1 per window). Stages the
        consensus of every window over the first n_targets staged sequences
        with the layers assembled on the device (rb_poa_stage_overlaps)."""
        n = len(overlaps)
        arr = (_LayerOverlap * max(1, n))()
        flat, offs = [], [0]
        for i, o in enumerate(overlaps):
            arr[i] = _LayerOverlap(o["q_id"], o["t_id"], int(o.get("strand", 0)))
            for t, q in o["breakpoints"]:
                flat += [t, q]
            offs.append(len(flat))
        bp = (ctypes.c_uint32 * max(1, len(flat)))(*flat)
        off = (ctypes.c_uint64 * len(offs))(*offs)
        self._check(self.lib.rb_poa_stage_overlaps(self.ptr, n_targets, arr, n, bp, off, quality_threshold,
                                                   int(tgs), int(trim)))
        w = self.window_length
        self._staged_windows = sum((n + w - 1) // w for n in self._seq_lengths[:n_targets])
        return self._staged_windows

    @staticmethod
    def _store_pairs(pairs):
        arr = (_StorePair * max(1, len(pairs)))()
        for i, p in enumerate(pairs):
            arr[i] = _StorePair(p["q_id"], p["q_begin"], p["q_end"], p["t_id"], p["t_begin"], p["t_end"],
                                int(p.get("strand", 0)))
        return arr

    def align_overlaps(self, pairs, want_cigar=True):
        """Aligns pairs cut from the staged sequence table (dicts with q_id,
        q_begin, q_end, t_id, t_begin, t_end, strand; forward coordinates):
        rb_align_stage_overlaps + rb_align_run + rb_align_fetch."""
        arr = self._store_pairs(pairs)
        self._check(self.lib.rb_align_stage_overlaps(self.ptr, arr, len(pairs), int(want_cigar)))
        self._check(self.lib.rb_align_run(self.ptr))
        r = _AlnResult()
        self._check(self.lib.rb_align_fetch(self.ptr, ctypes.byref(r)))
        return self._aln_out(r, len(pairs), want_cigar)

    def poa_stage_alignments(self, n_targets, pairs, quality_threshold=10.0, tgs=True, trim=True):
        """Aligns the pairs from the staged table and stages window consensus
        with their breaking points turned into layers on the device
        (rb_poa_stage_alignments). Returns [(edit distance, breakpoints)]."""
        arr = self._store_pairs(pairs)
        r = _AlnResult()
        self._check(self.lib.rb_poa_stage_alignments(self.ptr, n_targets, arr, len(pairs), quality_threshold,
                                                     int(tgs), int(trim), ctypes.byref(r)))
        w = self.window_length
        self._staged_windows = sum((n + w - 1) // w for n in self._seq_lengths[:n_targets])
        return [(x["edit_distance"], x["breakpoints"]) for x in self._aln_out(r, len(pairs), False)]

    def poa_stage_job_device(self, job, trim=True, quality_threshold=None):
        """Stages a Job's windows through the device layer assembly: its
        sequence table to the device store, then its overlaps' breaking
        points (host buffers, copies included)."""
        inp = job.layer_input()
        self._check(self.lib.rb_sequences_stage(self.ptr, inp["sequences"], inp["n_sequences"]))
        q = job.quality_threshold if quality_threshold is None else quality_threshold
        self._check(self.lib.rb_poa_stage_overlaps(self.ptr, inp["n_targets"], inp["overlaps"], inp["n_overlaps"],
                                                   inp["breakpoints"], inp["bp_offsets"], q, inp["tgs"],
                                                   int(trim)))
        self._staged_windows = job.n

    def layer_stats(self):
        s = Stats()
        self._check(self.lib.rb_layer_stats(self.ptr, ctypes.byref(s)))
        return s

    def sequence_stats(self):
        s = Stats()
        self._check(self.lib.rb_sequence_stats(self.ptr, ctypes.byref(s)))
        return s

    def set_yield(self, consensus_windows, alignment_items):
        """Work a warp takes per launch (0: persistent kernels); rb_set_yield."""
        self._check(self.lib.rb_set_yield(self.ptr, consensus_windows, alignment_items))

    def set_sm_share(self, percent):
        """Percent of the SMs the persistent kernels fill; rb_set_sm_share."""
        self._check(self.lib.rb_set_sm_share(self.ptr, percent))

    def autotune(self, consensus=True, alignment=False):
        """rb_autotune on the staged batch(es): keeps the fastest launch
        choices for the device; returns them as a dict."""
        self._check(self.lib.rb_autotune(self.ptr, (1 if consensus else 0) | (2 if alignment else 0)))
        return tuning_get(self.device)

    def set_priority(self, high):
        """High- or normal-priority stream for this context; rb_set_priority."""
        self._check(self.lib.rb_set_priority(self.ptr, int(high)))

    def poa_stats(self):
        s = Stats()
        self._check(self.lib.rb_poa_stats(self.ptr, ctypes.byref(s)))
        return s

    def align_stats(self):
        s = Stats()
        self._check(self.lib.rb_align_stats(self.ptr, ctypes.byref(s)))
        return s


def polish_files(sequences, overlaps, targets, fragment=False, window_length=500, quality_threshold=10.0,
                 error_threshold=0.3, trim=True, match=3, mismatch=-5, gap=-4, threads=1,
                 drop_unpolished=True, device=0, stage_seconds=None):
    """racon's pipeline on the device; returns the polished FASTA text."""
    lib = load()
    out = ctypes.c_void_p()
    st = (ctypes.c_double * 4)()
    rc = lib.rb_polish_files(_b(sequences), _b(overlaps), _b(targets), int(fragment), window_length,
                             quality_threshold, error_threshold, int(trim), match, mismatch, gap, threads,
                             int(drop_unpolished), device, ctypes.byref(out), st)
    if rc != RB_OK:
        raise RaconB200Error(rc, lib.rb_pipeline_error().decode())
    try:
        text = ctypes.string_at(out.value).decode()
    finally:
        lib.rb_free(out)
    if stage_seconds is not None:
        stage_seconds[:] = list(st)
    return text


class Job:
    """racon's initialize() with the device aligner (rb_job_prepare): loading,
    overlap filtering, breaking points, windows and layers. .windows / .n are
    the rb_window views of every window, in racon's order."""

    def __init__(self, sequences, overlaps, targets, fragment=False, window_length=500, quality_threshold=10.0,
                 error_threshold=0.3, match=3, mismatch=-5, gap=-4, device=0):
        self.lib = load()
        st = (ctypes.c_double * 3)()
        self.ptr = self.lib.rb_job_prepare(_b(sequences), _b(overlaps), _b(targets), int(fragment), window_length,
                                           quality_threshold, error_threshold, match, mismatch, gap, device, st)
        if not self.ptr:
            raise RaconB200Error(1, self.lib.rb_pipeline_error().decode())
        self.stage_seconds = list(st)
        self.quality_threshold = quality_threshold
        wp = ctypes.POINTER(_Window)()
        self.n = self.lib.rb_job_windows(self.ptr, ctypes.byref(wp))
        self.windows = wp

    def close(self):
        if self.ptr:
            self.lib.rb_job_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def window(self, i):
        """Window i as a dict (backbone, backbone_quality, layers, qualities,
        begins, ends, tgs, id, rank)."""
        w = self.windows[i]
        bl = w.backbone_length
        bb = ctypes.string_at(w.backbone, bl)
        bq = ctypes.string_at(w.backbone_quality, bl) if w.backbone_quality else None
        layers, quals, begins, ends = [], [], [], []
        for j in range(w.n_layers):
            ln = w.layer_lengths[j]
            layers.append(ctypes.string_at(w.layers[j], ln))
            q = w.layer_qualities[j] if w.layer_qualities else None
            quals.append(ctypes.string_at(q, ln) if q else None)
            begins.append(w.begins[j])
            ends.append(w.ends[j])
        return {"backbone": bb, "backbone_quality": bq, "layers": layers, "qualities": quals, "begins": begins,
                "ends": ends, "tgs": w.tgs, "id": w.id, "rank": w.rank}

    def device_stats(self):
        """Counters of the job's own device work: {"align", "layers",
        "sequences"} -> Stats (rb_align_stats, rb_layer_stats and
        rb_sequence_stats of the job's context; align covers the last batch)."""
        ctx = self.lib.rb_job_context(self.ptr)
        out = {}
        for name, fn in (("align", self.lib.rb_align_stats), ("layers", self.lib.rb_layer_stats),
                         ("sequences", self.lib.rb_sequence_stats)):
            s = Stats()
            fn(ctypes.c_void_p(ctx), ctypes.byref(s))
            out[name] = s
        return out

    def layer_input(self):
        """The job as device layer assembly input (rb_job_layer_input): ctypes
        views of its sequence table, overlaps and breaking points."""
        seqs = ctypes.POINTER(_Sequence)()
        ovl = ctypes.POINTER(_LayerOverlap)()
        bp = ctypes.POINTER(ctypes.c_uint32)()
        off = ctypes.POINTER(ctypes.c_uint64)()
        ns, nt, no = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
        tgs = ctypes.c_int()
        rc = self.lib.rb_job_layer_input(self.ptr, ctypes.byref(seqs), ctypes.byref(ns), ctypes.byref(nt),
                                         ctypes.byref(ovl), ctypes.byref(no), ctypes.byref(bp), ctypes.byref(off),
                                         ctypes.byref(tgs))
        if rc != RB_OK:
            raise RaconB200Error(rc, "rb_job_layer_input failed")
        return {"sequences": seqs, "n_sequences": ns.value, "n_targets": nt.value, "overlaps": ovl,
                "n_overlaps": no.value, "breakpoints": bp, "bp_offsets": off, "tgs": tgs.value}

    def layer_stats(self):
        """(windows, layers, layer bases, backbone bases)."""
        nl = lb = bb = 0
        for i in range(self.n):
            w = self.windows[i]
            nl += w.n_layers
            bb += w.backbone_length
            lb += sum(w.layer_lengths[j] for j in range(w.n_layers))
        return self.n, nl, lb, bb


class Server:
    """Serving loop (rb_server_*): polishing jobs submitted while others run.

    workers jobs run at once, each on a long-lived device context of its own;
    queued jobs are admitted first in first out when a worker is idle and the
    job's estimated device footprint fits in hbm_budget beside the jobs in
    flight. With shared_consensus (the default) one persistent consensus
    kernel takes the windows of every job in flight from a shared device
    queue (continuous batching); jobs of at most priority_windows windows go
    first. With shared_alignment (the default) one persistent alignment
    kernel does the same for the jobs' overlap alignments (jobs of at most
    priority_pairs pairs first; spans up to alignment_max_span bases). With
    large_first_every = k, every k-th warp of both kernels takes the largest
    jobs first. submit() returns a ticket; wait(ticket) returns (fasta, times)."""

    def __init__(self, device=0, workers=4, hbm_budget=0, match=3, mismatch=-5, gap=-4, window_length=500,
                 shared_consensus=True, consensus_ctas_per_sm=0, priority_windows=0, alignment_yield=0,
                 alignment_share=0, shared_alignment=True, alignment_ctas_per_sm=0, alignment_max_span=0,
                 priority_pairs=0, large_first_every=0):
        self.lib = load()
        p = _ServerParams(device, workers, hbm_budget, match, mismatch, gap, window_length, int(shared_consensus),
                          consensus_ctas_per_sm, priority_windows, alignment_yield, alignment_share,
                          int(shared_alignment), alignment_ctas_per_sm, alignment_max_span, priority_pairs,
                          large_first_every)
        self.ptr = self.lib.rb_server_create(ctypes.byref(p))
        if not self.ptr:
            msg = self.lib.rb_server_error().decode() or self.lib.rb_create_error().decode()
            raise RaconB200Error(5, msg)

    def submit(self, sequences, overlaps, targets, fragment=False, quality_threshold=10.0, error_threshold=0.3,
               trim=True, drop_unpolished=True):
        j = _ServerJob(_b(sequences), _b(overlaps), _b(targets), int(fragment), quality_threshold,
                       error_threshold, int(trim), int(drop_unpolished))
        t = ctypes.c_uint64()
        rc = self.lib.rb_server_submit(self.ptr, ctypes.byref(j), ctypes.byref(t))
        if rc != RB_OK:
            raise RaconB200Error(rc, self.lib.rb_server_error().decode())
        return t.value

    def wait(self, ticket):
        out = ctypes.c_void_p()
        tm = ServerTimes()
        rc = self.lib.rb_server_wait(self.ptr, ticket, ctypes.byref(out), ctypes.byref(tm))
        if rc != RB_OK:
            raise RaconB200Error(rc, self.lib.rb_server_error().decode())
        try:
            text = ctypes.string_at(out.value).decode()
        finally:
            self.lib.rb_free(out)
        return text, {"submitted": tm.submitted, "admitted": tm.admitted, "finished": tm.finished,
                      "stage_seconds": list(tm.stage_seconds), "footprint": tm.footprint, "worker": tm.worker}

    def load(self):
        q, f, b = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint64()
        self.lib.rb_server_load(self.ptr, ctypes.byref(q), ctypes.byref(f), ctypes.byref(b))
        return q.value, f.value, b.value

    def close(self):
        if self.ptr:
            self.lib.rb_server_destroy(self.ptr)
            self.ptr = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tuning_get(device=0):
    """The device's launch choices (rb_tuning_get) as a dict."""
    t = Tuning()
    rc = load().rb_tuning_get(device, ctypes.byref(t))
    if rc != RB_OK:
        raise RaconB200Error(rc, "rb_tuning_get failed")
    return t.as_dict()


def tuning_set(device=0, **values):
    """Pins some of the device's launch choices (rb_tuning_set); the others
    keep their current values."""
    cur = tuning_get(device)
    cur.update(values)
    t = Tuning(**{k: cur[k] for k, _ in Tuning._fields_})
    rc = load().rb_tuning_set(device, ctypes.byref(t))
    if rc != RB_OK:
        raise RaconB200Error(rc, "rb_tuning_set failed")
