"""A restatement of racon's window creation and layer loop
(src/polisher.cpp:384-457 with Window::add_layer, src/window.cpp:42-63), for
tests: windows as dicts for racon_b200.Context.poa, in racon's window order,
each window's layers in the order racon appends them.

sequences: racon's sequence table (targets first) as dicts with data and
quality (str or bytes, quality None for FASTA or all-'!'), and optionally the
reverse complement "rc" and reversed quality "rquality" (computed from data
when absent). overlaps: dicts with q_id, t_id, strand and breakpoints, the
(t, q) points of find_breaking_points.
"""

COMP = {ord("A"): ord("T"), ord("T"): ord("A"), ord("C"): ord("G"), ord("G"): ord("C")}


def _bytes(x):
    if x is None:
        return None
    return x.encode("latin-1") if isinstance(x, str) else bytes(x)


def revcomp(data):
    b = _bytes(data)
    return bytes(COMP.get(c, c) for c in reversed(b))


def host_windows(sequences, n_targets, overlaps, w, q_thr, tgs):
    windows, first = [], []
    for t in range(n_targets):
        first.append(len(windows))
        d, qd = _bytes(sequences[t]["data"]), _bytes(sequences[t].get("quality"))
        for r, j in enumerate(range(0, len(d), w)):
            bl = min(j + w, len(d)) - j
            windows.append({"backbone": d[j:j + bl], "backbone_quality": qd[j:j + bl] if qd else None,
                            "layers": [], "qualities": [], "begins": [], "ends": [], "tgs": tgs, "id": t,
                            "rank": r})
    for o in overlaps:
        s = sequences[o["q_id"]]
        if o["strand"]:
            data = _bytes(s["rc"]) if s.get("rc") is not None else revcomp(s["data"])
            if s.get("rquality") is not None:
                qual = _bytes(s["rquality"])
            else:
                q = _bytes(s.get("quality"))
                qual = q[::-1] if q is not None else None
        else:
            data = _bytes(s["data"])
            qual = _bytes(s.get("quality"))
        bp = o["breakpoints"]
        for j in range(0, len(bp), 2):
            (t0, q0), (t1, q1) = bp[j], bp[j + 1]
            if q1 - q0 < 0.02 * w:
                continue
            if qual is not None:
                # (uint32)char - 33 summed into a double: exact integers
                total = 0
                for c in qual[q0:q1]:
                    signed = c - 256 if c >= 128 else c
                    total += (signed - 33) % (1 << 32)
                if total / (q1 - q0) < q_thr:
                    continue
            win = first[o["t_id"]] + t0 // w
            ws = (t0 // w) * w
            b, e = t0 - ws, t1 - ws - 1
            if b == e:
                continue
            W = windows[win]
            W["layers"].append(data[q0:q1])
            W["qualities"].append(qual[q0:q1] if qual is not None else None)
            W["begins"].append(b)
            W["ends"].append(e)
    return windows
