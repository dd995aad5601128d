"""Small FASTA/FASTQ/PAF readers used by the tests to build device inputs."""
import gzip


def _open(path):
    return gzip.open(path, "rt") if path.endswith(".gz") else open(path)


def read_fastx(path):
    """{name: (sequence upper-case, quality or None)}; names end at whitespace."""
    out = {}
    with _open(path) as fh:
        lines = [l.rstrip("\n\r") for l in fh]
    i = 0
    if lines and lines[0].startswith(">"):
        name, seq = None, []
        for l in lines:
            if l.startswith(">"):
                if name is not None:
                    out[name] = ("".join(seq).upper(), None)
                name, seq = l[1:].split()[0], []
            else:
                seq.append(l.strip())
        if name is not None:
            out[name] = ("".join(seq).upper(), None)
        return out
    while i < len(lines):
        if not lines[i].startswith("@"):
            i += 1
            continue
        name = lines[i][1:].split()[0]
        i += 1
        seq = []
        while not lines[i].startswith("+"):
            seq.append(lines[i].strip())
            i += 1
        i += 1
        s = "".join(seq)
        q = []
        while sum(len(x) for x in q) < len(s):
            q.append(lines[i].strip())
            i += 1
        qual = "".join(q)
        if all(c == "!" for c in qual):
            qual = None
        out[name] = (s.upper(), qual)
    return out


def revcomp(s):
    t = {"A": "T", "T": "A", "C": "G", "G": "C"}
    return "".join(t.get(c, c) for c in reversed(s))


def read_paf(path):
    rows = []
    with _open(path) as fh:
        for l in fh:
            f = l.rstrip("\n").split("\t")
            if len(f) < 12:
                continue
            rows.append({"q": f[0], "ql": int(f[1]), "qb": int(f[2]), "qe": int(f[3]), "strand": f[4] == "-",
                         "t": f[5], "tl": int(f[6]), "tb": int(f[7]), "te": int(f[8])})
    return rows


def paf_pairs(reads, targets, rows):
    """Device pairs as racon cuts them (src/overlap.cpp:193-197)."""
    pairs = []
    for r in rows:
        if r["q"] == r["t"]:
            continue
        q = reads[r["q"]][0]
        t = targets[r["t"]][0]
        if r["strand"]:
            qs = revcomp(q)[r["ql"] - r["qe"]:r["ql"] - r["qb"]]
            qoff = r["ql"] - r["qe"]
        else:
            qs = q[r["qb"]:r["qe"]]
            qoff = r["qb"]
        pairs.append({"query": qs, "target": t[r["tb"]:r["te"]], "q_offset": qoff, "t_begin": r["tb"],
                      "row": r})
    return pairs
