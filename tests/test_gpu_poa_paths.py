"""Window consensus on the less travelled device paths, against the oracle
(byte-identical): graphs that outgrow the starting slot (overflow and retry
with four times the capacity, and the global-memory forms of the adjacency
lists and descriptors), scores with match below mismatch (every layer takes
the chunked DP with byte decisions), and all-zero scores (every cell ties, so
spoa's tie-breaking decides everything)."""
import random

import pytest

pytestmark = pytest.mark.gpu


def _mutate(rng, s, err):
    out = []
    for c in s:
        u = rng.random()
        if u < err / 3:
            continue
        out.append(rng.choice("ACGT") if u < 2 * err / 3 else c)
        if rng.random() < err / 3:
            out.append(rng.choice("ACGT"))
    return "".join(out) or "A"


def _window(rng, bl, nl, err, partial=True, qual=True):
    truth = "".join(rng.choice("ACGT") for _ in range(bl))
    bb = _mutate(rng, truth, 0.03)[:65535]
    n = len(bb)
    layers, quals, begins, ends = [], [], [], []
    for k in range(nl):
        if partial and k % 3 == 0 and n > 20:
            b = rng.randint(0, n // 3)
            e = rng.randint(2 * n // 3, n - 1)
        else:
            b, e = 0, n - 1
        lo, hi = b * len(truth) // n, max(b * len(truth) // n + 1, (e + 1) * len(truth) // n)
        s = _mutate(rng, truth[lo:hi], err)
        layers.append(s)
        quals.append("".join(chr(33 + rng.randint(3, 40)) for _ in s) if qual else None)
        begins.append(b)
        ends.append(e)
    return {"backbone": bb, "backbone_quality": None, "layers": layers, "qualities": quals, "begins": begins,
            "ends": ends, "tgs": 1}


def _compare(native_lib, oracle_lib, wins, m, x, g, w=500, trim=True):
    with native_lib.Context(0, m, x, g, w) as ctx:
        got = ctx.poa(wins, trim=trim)
        st = ctx.poa_stats()
    bad = [i for i, (win, gv) in enumerate(zip(wins, got))
           if oracle_lib.window_consensus(win, m, x, g, trim)[:2] != gv]
    assert not bad, "%d of %d windows differ: %s" % (len(bad), len(wins), bad[:10])
    return st


def test_deep_window_overflow_retry(native_lib, oracle_lib, monkeypatch):
    # 200 reads at 25% error over 400 bases: about 1800 nodes, beyond what the
    # shared-memory lists and descriptors hold (global-memory forms). A
    # 1024-node starting slot makes the window overflow and run again.
    rng = random.Random(5)
    wins = [_window(rng, 400, 200, 0.25), _window(rng, 300, 12, 0.1)]
    monkeypatch.setenv("RB_POA_NCAP", "1024")
    st = _compare(native_lib, oracle_lib, wins, 3, -5, -4)
    assert st.max_nodes == 4096
    assert st.launches == 2
    monkeypatch.delenv("RB_POA_NCAP")
    st = _compare(native_lib, oracle_lib, wins, 3, -5, -4)
    assert st.launches == 1


@pytest.mark.parametrize("m,x,g", [(-1, 2, -3), (0, 0, 0), (2, 2, -1)])
def test_unusual_scores(native_lib, oracle_lib, m, x, g):
    rng = random.Random(7 + m)
    wins = [_window(rng, rng.randint(30, 200), rng.randint(2, 14), 0.15, qual=k % 2 == 0) for k in range(24)]
    _compare(native_lib, oracle_lib, wins, m, x, g, trim=bool(m % 2))
