"""The consensus DP's cross-lane horizontal scan (racon_b200/csrc/poa_consensus.cu,
dp_layer_fast), restated in Python: the max-plus prefix of 32 lane aggregates
with a uniform penalty per lane, computed by rounds of offset 1, 2, 4, 8, 16
that stop at the first round in which no lane changes. It must equal the
exact prefix max over m <= l of (x_m + (l - m) * penalty) on every input,
including minus-infinity lanes, and never need more than five rounds."""
import random

NEG_INF = -(1 << 29)


def doubling_scan(x, pen):
    x = list(x)
    rounds = 0
    o = 1
    while o < 32:
        rounds += 1
        y = [NEG_INF if l < o else x[l - o] for l in range(32)]
        nx = [max(y[l] + o * pen, x[l]) for l in range(32)]
        changed = any(a != b for a, b in zip(nx, x))
        x = nx
        if not changed:
            break
        o <<= 1
    return x, rounds


def exact_prefix(x, pen):
    return [max(x[m] + (l - m) * pen for m in range(l + 1)) for l in range(32)]


def test_doubling_scan_with_early_exit_is_exact():
    rng = random.Random(9)
    for it in range(3000):
        pen = -rng.choice([1, 4, 8, 20, 96])  # S x gap for S = 4..24, gap -1..-4
        kind = it % 4
        if kind == 0:    # scores near each other: few changes
            x = [rng.randint(-50, 50) for _ in range(32)]
        elif kind == 1:  # a high lane far left: its run crosses many lanes
            x = [rng.randint(-5000, -4000) for _ in range(32)]
            x[rng.randint(0, 8)] = rng.randint(0, 100)
        elif kind == 2:  # decreasing to the right by more than the penalty
            base = rng.randint(0, 100)
            x = [base + l * pen * 2 + rng.randint(-3, 3) for l in range(32)]
        else:            # minus-infinity lanes mixed in
            x = [NEG_INF if rng.random() < 0.3 else rng.randint(-300, 300) for _ in range(32)]
        got, rounds = doubling_scan(x, pen)
        assert got == exact_prefix(x, pen)
        assert rounds <= 5
