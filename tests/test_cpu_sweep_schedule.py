"""The overlap aligner's two sweep schedules (racon_b200/csrc/nw_align.cu),
restated in Python lane by lane: strips of 32 64-row blocks with carry
buffers between strips (warp_sweep), and one diagonal wavefront over all
blocks with a rotating shuffle from lane 31 to lane 0 (warp_sweep_diag, for
bands within 1900 diagonals). Both must compute the same (block, column)
states, the same distance and the same give-up row, for every band the
diagonal schedule accepts. This pins the schedule argument on the CPU; the
GPU parity tests check the kernels against the oracle."""
import random

M64 = (1 << 64) - 1
INT_MAX = 2**31 - 1
DIAG_BAND = 1900


def make_band(m, n, k):
    d = m - n
    return dict(m=m, n=n, k=k, dlo=-((k - d) // 2), dhi=(d + k) // 2, nb=(m + 63) // 64)


def myers_step(pv, mv, eq, hin):
    neg = 1 if hin < 0 else 0
    xv = eq | mv
    eq |= neg
    xh = ((((eq & pv) + pv) & M64) ^ pv) | eq
    ph = (mv | (~(xh | pv) & M64)) & M64
    mh = pv & xh
    hout = (ph >> 63) - (mh >> 63)
    ph2 = ((ph << 1) & M64) | (1 if hin > 0 else 0)
    mh2 = ((mh << 1) & M64) | neg
    return (mh2 | (~(xv | ph2) & M64)) & M64, ph2 & xv, hout


def block_value(pv, mv, score, i):
    if i == 63:
        return score
    return score - bin(pv >> (i + 1)).count("1") + bin(mv >> (i + 1)).count("1")


def masks(q, m, v, nsym):
    tab = [0] * nsym
    rows = min(64, m - 64 * v)
    for i in range(rows):
        tab[q[64 * v + i]] |= 1 << i
    if rows < 64:
        tab = [x | ((M64 << rows) & M64) for x in tab]
    return tab


def unpack(ip):
    return (ip & 3) - 1, (ip >> 2) & 1, ip >> 3


def strips(q, t, ncols, B, nsym, rev, trace):
    m, n, nb, dlo, dhi, k = B["m"], B["n"], B["nb"], B["dlo"], B["dhi"], B["k"]
    result = INT_MAX
    carry_h = [[0] * (ncols + 64) for _ in range(2)]
    carry_s = [[0] * (ncols + 64) for _ in range(2)]
    for s in range((nb + 31) // 32):
        s_lo = max(0, 2048 * s - dhi)
        s_hi = min(ncols - 1, 64 * min(nb - 1, 32 * s + 31) + 63 - dlo)
        if s_lo > s_hi:
            break
        prev_hi = min(ncols - 1, 2048 * s - 1 - dlo)
        lanes = []
        for lane in range(32):
            b = 32 * s + lane
            lanes.append(dict(b=b, ok=b < nb, lo=max(0, 64 * b - dhi), hi=min(ncols - 1, 64 * b + 63 - dlo),
                              eq=masks(q, m, b, nsym) if b < nb else None, pv=0, mv=0, sc=0, st=False, ip=0,
                              bmin=INT_MAX))
        cho, cso, chi, csi = carry_h[s & 1], carry_s[s & 1], carry_h[(s + 1) & 1], carry_s[(s + 1) & 1]
        for step in range((s_hi - s_lo) + 32):
            packs = []
            for lane, L in enumerate(lanes):
                c = s_lo + step - lane
                act = L["ok"] and L["lo"] <= c <= L["hi"]
                hout = 0
                if act:
                    up_h, up_p, up_s = unpack(L["ip"])
                    if lane == 0:
                        hin = 1 if (s == 0 or c > prev_hi) else chi[c]
                    else:
                        hin = up_h if up_p else 1
                    if not L["st"]:
                        L["st"], L["pv"], L["mv"] = True, M64, 0
                        if c == 0:
                            L["sc"] = 64 * (L["b"] + 1)
                        else:
                            L["sc"] = (csi[c - 1] if lane == 0 else (up_s - up_h if up_p else up_s)) + 64
                    tc = t[n - 1 - c] if rev else t[c]
                    L["pv"], L["mv"], hout = myers_step(L["pv"], L["mv"], L["eq"][tc], hin)
                    L["sc"] += hout
                    trace.append((L["b"], c, L["pv"], L["mv"], L["sc"]))
                    if L["b"] == nb - 1 and c == n - 1:
                        result = block_value(L["pv"], L["mv"], L["sc"], (m - 1) & 63)
                    if lane == 31:
                        L["bmin"] = min(L["bmin"], L["sc"])
                        cho[c], cso[c] = hout, L["sc"]
                packs.append((L["sc"] << 3) | ((1 if act else 0) << 2) | (hout + 1))
            for lane in range(32):
                lanes[lane]["ip"] = packs[lane - 1] if lane > 0 else packs[0]
        if 32 * s + 31 < nb - 1:
            R = 64 * (32 * s + 31) + 63
            if lanes[31]["bmin"] > k and R + 1 > k:
                return INT_MAX, (R, lanes[31]["bmin"])
    return result, None


def diagonal(q, t, ncols, B, nsym, rev, trace):
    m, n, nb, dlo, dhi, k = B["m"], B["n"], B["nb"], B["dlo"], B["dhi"], B["k"]
    tbl = [masks(q, m, v, nsym) for v in range(nb)]
    last = lambda v: min(ncols - 1, 64 * v + 63 - dlo) + v
    v_last = min(nb - 1, (ncols - 1 + dhi) // 64)
    t_stop = last(v_last)
    g_last = 32 * (v_last // 32) + 31
    if g_last < nb - 1:
        t_stop = max(t_stop, last(g_last))
    chk_v, result = 31, INT_MAX
    lanes = [dict(v=l, lo=max(0, 64 * l - dhi), hi=min(ncols - 1, 64 * l + 63 - dlo), pv=0, mv=0, sc=0, st=False,
                  ip=0, bmin=INT_MAX) for l in range(32)]
    for step in range(t_stop + 1):
        packs = []
        for lane, L in enumerate(lanes):
            c = step - L["v"]
            if c > L["hi"]:
                L["v"] += 32
                c -= 32
                L["lo"], L["hi"] = max(0, 64 * L["v"] - dhi), min(ncols - 1, 64 * L["v"] + 63 - dlo)
                L["st"], L["bmin"] = False, INT_MAX
            v = L["v"]
            act = v < nb and L["lo"] <= c <= L["hi"]
            hout = 0
            if act:
                up_h, up_p, up_s = unpack(L["ip"])
                hin = 1 if (v == 0 or not up_p) else up_h
                if not L["st"]:
                    L["st"], L["pv"], L["mv"] = True, M64, 0
                    L["sc"] = 64 * (v + 1) if c == 0 else (up_s - up_h if up_p else up_s) + 64
                tc = t[n - 1 - c] if rev else t[c]
                L["pv"], L["mv"], hout = myers_step(L["pv"], L["mv"], tbl[v][tc], hin)
                L["sc"] += hout
                trace.append((v, c, L["pv"], L["mv"], L["sc"]))
                if v == nb - 1 and c == n - 1:
                    result = block_value(L["pv"], L["mv"], L["sc"], (m - 1) & 63)
                if lane == 31:
                    L["bmin"] = min(L["bmin"], L["sc"])
            packs.append((L["sc"] << 3) | ((1 if act else 0) << 2) | (hout + 1))
        for lane in range(32):
            lanes[lane]["ip"] = packs[(lane + 31) & 31]
        if step == last(chk_v):
            if chk_v < nb - 1:
                R = 64 * chk_v + 63
                if lanes[31]["bmin"] > k and R + 1 > k:
                    return INT_MAX, (R, lanes[31]["bmin"])
            chk_v += 32
    return result, None


def _mutate(rng, s, e, nsym):
    out = []
    for c in s:
        u = rng.random()
        if u < e / 4:
            continue
        out.append(rng.randrange(nsym) if u < e * 3 / 4 else c)
        if rng.random() < e / 4:
            out.append(rng.randrange(nsym))
    return out or [0]


def test_diagonal_schedule_equals_strips():
    rng = random.Random(5)
    checked = 0
    for n, err, nsym, cut in [(40, 0.1, 4, False), (700, 0.2, 5, False), (2500, 0.1, 4, False),
                              (2300, 0.3, 8, True), (130, 0.4, 4, False), (2200, 0.15, 4, False)]:
        t = [rng.randrange(nsym) for _ in range(n)]
        q = _mutate(rng, t, err, nsym)
        if cut:
            q = q[: len(q) // 3]
        m = len(q)
        base = max(64, abs(m - n))
        for k in sorted({base, min(2 * base, 1800), rng.randint(base, base + 1200)}):
            B = make_band(m, n, k)
            if B["dhi"] > DIAG_BAND or B["dhi"] - B["dlo"] > DIAG_BAND:
                continue
            for rev, ncols in ((False, n), (False, max(1, n // 2)), (True, max(1, n - n // 2))):
                ta, tb = [], []
                ra = strips(q, t, ncols, B, nsym, rev, ta)
                rb = diagonal(q, t, ncols, B, nsym, rev, tb)
                if ncols == n and not rev:
                    assert ra == rb, (m, n, k)
                if ra[1] is None and rb[1] is None:
                    assert sorted(ta) == sorted(tb), (m, n, k, rev, ncols)
                checked += 1
    assert checked >= 20
