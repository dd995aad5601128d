// ORACLE — test infrastructure only (see edlib_nw.hpp).
//
// Restatement of edlib's NW path algorithm. Structure:
//   band_sweep()        one banded Myers sweep over the target columns
//                       (k bound, Ukkonen block band, optional stop column,
//                       optional storage of every column for traceback)
//   traceback_stored()  walk back from the last cell over stored columns,
//                       preferring up (I), then left (D), then diagonal
//   split_hirschberg()  forward sweep over the left half + reverse sweep over
//                       the right half, first query row whose two halves sum
//                       to the known score, recurse on both quadrants
//   align_known()       choose traceback (stored data < 1 MiB) or Hirschberg
//   nw_align()          k doubling from 64 until the band holds a solution,
//                       then align_known() with the exact distance.
#include "edlib_nw.hpp"

#include <algorithm>
#include <cstdlib>
#include <cstring>

namespace oracle {
namespace {

using Word = uint64_t;
constexpr int kW = 64;
constexpr Word kHigh = Word(1) << 63;

inline int ceil_div(int a, int b) { return a % b ? a / b + 1 : a / b; }

struct Block {
    Word pv = 0, mv = 0;  // vertical +1 / -1 delta bits, bit i = row i of block
    int score = 0;        // score of the block's last row
};

// One column step of a 64-row block (Myers/Hyyro). hin in {-1,0,+1} is the
// horizontal delta of the row above the block; returns the delta of the last
// row of the block.
inline int block_step(Word& pv, Word& mv, Word eq, int hin) {
    const Word neg_in = hin < 0 ? 1 : 0;
    const Word xv = eq | mv;
    eq |= neg_in;
    const Word xh = (((eq & pv) + pv) ^ pv) | eq;
    Word ph = mv | ~(xh | pv);
    Word mh = pv & xh;
    int hout = 0;
    if (ph & kHigh) hout = 1;
    if (mh & kHigh) hout = -1;
    ph <<= 1;
    mh <<= 1;
    mh |= neg_in;
    if (hin > 0) ph |= 1;
    pv = mh | ~(xv | ph);
    mv = ph & xv;
    return hout;
}

// Values of the 64 rows of a block, index i = row (63 - i) of the block.
inline void block_rows_desc(const Block& b, int* out) {
    int s = b.score;
    Word mask = kHigh;
    for (int i = 0; i < kW - 1; ++i) {
        out[i] = s;
        if (b.pv & mask) --s;
        if (b.mv & mask) ++s;
        mask >>= 1;
    }
    out[kW - 1] = s;
}

inline bool block_all_above(const Block& b, int k) {
    int v[kW];
    block_rows_desc(b, v);
    for (int i = 0; i < kW; ++i)
        if (v[i] <= k) return false;
    return true;
}

// Query bit masks: eq[sym * nblocks + b], bit i set when query row 64b+i
// equals sym; rows past the query end act as wildcards (all symbols match).
struct Profile {
    int nblocks = 0;
    int pad = 0;
    std::vector<Word> eq;
    Profile(const uint8_t* q, int m, int alphabet) {
        nblocks = ceil_div(m, kW);
        pad = nblocks * kW - m;
        eq.assign(size_t(alphabet + 1) * nblocks, 0);
        for (int s = 0; s <= alphabet; ++s) {
            for (int b = 0; b < nblocks; ++b) {
                Word w = 0;
                for (int r = (b + 1) * kW - 1; r >= b * kW; --r) {
                    w <<= 1;
                    if (s == alphabet || r >= m || q[r] == s) w |= 1;
                }
                eq[size_t(s) * nblocks + b] = w;
            }
        }
    }
};

struct Stored {
    int nblocks = 0;
    std::vector<Word> pv, mv;
    std::vector<int> score, first, last;
    void init(int nb, int ncols) {
        nblocks = nb;
        pv.assign(size_t(nb) * ncols, 0);
        mv.assign(size_t(nb) * ncols, 0);
        score.assign(size_t(nb) * ncols, 0);
        first.assign(ncols, 0);
        last.assign(ncols, -1);
    }
};

struct SweepOut {
    int best = -1;  // score at (m-1, n-1), -1 when not within k
    // filled when stop_col >= 0: the band of that column
    std::vector<Block> stop_blocks;
    int stop_first = 0, stop_last = -1;
};

// Banded sweep. stop_col >= 0 stops after that column and reports its band;
// store != nullptr keeps every column for traceback.
void band_sweep(const Profile& prof, int m, const uint8_t* t, int n, int k,
                int stop_col, Stored* store, SweepOut& out) {
    constexpr int kStrongReduce = 2048;
    out = SweepOut();
    if (k < std::abs(n - m)) return;
    const int nb = prof.nblocks, pad = prof.pad;
    k = std::min(k, std::max(m, n));
    int first = 0;
    int last = std::min(nb, ceil_div(std::min(k, (k + m - n) / 2) + 1, kW)) - 1;
    std::vector<Block> blk(nb);
    for (int b = 0; b <= last; ++b) {
        blk[b].score = (b + 1) * kW;
        blk[b].pv = ~Word(0);
        blk[b].mv = 0;
    }
    if (store) store->init(nb, n);

    for (int c = 0; c < n; ++c) {
        const Word* eqc = &prof.eq[size_t(t[c]) * nb];
        int hout = 1;
        for (int b = first; b <= last; ++b) {
            hout = block_step(blk[b].pv, blk[b].mv, eqc[b], hout);
            blk[b].score += hout;
        }
        // tighten k with the best completion through the last block
        k = std::min(k, blk[last].score +
                            std::max(n - c - 1, m - ((1 + last) * kW - 1) - 1) +
                            (last == nb - 1 ? pad : 0));
        // grow the band by one block at the bottom when it is not beneath it
        if (last + 1 < nb &&
            !((last + 1) * kW - 1 > k - blk[last].score + 2 * kW - 2 - n + c + m)) {
            ++last;
            blk[last].pv = ~Word(0);
            blk[last].mv = 0;
            const int nh = block_step(blk[last].pv, blk[last].mv, eqc[last], hout);
            blk[last].score = blk[last - 1].score - hout + kW + nh;
            hout = nh;
        }
        // shrink from the bottom
        while (last >= first &&
               (blk[last].score >= k + kW ||
                ((last + 1) * kW - 1 > k - blk[last].score + 2 * kW - 2 - n + c + m + 1)))
            --last;
        // shrink from the top
        while (first <= last &&
               (blk[first].score >= k + kW ||
                ((first + 1) * kW - 1 < blk[first].score - k - n + m + c)))
            ++first;
        if (c % kStrongReduce == 0) {
            while (last >= 0 && last >= first && block_all_above(blk[last], k)) --last;
            while (first <= last && block_all_above(blk[first], k)) ++first;
        }
        if (last < first) return;  // no solution within k

        if (store) {
            for (int b = first; b <= last; ++b) {
                const size_t at = size_t(c) * nb + b;
                store->pv[at] = blk[b].pv;
                store->mv[at] = blk[b].mv;
                store->score[at] = blk[b].score;
            }
            store->first[c] = first;
            store->last[c] = last;
        }
        if (c == stop_col) {
            out.stop_blocks.assign(blk.begin(), blk.end());
            out.stop_first = first;
            out.stop_last = last;
            return;
        }
    }
    if (last == nb - 1) {
        int v[kW];
        block_rows_desc(blk[last], v);
        if (v[pad] <= k) out.best = v[pad];
    }
}

// Walk back from (m-1, n-1) over stored columns. Appends ops in reverse order.
bool traceback_stored(int m, int n, int best, const Stored& st,
                      std::vector<uint8_t>& rev) {
    const int nb = st.nblocks;
    const int pad = nb * kW - m;
    int c = n - 1, b = nb - 1, cur = best;
    int l_score = -1, u_score = -1, ul_score = -1;
    auto in_band = [&](int col, int blkid) {
        return blkid >= st.first[col] && blkid <= st.last[col];
    };
    Word cp = st.pv[size_t(c) * nb + b], cm = st.mv[size_t(c) * nb + b];
    bool has_left = c > 0 && in_band(c - 1, b);
    Word lp = 0, lm = 0;
    if (has_left) {
        lp = st.pv[size_t(c - 1) * nb + b];
        lm = st.mv[size_t(c - 1) * nb + b];
    }
    cp <<= pad;
    cm <<= pad;
    int pos = kW - pad - 1;  // row of the current cell inside block b

    while (true) {
        if (c == 0) {
            has_left = true;
            l_score = b * kW + pos + 1;
            ul_score = l_score - 1;
        }
        if (l_score == -1 && has_left) {
            l_score = st.score[size_t(c - 1) * nb + b];
            for (int i = 0; i < kW - pos - 1; ++i) {
                if (lp & kHigh) --l_score;
                if (lm & kHigh) ++l_score;
                lp <<= 1;
                lm <<= 1;
            }
        }
        if (ul_score == -1) {
            if (l_score != -1) {
                ul_score = l_score;
                if (lp & kHigh) --ul_score;
                if (lm & kHigh) ++ul_score;
            } else if (c > 0 && in_band(c - 1, b - 1)) {
                ul_score = st.score[size_t(c - 1) * nb + b - 1];
            }
        }
        if (u_score == -1) {
            u_score = cur;
            if (cp & kHigh) --u_score;
            if (cm & kHigh) ++u_score;
            cp <<= 1;
            cm <<= 1;
        }

        if (u_score != -1 && u_score + 1 == cur) {  // up: query base unmatched
            cur = u_score;
            l_score = ul_score;
            u_score = ul_score = -1;
            if (pos == 0) {
                if (b == 0) {
                    rev.push_back(kInsert);
                    for (int i = 0; i < c + 1; ++i) rev.push_back(kDelete);
                    break;
                }
                pos = kW - 1;
                --b;
                cp = st.pv[size_t(c) * nb + b];
                cm = st.mv[size_t(c) * nb + b];
                if (c > 0 && in_band(c - 1, b)) {
                    has_left = true;
                    lp = st.pv[size_t(c - 1) * nb + b];
                    lm = st.mv[size_t(c - 1) * nb + b];
                } else {
                    has_left = false;
                }
            } else {
                --pos;
                lp <<= 1;
                lm <<= 1;
            }
            rev.push_back(kInsert);
        } else if (l_score != -1 && l_score + 1 == cur) {  // left: target base
            cur = l_score;
            u_score = ul_score;
            l_score = ul_score = -1;
            --c;
            if (c == -1) {
                rev.push_back(kDelete);
                const int up = b * kW + pos + 1;
                for (int i = 0; i < up; ++i) rev.push_back(kInsert);
                break;
            }
            cp = lp;
            cm = lm;
            if (c > 0 && in_band(c - 1, b)) {
                has_left = true;
                lp = st.pv[size_t(c - 1) * nb + b];
                lm = st.mv[size_t(c - 1) * nb + b];
            } else if (c == 0) {
                has_left = true;
                l_score = b * kW + pos + 1;
                ul_score = l_score - 1;
            } else {
                has_left = false;
            }
            rev.push_back(kDelete);
        } else if (ul_score != -1) {  // diagonal
            const uint8_t op = ul_score == cur ? kMatch : kMismatch;
            cur = ul_score;
            u_score = l_score = ul_score = -1;
            --c;
            if (c == -1) {
                rev.push_back(op);
                const int up = b * kW + pos;
                for (int i = 0; i < up; ++i) rev.push_back(kInsert);
                break;
            }
            if (pos == 0) {
                if (b == 0) {
                    rev.push_back(op);
                    for (int i = 0; i < c + 1; ++i) rev.push_back(kDelete);
                    break;
                }
                pos = kW - 1;
                --b;
                cp = st.pv[size_t(c) * nb + b];
                cm = st.mv[size_t(c) * nb + b];
            } else {
                --pos;
                cp = lp;
                cm = lm;
                cp <<= 1;
                cm <<= 1;
            }
            if (c > 0 && in_band(c - 1, b)) {
                has_left = true;
                lp = st.pv[size_t(c - 1) * nb + b];
                lm = st.mv[size_t(c - 1) * nb + b];
            } else if (c == 0) {
                has_left = true;
                l_score = b * kW + pos + 1;
                ul_score = l_score - 1;
            } else {
                has_left = false;
            }
            rev.push_back(op);
        } else {
            break;  // no move left: cannot happen for a correct band
        }
    }
    return true;
}

bool align_known(const uint8_t* q, const uint8_t* rq, int m, const uint8_t* t,
                 const uint8_t* rt, int n, int alphabet, int best,
                 std::vector<uint8_t>& out);

bool split_hirschberg(const uint8_t* q, const uint8_t* rq, int m,
                      const uint8_t* t, const uint8_t* rt, int n, int alphabet,
                      int best, std::vector<uint8_t>& out) {
    const Profile fwd(q, m, alphabet), rev(rq, m, alphabet);
    const int nb = fwd.nblocks, pad = fwd.pad;
    const int lw = n / 2, rw = n - lw;
    SweepOut lo, ro;
    band_sweep(fwd, m, t, n, best, lw - 1, nullptr, lo);
    band_sweep(rev, m, rt, n, best, rw - 1, nullptr, ro);
    if (lo.stop_last < lo.stop_first || ro.stop_last < ro.stop_first) return false;

    // left column scores by query row (ascending)
    const int lf = lo.stop_first, ll = lo.stop_last;
    std::vector<int> left((ll - lf + 1) * kW);
    for (int b = lf; b <= ll; ++b) {
        int v[kW];
        block_rows_desc(lo.stop_blocks[b], v);
        for (int i = 0; i < kW; ++i) left[(b - lf) * kW + (kW - 1 - i)] = v[i];
    }
    const int left_start = lf * kW;
    int left_len = (ll - lf + 1) * kW;
    if (ll == nb - 1) left_len -= pad;

    // right column scores, reversed back to forward query rows
    const int rf = ro.stop_first, rl = ro.stop_last;
    std::vector<int> right_all((rl - rf + 1) * kW);
    for (int b = rf; b <= rl; ++b) {
        int v[kW];
        block_rows_desc(ro.stop_blocks[b], v);
        for (int i = 0; i < kW; ++i) right_all[(rl - b) * kW + i] = v[i];
    }
    const int* right = right_all.data();
    int right_start = m - (rl + 1) * kW;
    int right_len = (rl - rf + 1) * kW;
    if (right_start < 0) {
        right += pad;
        right_start += pad;
        right_len -= pad;
    }

    const int qs = std::max(left_start, right_start - 1);
    const int qe = std::min(left_start + left_len - 1, right_start + right_len - 2);
    int lscore = -1, rscore = -1, split = -1;
    bool found = false;
    for (int qi = qs; qi <= qe; ++qi) {
        lscore = left[qi - left_start];
        rscore = right[qi + 1 - right_start];
        if (lscore + rscore == best) {
            split = qi;
            found = true;
            break;
        }
    }
    if (!found && left_start == 0 && right_start == 0) {
        lscore = lw;
        rscore = right[0];
        if (lscore + rscore == best) {
            split = -1;
            found = true;
        }
    }
    if (!found && left_start + left_len == m && right_start + right_len == m) {
        lscore = left[left_len - 1];
        rscore = rw;
        if (lscore + rscore == best) {
            split = m - 1;
            found = true;
        }
    }
    if (!found) return false;

    const int uh = split + 1, lh = m - uh;
    std::vector<uint8_t> ul, lr;
    if (!align_known(q, rq + lh, uh, t, rt + rw, lw, alphabet, lscore, ul)) return false;
    if (!align_known(q + uh, rq, lh, t + lw, rt, rw, alphabet, rscore, lr)) return false;
    out.insert(out.end(), ul.begin(), ul.end());
    out.insert(out.end(), lr.begin(), lr.end());
    return true;
}

bool align_known(const uint8_t* q, const uint8_t* rq, int m, const uint8_t* t,
                 const uint8_t* rt, int n, int alphabet, int best,
                 std::vector<uint8_t>& out) {
    out.clear();
    if (m == 0 || n == 0) {
        out.assign(size_t(m + n), m == 0 ? kDelete : kInsert);
        return true;
    }
    const int nb = ceil_div(m, kW);
    const long long bytes = (2LL * sizeof(Word) + sizeof(int)) * nb * n;
    if (bytes < 1024 * 1024) {
        const Profile prof(q, m, alphabet);
        Stored st;
        SweepOut so;
        band_sweep(prof, m, t, n, best, -1, &st, so);
        std::vector<uint8_t> rev;
        if (!traceback_stored(m, n, best, st, rev)) return false;
        out.assign(rev.rbegin(), rev.rend());
        return true;
    }
    return split_hirschberg(q, rq, m, t, rt, n, alphabet, best, out);
}

}  // namespace

NwResult nw_align(const char* query, int m, const char* target, int n,
                  bool with_path) {
    NwResult res;
    // symbols numbered by first appearance, query first, then target
    int idx[256];
    std::fill(idx, idx + 256, -1);
    int alphabet = 0;
    std::vector<uint8_t> q(m), t(n);
    for (int i = 0; i < m; ++i) {
        const uint8_t c = uint8_t(query[i]);
        if (idx[c] < 0) idx[c] = alphabet++;
        q[i] = uint8_t(idx[c]);
    }
    for (int i = 0; i < n; ++i) {
        const uint8_t c = uint8_t(target[i]);
        if (idx[c] < 0) idx[c] = alphabet++;
        t[i] = uint8_t(idx[c]);
    }
    if (m == 0 || n == 0) {
        // edlib reports the distance and no alignment for an empty side
        res.edit_distance = std::max(m, n);
        res.ok = true;
        return res;
    }
    const Profile prof(q.data(), m, alphabet);
    int k = kW;
    SweepOut so;
    do {
        band_sweep(prof, m, t.data(), n, k, -1, nullptr, so);
        k *= 2;
    } while (so.best == -1);
    res.edit_distance = so.best;
    res.ok = true;
    if (!with_path) return res;
    std::vector<uint8_t> rq(q.rbegin(), q.rend()), rt(t.rbegin(), t.rend());
    res.ok = align_known(q.data(), rq.data(), m, t.data(), rt.data(), n, alphabet,
                         res.edit_distance, res.ops);
    return res;
}

std::string ops_to_cigar(const std::vector<uint8_t>& ops) {
    static const char kChar[4] = {'M', 'I', 'D', 'M'};
    std::string out;
    size_t i = 0;
    while (i < ops.size()) {
        const char ch = kChar[ops[i]];
        size_t j = i;
        while (j < ops.size() && kChar[ops[j]] == ch) ++j;
        out += std::to_string(j - i);
        out += ch;
        i = j;
    }
    return out;
}

}  // namespace oracle
