// Overlap alignment on the device: edit distance, alignment path and window
// breaking points with the semantics of racon's
//   src/overlap.cpp:205-224  edlibAlign(NW, PATH, k = -1) + standard CIGAR
//   src/overlap.cpp:226-292  find_breaking_points_from_cigar
//
// Design (B200, sm_100a). One warp owns one subproblem at a time; warps are
// persistent and pull work from an atomic queue (pairs sorted by size).
//
// * Block sweep. The query is cut into 64-row blocks (one uint64 of vertical
//   +1/-1 delta bits per block, Myers 1999 / Hyyro). Blocks are grouped into
//   strips of 32, one block per lane; a strip is swept as a diagonal wavefront
//   (lane l works on column c - l), the horizontal carry of each column moves
//   one lane down per step through a warp shuffle, and the bottom lane's carry
//   is kept in a per-warp column buffer for the next strip.
// * Band. Only blocks that meet the Ukkonen band of the subproblem are
//   computed: a cell (r, c) can lie on a path of cost <= k only if
//   |r - c| + |(m - n) - (r - c)| <= k, i.e. r - c in
//   [ceil((m-n-k)/2), floor((m-n+k)/2)]. Cells outside the band are taken as
//   the cost of a real (not necessarily optimal) path, so every computed value
//   is an upper bound and every cell on an optimal path is exact. Therefore
//   the edit distance, the Hirschberg split row and every traceback decision
//   equal those of the unbanded dynamic program.
// * Distance. k doubles from max(64, |m - n|) until the band holds the corner
//   (the first k >= distance returns the exact distance).
// * Path. edlib's recursion is followed exactly: a subproblem is traced back
//   from stored columns when (2*8+4) * ceil(m/64) * n < 1 MiB, else it is
//   split at target column n/2: forward sweep of the left half and reverse
//   sweep of the right half capture one column each, the split row is the
//   first query row whose two halves sum to the subproblem's score, then the
//   row -1 and row m-1 boundaries. Levels of the recursion tree are processed
//   breadth-first, one launch per level.
// * Traceback. The leaf sweep stores, per (column, band block), the vertical
//   +1 bits after the step and the horizontal +1 bits of the step. At a cell
//   the walk moves up (query base inserted) if the vertical bit is set, left
//   (target base deleted) if the horizontal bit is set, else diagonally -
//   edlib's preference order. The 32 lanes prefetch 32 columns; the row is
//   passed lane to lane.
// * Output. The path is recorded as mq[t] = matched query position or -1 for
//   every target position. An optimal alignment never has an insertion next
//   to a deletion (a diagonal step is cheaper), so the op string, the CIGAR
//   and racon's breaking points all follow from mq.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

#include "rb_internal.hpp"
#include "ring_queue.cuh"

namespace rb {
namespace {

typedef unsigned long long u64;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarpsPerBlock = 4;
constexpr int kMaxSym = 32;        // symbols whose bit masks fit the shared-memory table
constexpr int kMaxSymWide = 256;   // any byte alphabet: the masks then live in the warp's scratch
constexpr long long kLeafBytes = 1024 * 1024;  // edlib's traceback threshold
// The diagonal sweep (warp_sweep_diag) handles alphabets of up to kDiagSym
// symbols and bands whose diagonals stay within kDiagBand of the main one.
constexpr int kDiagSym = 8;
constexpr int kDiagBand = 1900;

enum NwStatus : int {
    kNwOk = 0,
    kNwSplitMissing = 1,
    kNwTraceOutOfBand = 2,
    kNwTaskOverflow = 3,
    kNwBadSymbol = 4,
};

struct NwTask {
    uint32_t pair;
    uint32_t qa, m;
    uint32_t ta, n;
    int32_t score;
};

struct NwDevArgs {
    const uint8_t* codes;
    const NwPairDev* pairs;
    const uint32_t* order;
    uint32_t npairs;
    int32_t* dist;
    int32_t* mq;
    uint32_t* bp;
    uint32_t* bp_count;
    uint32_t window_length;
    // per-warp scratch
    uint8_t* scratch;
    size_t scratch_stride;
    uint32_t scratch_warps;
    uint32_t max_n, max_nb;
    // work queues
    unsigned int* counters;  // [0] pair/task cursor, [1] next-level count, [2] status
    const NwTask* tasks_in;
    uint32_t ntasks_in;
    NwTask* tasks_out;
    uint32_t tasks_out_cap;
    uint32_t per_warp_cap;   // pairs / tasks a warp takes per launch (0: until the queue is empty)
};

__device__ __forceinline__ int fdiv64(int a) { return a >= 0 ? a / 64 : -((-a + 63) / 64); }
__device__ __forceinline__ int fdiv2(int a) { return a >= 0 ? a / 2 : -((-a + 1) / 2); }

struct Band {
    int m, n, k, dlo, dhi, nb;
};

__device__ __forceinline__ Band make_band(int m, int n, int k) {
    Band B;
    B.m = m;
    B.n = n;
    B.k = k;
    const int d = m - n;
    B.dlo = -fdiv2(k - d);  // ceil((d - k) / 2)
    B.dhi = fdiv2(d + k);   // floor((d + k) / 2)
    B.nb = (m + 63) / 64;
    return B;
}
__device__ __forceinline__ int band_lo_block(const Band& B, int c) { return max(0, fdiv64(c + B.dlo)); }
__device__ __forceinline__ int band_hi_block(const Band& B, int c) {
    return min(B.nb - 1, fdiv64(c + B.dhi));
}

__device__ __forceinline__ int myers_step(u64& pv, u64& mv, u64 eq, int hin, u64& ph_out) {
    const u64 neg = hin < 0 ? 1ull : 0ull;
    const u64 xv = eq | mv;
    eq |= neg;
    const u64 xh = (((eq & pv) + pv) ^ pv) | eq;
    u64 ph = mv | ~(xh | pv);
    u64 mh = pv & xh;
    ph_out = ph;
    const int hout = int(ph >> 63) - int(mh >> 63);
    ph = (ph << 1) | (hin > 0 ? 1ull : 0ull);
    mh = (mh << 1) | neg;
    pv = mh | ~(xv | ph);
    mv = ph & xv;
    return hout;
}

// Value of row i (0..63) of a block whose last row holds `score`.
__device__ __forceinline__ int block_value(u64 pv, u64 mv, int score, int i) {
    if (i == 63) return score;
    return score - __popcll(pv >> (i + 1)) + __popcll(mv >> (i + 1));
}

__device__ __forceinline__ void set_status(unsigned int* counters, int code) {
    atomicCAS(&counters[2], 0u, unsigned(code));
}

// Per-warp scratch layout.
struct WarpScratch {
    int8_t* carry_h[2];
    int32_t* carry_s[2];
    u64* capl_pv;
    u64* capl_mv;
    int32_t* capl_sc;
    u64* capr_pv;
    u64* capr_mv;
    int32_t* capr_sc;
    uint4* leaf;  // followed by the [kMaxSymWide][32] bit masks of pairs with more than kMaxSym symbols
    u64* block_peq;  // [max_nb][kDiagSym] query masks per block (diagonal sweep); nullptr: strips only
};

// Bit masks of a wide-alphabet pair: the region after the leaf store.
__device__ __forceinline__ u64* peq_wide(const WarpScratch& ws) {
    return reinterpret_cast<u64*>(reinterpret_cast<uint8_t*>(ws.leaf) + kLeafBytes);
}

__device__ WarpScratch warp_scratch(const NwDevArgs& a, uint32_t slot) {
    uint8_t* p = a.scratch + size_t(slot) * a.scratch_stride;
    WarpScratch w;
    const size_t n = a.max_n, nb = a.max_nb;
    auto take = [&](size_t bytes) {
        uint8_t* r = p;
        p += (bytes + 255) & ~size_t(255);
        return r;
    };
    w.carry_h[0] = reinterpret_cast<int8_t*>(take(n));
    w.carry_h[1] = reinterpret_cast<int8_t*>(take(n));
    w.carry_s[0] = reinterpret_cast<int32_t*>(take(n * 4));
    w.carry_s[1] = reinterpret_cast<int32_t*>(take(n * 4));
    w.capl_pv = reinterpret_cast<u64*>(take(nb * 8));
    w.capl_mv = reinterpret_cast<u64*>(take(nb * 8));
    w.capl_sc = reinterpret_cast<int32_t*>(take(nb * 4));
    w.capr_pv = reinterpret_cast<u64*>(take(nb * 8));
    w.capr_mv = reinterpret_cast<u64*>(take(nb * 8));
    w.capr_sc = reinterpret_cast<int32_t*>(take(nb * 4));
    w.leaf = reinterpret_cast<uint4*>(take(kLeafBytes));  // kLeafBytes is a multiple of 256
    take(size_t(kMaxSymWide) * 32 * 8);                     // wide-alphabet masks (peq_wide)
    w.block_peq = reinterpret_cast<u64*>(take(nb * kDiagSym * 8));
    return w;
}

size_t warp_scratch_bytes(size_t n, size_t nb) {
    auto r = [](size_t b) { return (b + 255) & ~size_t(255); };
    return 2 * r(n) + 2 * r(n * 4) + 2 * (2 * r(nb * 8) + r(nb * 4)) + r(kLeafBytes) +
           r(size_t(kMaxSymWide) * 32 * 8) + r(nb * kDiagSym * 8);
}

enum SweepMode { kDistance = 0, kCapture = 1, kLeaf = 2 };

struct SweepIO {
    const uint8_t* q;  // subproblem query codes (forward start)
    const uint8_t* t;  // subproblem target codes (forward start)
    bool rev;          // sweep the reversed subproblem
    int ncols;         // columns swept: [0, ncols)
    int nsym;
    u64* peq;          // shared memory, [kMaxSym][32] per warp
    u64* cap_pv;
    u64* cap_mv;
    int32_t* cap_sc;
    uint4* leaf;
    int bw;            // leaf: blocks stored per column
};

// Where a kDistance sweep gave up: the bottom row of the strip whose cells
// all exceeded k, and their minimum (row = -1: it did not give up early).
struct SweepFail {
    int row = -1;
    int min = 0;
};

// The banded block sweep below (warp_sweep) as one diagonal wavefront over
// all blocks instead of strips, for narrow bands. Block v runs on lane
// v % 32 and meets column c at step c + v, so it gets the carry of block
// v - 1 at the same column from the lane before at the previous step (lane
// 31 to lane 0 by a rotating shuffle, no carry buffer), and a lane moves on
// to block v + 32 when block v leaves the band. With both band edges within
// kDiagBand (< 1953) diagonals of the main one, block v + 32 starts at least
// 32 steps after block v ends, and block v + 31 (the next block of the lane
// before) starts only after the last step at which block v reads its carry,
// so a lane never holds two blocks at once and the carry it reads is always
// block v - 1's. The steps are about n + m / 64 instead of
// (m / 2048) * (2048 + k) for strips, and every cell gets the same inputs
// as in the strip sweep (the carry of the block above at the same column,
// +1 where that block is outside the band, the block's first score from the
// block above one column to the left), so every value, the give-up checks
// and their rows are the strip sweep's. Query masks come from a per-block
// table built once per sweep (at most kDiagSym symbols). A form with two
// blocks in flight per lane (two slots, bands up to 3900 diagonals) gave the
// same cells but was slower than strips on the config-2 batch (18217
// against 19101 pairs/s at 20000 pairs): the per-slot bookkeeping outweighs
// the second chain.
__device__ __forceinline__ bool diag_sweep_ok(const SweepIO& io, const Band& B, const WarpScratch& ws) {
    return ws.block_peq != nullptr && io.nsym <= kDiagSym && B.dhi <= kDiagBand && B.dhi - B.dlo <= kDiagBand;
}

template <int MODE>
__device__ int warp_sweep_diag(const SweepIO& io, const Band& B, const WarpScratch& ws, int lane,
                               SweepFail* fail) {
    const int m = B.m, n = B.n, nb = B.nb, nsym = io.nsym;
    const int ncols = io.ncols;
    // masks of every block (lane v % 32 builds block v, and only it reads
    // them back), built in the lane's column of the shared table
    for (int v0 = 0; v0 < nb; v0 += 32) {
        const int v = v0 + lane;
        if (v < nb) {
            for (int sym = 0; sym < nsym; ++sym) io.peq[sym * 32 + lane] = 0ull;
            const int r0 = 64 * v;
            const int rows = min(64, m - r0);
            for (int i = 0; i < rows; ++i) {
                const int r = r0 + i;
                const int code = io.rev ? io.q[m - 1 - r] : io.q[r];
                io.peq[code * 32 + lane] |= (1ull << i);
            }
            const u64 pad = rows < 64 ? (~0ull << rows) : 0ull;  // rows past the query end match anything
            for (int sym = 0; sym < nsym; ++sym) ws.block_peq[v * kDiagSym + sym] = io.peq[sym * 32 + lane] | pad;
        }
    }
    // the last block that meets the swept columns, and the last step; a
    // distance sweep also runs to the last step of the bottom block of that
    // block's 32-block group, where the strip sweep checks the group's row
    const int v_last = min(nb - 1, (ncols - 1 + B.dhi) / 64);
    auto last_step = [&](int v) { return min(ncols - 1, 64 * v + 63 - B.dlo) + v; };
    int t_stop = last_step(v_last);
    const int g_last = 32 * (v_last / 32) + 31;
    if (MODE == kDistance && g_last < nb - 1) t_stop = max(t_stop, last_step(g_last));
    int chk_v = 31;                  // next group-bottom block whose row is checked
    int chk_t = last_step(chk_v);    // ... at the end of this step
    int result = INT_MAX;
    int v = lane;
    int cb_lo = max(0, 64 * v - B.dhi), cb_hi = min(ncols - 1, 64 * v + 63 - B.dlo);
    const u64* mask = ws.block_peq + v * kDiagSym;
    u64 pv = 0, mv = 0;
    int score = 0;
    bool started = false;
    int bottom_min = INT_MAX;  // kDistance, lane 31: minimum of its block's bottom row
    int in_pack = 0;           // previous step of the lane before: (score << 3) | (processed << 2) | (hout + 1)
    const int src = (lane + 31) & 31;
    for (int t = 0; t <= t_stop; ++t) {
        int c = t - v;
        if (c > cb_hi) {  // the lane's block left the band: its next block
            v += 32;
            c -= 32;
            cb_lo = max(0, 64 * v - B.dhi);
            cb_hi = min(ncols - 1, 64 * v + 63 - B.dlo);
            mask = ws.block_peq + v * kDiagSym;
            started = false;
            bottom_min = INT_MAX;
        }
        const bool active = v < nb && c >= cb_lo && c <= cb_hi;
        int hout = 0;
        if (active) {
            const int up_h = (in_pack & 3) - 1;
            const bool up_proc = (in_pack >> 2) & 1;
            const int up_score = in_pack >> 3;
            const int hin = (v == 0 || !up_proc) ? 1 : up_h;
            if (!started) {
                started = true;
                pv = ~0ull;
                mv = 0ull;
                score = c == 0 ? 64 * (v + 1) : (up_proc ? up_score - up_h : up_score) + 64;
            }
            const int tc = io.rev ? io.t[n - 1 - c] : io.t[c];
            const u64 eq = mask[tc];
            u64 ph;
            hout = myers_step(pv, mv, eq, hin, ph);
            score += hout;
            if (MODE == kLeaf) {
                const int blo = band_lo_block(B, c);
                io.leaf[size_t(c) * io.bw + (v - blo)] =
                    make_uint4(unsigned(pv), unsigned(pv >> 32), unsigned(ph), unsigned(ph >> 32));
            }
            if (MODE == kCapture && c == ncols - 1) {
                io.cap_pv[v] = pv;
                io.cap_mv[v] = mv;
                io.cap_sc[v] = score;
            }
            if (MODE == kDistance && v == nb - 1 && c == n - 1) {
                result = block_value(pv, mv, score, (m - 1) & 63);
            }
            if (MODE == kDistance && lane == 31) bottom_min = min(bottom_min, score);
        }
        const int pack = (score << 3) | ((active ? 1 : 0) << 2) | (hout + 1);
        in_pack = __shfl_sync(kFull, pack, src);
        if (MODE == kDistance && t == chk_t) {
            // the group whose bottom block is chk_v is done (the strip
            // sweep's check after that strip)
            if (chk_v < nb - 1) {
                const int row_min = __shfl_sync(kFull, bottom_min, 31);
                const int R = 64 * chk_v + 63;
                if (row_min > B.k && R + 1 > B.k) {
                    if (fail) {
                        fail->row = R;
                        fail->min = row_min;
                    }
                    result = INT_MAX;
                    break;
                }
            }
            chk_v += 32;
            chk_t = last_step(chk_v);
        }
    }
    if (MODE == kDistance) {
        for (int o = 16; o > 0; o >>= 1) result = min(result, __shfl_xor_sync(kFull, result, o));
    }
    return result;
}

// Banded block sweep of one subproblem by one warp. MODE kDistance returns
// the value of cell (m-1, n-1) (INT_MAX if the band never reached it). It
// also stops early, returning INT_MAX, once every computed cell of a full
// strip's bottom row R exceeds k and so does the left boundary (R + 1): costs
// never fall along a path, every path of cost <= k stays inside the band, and
// a computed in-band value is at most the cost of any path to it inside the
// band, so no path of cost <= k crosses row R. (Out-of-band cells only lower
// the minimum.) The distance of a pass that reaches the end is unchanged.
template <int MODE>
__device__ int warp_sweep(const SweepIO& io, const Band& B, const WarpScratch& ws, int lane,
                          unsigned int* counters, SweepFail* fail = nullptr) {
    if (diag_sweep_ok(io, B, ws)) return warp_sweep_diag<MODE>(io, B, ws, lane, fail);
    int result = INT_MAX;
    const int nstrips = (B.nb + 31) / 32;
    const int m = B.m, n = B.n;
    for (int s = 0; s < nstrips; ++s) {
        const int b = 32 * s + lane;
        const bool lane_valid = b < B.nb;
        const int cb_lo = max(0, 64 * b - B.dhi);
        const int cb_hi = min(io.ncols - 1, 64 * b + 63 - B.dlo);
        const int s_lo = max(0, 64 * 32 * s - B.dhi);
        const int last_b = min(B.nb - 1, 32 * s + 31);
        const int s_hi = min(io.ncols - 1, 64 * last_b + 63 - B.dlo);
        if (s_lo > s_hi) break;  // the band leaves the swept columns above this strip
        const int prev_hi = min(io.ncols - 1, 64 * 32 * s - 1 - B.dlo);

        // query bit masks of this lane's block
        for (int sym = 0; sym < io.nsym; ++sym) io.peq[sym * 32 + lane] = 0ull;
        if (lane_valid) {
            const int r0 = 64 * b;
            const int rows = min(64, m - r0);
            for (int i = 0; i < rows; ++i) {
                const int r = r0 + i;
                const int code = io.rev ? io.q[m - 1 - r] : io.q[r];
                io.peq[code * 32 + lane] |= (1ull << i);
            }
            if (rows < 64) {
                const u64 pad = ~0ull << rows;  // rows past the query end match anything
                for (int sym = 0; sym < io.nsym; ++sym) io.peq[sym * 32 + lane] |= pad;
            }
        }
        __syncwarp();

        u64 pv = 0, mv = 0;
        int score = 0;
        int bottom_min = INT_MAX;  // kDistance, lane 31: minimum of the strip's bottom row
        bool started = false;
        int in_pack = 0;  // previous step of lane-1: (score << 3) | (processed << 2) | (hout + 1)
        const int steps = (s_hi - s_lo) + 32;
        int8_t* carry_h_out = ws.carry_h[s & 1];
        int32_t* carry_s_out = ws.carry_s[s & 1];
        const int8_t* carry_h_in = ws.carry_h[(s + 1) & 1];
        const int32_t* carry_s_in = ws.carry_s[(s + 1) & 1];
        for (int st = 0; st < steps; ++st) {
            const int c = s_lo + st - lane;
            const bool active = lane_valid && c >= cb_lo && c <= cb_hi;
            int hout = 0;
            if (active) {
                const int up_h = (in_pack & 3) - 1;
                const bool up_proc = (in_pack >> 2) & 1;
                const int up_score = in_pack >> 3;
                int hin;
                if (lane == 0) {
                    hin = (s == 0 || c > prev_hi) ? 1 : int(carry_h_in[c]);
                } else {
                    hin = up_proc ? up_h : 1;
                }
                if (!started) {
                    started = true;
                    pv = ~0ull;
                    mv = 0ull;
                    if (c == 0) {
                        score = 64 * (b + 1);
                    } else {
                        const int v = (lane == 0) ? carry_s_in[c - 1]
                                                  : (up_proc ? up_score - up_h : up_score);
                        score = v + 64;
                    }
                }
                const int tc = io.rev ? io.t[n - 1 - c] : io.t[c];
                const u64 eq = io.peq[tc * 32 + lane];
                u64 ph;
                hout = myers_step(pv, mv, eq, hin, ph);
                score += hout;
                if (MODE == kLeaf) {
                    const int blo = band_lo_block(B, c);
                    io.leaf[size_t(c) * io.bw + (b - blo)] =
                        make_uint4(unsigned(pv), unsigned(pv >> 32), unsigned(ph), unsigned(ph >> 32));
                }
                if (MODE == kCapture && c == io.ncols - 1) {
                    io.cap_pv[b] = pv;
                    io.cap_mv[b] = mv;
                    io.cap_sc[b] = score;
                }
                if (MODE == kDistance && b == B.nb - 1 && c == n - 1) {
                    result = block_value(pv, mv, score, (m - 1) & 63);
                }
                if (MODE == kDistance && lane == 31) bottom_min = min(bottom_min, score);
                if (lane == 31) {
                    carry_h_out[c] = int8_t(hout);
                    carry_s_out[c] = score;
                }
            }
            const int pack = (score << 3) | ((active ? 1 : 0) << 2) | (hout + 1);
            in_pack = __shfl_up_sync(kFull, pack, 1);
        }
        __syncwarp();
        if (MODE == kDistance && 32 * s + 31 < B.nb - 1) {
            const int row_min = __shfl_sync(kFull, bottom_min, 31);
            const int R = 64 * (32 * s + 31) + 63;
            if (row_min > B.k && R + 1 > B.k) {
                if (fail) {
                    fail->row = R;
                    fail->min = row_min;
                }
                result = INT_MAX;
                break;
            }
        }
    }
    if (MODE == kDistance) {
        for (int o = 16; o > 0; o >>= 1) result = min(result, __shfl_xor_sync(kFull, result, o));
    }
    (void)counters;
    return result;
}

// k of the next distance pass after a pass with k failed: at least twice k;
// when the pass gave up at row f.row with minimum cost f.min, the cost per
// row so far projected over the longer side (x 1.1), up to 8k. Any k gives
// the same distance once k >= distance; this only picks how many passes.
__device__ __forceinline__ int next_k(int k, const SweepFail& f, int m, int n) {
    long long nk = 2LL * k;
    if (f.row >= 0) {
        const double est = double(f.min) * double(max(m, n)) / double(f.row + 1);
        const long long want = ((long long)(est * 1.1) + 63) / 64 * 64;
        nk = max(nk, min(8LL * k, want));
    }
    return int(min(nk, 1LL << 30));
}

__device__ void fill_deleted(int32_t* mq, int from, int count, int lane) {
    for (int i = lane; i < count; i += 32) mq[from + i] = -1;
}

// Leaf: store the band of every column, then walk back from (m-1, n-1).
__device__ void leaf_traceback(const NwDevArgs& a, const NwPairDev& P, const NwTask& T,
                               const WarpScratch& ws, u64* peq, int lane) {
    const int m = int(T.m), n = int(T.n);
    int32_t* mq = a.mq + P.mq_off + T.ta;
    const Band B = make_band(m, n, T.score);
    const int bw = min(B.nb, (B.dhi - B.dlo) / 64 + 2);
    SweepIO io;
    io.q = a.codes + P.q_off + T.qa;
    io.t = a.codes + P.t_off + T.ta;
    io.rev = false;
    io.ncols = n;
    io.nsym = int(P.nsym);
    io.peq = int(P.nsym) <= kMaxSym ? peq : peq_wide(ws);
    io.leaf = ws.leaf;
    io.bw = bw;
    warp_sweep<kLeaf>(io, B, ws, lane, a.counters);
    __syncwarp();

    int row = m - 1;
    int c0 = n - 1;
    while (c0 >= 0) {
        const int c = c0 - lane;
        const bool has = c >= 0;
        // prefetch the blocks holding the entry row and the one above it
        u64 pva = 0, pha = 0, pvb = 0, phb = 0;
        const int ba = row >= 0 ? row / 64 : -1;
        int clo = 0, chi = -1;
        if (has) {
            clo = band_lo_block(B, c);
            chi = band_hi_block(B, c);
            if (ba >= clo && ba <= chi) {
                const uint4 e = ws.leaf[size_t(c) * bw + (ba - clo)];
                pva = (u64(e.y) << 32) | e.x;
                pha = (u64(e.w) << 32) | e.z;
            }
            if (ba - 1 >= clo && ba - 1 <= chi) {
                const uint4 e = ws.leaf[size_t(c) * bw + (ba - 1 - clo)];
                pvb = (u64(e.y) << 32) | e.x;
                phb = (u64(e.w) << 32) | e.z;
            }
        }
        int r = row;
        int my_mq = -1;
        int r_out = r;
        for (int l = 0; l < 32; ++l) {
            if (c0 - l < 0) break;
            if (lane == l) {
                if (r < 0) {
                    my_mq = -1;
                    r_out = -1;
                } else {
                    int rr = r;
                    bool found = false;
                    while (rr >= 0) {
                        const int bb = rr >> 6, i = rr & 63;
                        u64 pvw, phw;
                        if (bb == ba) {
                            pvw = pva;
                            phw = pha;
                        } else if (bb == ba - 1) {
                            pvw = pvb;
                            phw = phb;
                        } else if (bb >= clo && bb <= chi) {
                            const uint4 e = ws.leaf[size_t(c) * bw + (bb - clo)];
                            pvw = (u64(e.y) << 32) | e.x;
                            phw = (u64(e.w) << 32) | e.z;
                        } else {
                            set_status(a.counters, kNwTraceOutOfBand);
                            break;
                        }
                        if (bb < clo || bb > chi) {
                            set_status(a.counters, kNwTraceOutOfBand);
                            break;
                        }
                        const u64 lowmask = (i == 63) ? ~0ull : ((2ull << i) - 1ull);
                        const u64 clear = ~pvw & lowmask;
                        if (clear) {
                            const int ip = 63 - __clzll(clear);
                            rr = 64 * bb + ip;
                            found = true;
                            if ((phw >> ip) & 1ull) {
                                my_mq = -1;
                                r_out = rr;
                            } else {
                                my_mq = rr;
                                r_out = rr - 1;
                            }
                            break;
                        }
                        rr = 64 * bb - 1;
                    }
                    if (!found) {
                        my_mq = -1;
                        r_out = -1;
                    }
                }
            }
            r = __shfl_sync(kFull, r_out, l);
        }
        if (has) mq[c] = my_mq >= 0 ? int(T.qa) + my_mq : -1;
        row = r;
        c0 -= 32;
    }
}

__device__ void hirschberg_split(const NwDevArgs& a, const NwPairDev& P, const NwTask& T,
                                 const WarpScratch& ws, u64* peq, int lane) {
    const int m = int(T.m), n = int(T.n);
    const int best = T.score;
    const int lw = n / 2, rw = n - lw;
    const Band B = make_band(m, n, best);
    SweepIO io;
    io.q = a.codes + P.q_off + T.qa;
    io.t = a.codes + P.t_off + T.ta;
    io.nsym = int(P.nsym);
    io.peq = int(P.nsym) <= kMaxSym ? peq : peq_wide(ws);
    io.leaf = nullptr;
    io.bw = 0;
    io.rev = false;
    io.ncols = lw;
    io.cap_pv = ws.capl_pv;
    io.cap_mv = ws.capl_mv;
    io.cap_sc = ws.capl_sc;
    warp_sweep<kCapture>(io, B, ws, lane, a.counters);
    io.rev = true;
    io.ncols = rw;
    io.cap_pv = ws.capr_pv;
    io.cap_mv = ws.capr_mv;
    io.cap_sc = ws.capr_sc;
    warp_sweep<kCapture>(io, B, ws, lane, a.counters);
    __syncwarp();

    const int llo = band_lo_block(B, lw - 1), lhi = band_hi_block(B, lw - 1);
    const int rlo = band_lo_block(B, rw - 1), rhi = band_hi_block(B, rw - 1);
    auto left = [&](int r) -> int {  // D(q[0..r], t[0..lw-1])
        const int bb = r >> 6;
        if (bb < llo || bb > lhi) return INT_MAX / 4;
        return block_value(ws.capl_pv[bb], ws.capl_mv[bb], ws.capl_sc[bb], r & 63);
    };
    auto right = [&](int r) -> int {  // D(q[r..m-1], t[lw..n-1])
        const int rr = m - 1 - r;
        const int bb = rr >> 6;
        if (bb < rlo || bb > rhi) return INT_MAX / 4;
        return block_value(ws.capr_pv[bb], ws.capr_mv[bb], ws.capr_sc[bb], rr & 63);
    };
    const int q_lo = max(max(0, 64 * llo), m - 2 - min(m - 1, 64 * rhi + 63));
    const int q_hi = min(min(m - 2, min(m - 1, 64 * lhi + 63)), m - 2 - 64 * rlo);
    int split = -2, ls = 0, rs = 0;
    for (int base = q_lo; base <= q_hi; base += 32) {
        const int qi = base + lane;
        int lv = 0, rv = 0;
        bool ok = false;
        if (qi <= q_hi) {
            lv = left(qi);
            rv = right(qi + 1);
            ok = lv + rv == best;
        }
        const unsigned hit = __ballot_sync(kFull, ok);
        if (hit) {
            const int src = __ffs(hit) - 1;
            split = base + src;
            ls = __shfl_sync(kFull, lv, src);
            rs = __shfl_sync(kFull, rv, src);
            break;
        }
    }
    if (split == -2) {
        const int rv = right(0);
        if (lw + rv == best) {
            split = -1;
            ls = lw;
            rs = rv;
        }
    }
    if (split == -2) {
        const int lv = left(m - 1);
        if (lv + rw == best) {
            split = m - 1;
            ls = lv;
            rs = rw;
        }
    }
    if (split == -2) {
        if (lane == 0) set_status(a.counters, kNwSplitMissing);
        return;
    }
    const int uh = split + 1;
    int32_t* mq = a.mq + P.mq_off;
    NwTask kids[2];
    kids[0] = NwTask{T.pair, T.qa, uint32_t(uh), T.ta, uint32_t(lw), ls};
    kids[1] = NwTask{T.pair, T.qa + uh, uint32_t(m - uh), T.ta + lw, uint32_t(rw), rs};
    for (int k = 0; k < 2; ++k) {
        const NwTask& K = kids[k];
        if (K.n == 0) continue;
        if (K.m == 0) {
            fill_deleted(mq, int(K.ta), int(K.n), lane);
            continue;
        }
        if (lane == 0) {
            const unsigned idx = atomicAdd(&a.counters[1], 1u);
            if (idx < a.tasks_out_cap) {
                a.tasks_out[idx] = K;
            } else {
                set_status(a.counters, kNwTaskOverflow);
            }
        }
    }
}

__device__ __forceinline__ bool is_leaf(uint32_t m, uint32_t n) {
    const long long nb = (m + 63) / 64;
    return (2LL * 8 + 4) * nb * n < kLeafBytes;
}

extern __shared__ u64 g_peq_smem[];

// Edit distance of pair pi by one warp (k doubling from max(64, |m - n|)),
// and, from lane 0, the pair's root task of the path recursion when both
// sides are non-empty (edlib returns no alignment for an empty side).
__device__ void distance_pair(const NwDevArgs& a, uint32_t pi, const WarpScratch& ws, u64* peq, int lane) {
    const NwPairDev P = a.pairs[pi];
    const int m = int(P.m), n = int(P.n);
    if (m == 0 || n == 0) {
        if (lane == 0) a.dist[pi] = max(m, n);
        return;
    }
    SweepIO io;
    io.q = a.codes + P.q_off;
    io.t = a.codes + P.t_off;
    io.rev = false;
    io.ncols = n;
    io.nsym = int(P.nsym);
    io.peq = int(P.nsym) > kMaxSym ? peq_wide(ws) : peq;
    io.leaf = nullptr;
    io.bw = 0;
    int k = max(64, abs(m - n));
    int d = INT_MAX;
    while (true) {
        const Band B = make_band(m, n, k);
        SweepFail f;
        d = warp_sweep<kDistance>(io, B, ws, lane, a.counters, &f);
        if (d <= k) break;
        k = next_k(k, f, m, n);
    }
    if (lane == 0) {
        a.dist[pi] = d;
        const unsigned idx = atomicAdd(&a.counters[1], 1u);
        if (idx < a.tasks_out_cap) {
            a.tasks_out[idx] = NwTask{pi, 0, P.m, 0, P.n, d};
        } else {
            set_status(a.counters, kNwTaskOverflow);
        }
    }
}

// Task i of the current recursion level: traceback of a leaf, or a
// Hirschberg split that appends the two halves to the next level.
__device__ void level_task(const NwDevArgs& a, uint32_t i, const WarpScratch& ws, u64* peq, int lane) {
    const NwTask T = a.tasks_in[i];
    const NwPairDev P = a.pairs[T.pair];
    if (is_leaf(T.m, T.n)) {
        leaf_traceback(a, P, T, ws, peq, lane);
    } else {
        hirschberg_split(a, P, T, ws, peq, lane);
    }
}

// Persistent distance pass of one engine: pairs in size order from an
// atomic cursor.
__global__ void __launch_bounds__(32 * kWarpsPerBlock)
nw_distance_kernel(NwDevArgs a) {
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const uint32_t slot = blockIdx.x * kWarpsPerBlock + wib;
    u64* peq = g_peq_smem + wib * kMaxSym * 32;
    const WarpScratch ws = warp_scratch(a, slot);
    for (uint32_t done = 0; a.per_warp_cap == 0 || done < a.per_warp_cap; ++done) {
        unsigned i = 0;
        if (lane == 0) i = atomicAdd(&a.counters[0], 1u);
        i = __shfl_sync(kFull, i, 0);
        if (i >= a.npairs) break;
        distance_pair(a, a.order[i], ws, peq, lane);
    }
}

// One recursion level of one engine: tasks from an atomic cursor.
__global__ void __launch_bounds__(32 * kWarpsPerBlock)
nw_level_kernel(NwDevArgs a) {
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const uint32_t slot = blockIdx.x * kWarpsPerBlock + wib;
    u64* peq = g_peq_smem + wib * kMaxSym * 32;
    const WarpScratch ws = warp_scratch(a, slot);
    for (uint32_t done = 0; a.per_warp_cap == 0 || done < a.per_warp_cap; ++done) {
        unsigned i = 0;
        if (lane == 0) i = atomicAdd(&a.counters[0], 1u);
        i = __shfl_sync(kFull, i, 0);
        if (i >= a.ntasks_in) break;
        level_task(a, i, ws, peq, lane);
        __syncwarp();
    }
}

}  // namespace

// One batch of the shared alignment queue (device record, written before
// its items are published): a distance pass over pairs, or one recursion
// level over tasks, of one engine's staged pairs.
struct NwJobDev {
    SvcJobHead head;
    uint32_t mode;           // 0: items are pair indices (distance), 1: task indices (level)
    uint32_t ntasks_in;
    uint32_t tasks_out_cap;
    uint32_t pad;
    const uint8_t* codes;
    const NwPairDev* pairs;
    int32_t* dist;
    int32_t* mq;
    unsigned int* counters;  // [1] tasks appended to tasks_out, [2] status
    const void* tasks_in;    // NwTask records of the level
    void* tasks_out;         // NwTask records of the next level
};

namespace {

constexpr uint32_t kJobDistance = 0, kJobLevel = 1;

// The alignment service's kernel arguments: the warps' scratch (sized for
// the service's longest span), the batch records, and the queue.
struct NwSvcArgs {
    NwDevArgs base;
    const NwJobDev* jobs;
    SvcQueueDev q;
};

// Persistent alignment over the shared queue: each warp owns one scratch
// slot and takes distance passes and recursion tasks of any job until the
// queue stays empty.
__global__ void __launch_bounds__(32 * kWarpsPerBlock)
nw_service_kernel(NwSvcArgs s) {
    __shared__ NwDevArgs a_all[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const uint32_t slot = blockIdx.x * kWarpsPerBlock + wib;
    u64* peq = g_peq_smem + wib * kMaxSym * 32;
    const WarpScratch ws = warp_scratch(s.base, slot);
    for (;;) {
        unsigned long long it = 0;
        if (lane == 0) it = svc_claim(s.q, slot);
        it = __shfl_sync(kFull, it, 0);
        if (it == ~0ull) break;
        const uint32_t job = uint32_t(it >> 32), idx = uint32_t(it);
        uint32_t mode = 0, total = 0, gen = 0;
        if (lane == 0) {
            // the record is rewritten for every batch that reuses the slot:
            // read it past L1
            const volatile NwJobDev& J = s.jobs[job];
            NwDevArgs a = s.base;
            a.codes = const_cast<const uint8_t*>(J.codes);
            a.pairs = const_cast<const NwPairDev*>(J.pairs);
            a.dist = const_cast<int32_t*>(J.dist);
            a.mq = const_cast<int32_t*>(J.mq);
            a.counters = const_cast<unsigned int*>(J.counters);
            a.tasks_in = static_cast<const NwTask*>(const_cast<const void*>(J.tasks_in));
            a.ntasks_in = J.ntasks_in;
            a.tasks_out = static_cast<NwTask*>(const_cast<void*>(J.tasks_out));
            a.tasks_out_cap = J.tasks_out_cap;
            mode = J.mode;
            total = J.head.total;
            gen = J.head.generation;
            a_all[wib] = a;
        }
        mode = __shfl_sync(kFull, mode, 0);
        __syncwarp();
        if (mode == kJobDistance) {
            distance_pair(a_all[wib], idx, ws, peq, lane);
        } else {
            level_task(a_all[wib], idx, ws, peq, lane);
        }
        __threadfence();
        __syncwarp();
        if (lane == 0) svc_item_done(s.q, job, total, gen);
    }
}

// Breaking points from mq: one window segment per floor(t / w); for each
// segment with a match, (first match t, q) and (last match t + 1, q + 1).
// Window breaking points of each pair from its match table, one warp per
// pair over 32-position chunks: racon's walk (src/overlap.cpp:244-290) emits,
// per window the target touches, the first matched (t, q) and the last
// matched (t + 1, q + 1). A matched position opens a window segment when the
// previous matched position (the highest matched lane below, or the carry of
// earlier chunks) lies in another window; it writes its segment's first pair
// and closes the previous segment's last pair.
__global__ void __launch_bounds__(256) nw_breakpoints_kernel(NwDevArgs a) {
    const int lane = threadIdx.x & 31;
    const unsigned below_mask = (1u << lane) - 1u;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < a.npairs; i += nwarps) {
        const NwPairDev P = a.pairs[i];
        uint32_t* out = a.bp + P.bp_off;
        uint32_t segs = 0;
        if (P.m != 0 && P.n != 0) {
            const int32_t* mq = a.mq + P.mq_off;
            const uint32_t w = a.window_length;
            uint32_t carry_sgm = 0xFFFFFFFFu, carry_t = 0, carry_q = 0;
            for (uint32_t c0 = 0; c0 < P.n; c0 += 32) {
                const uint32_t c = c0 + lane;
                const int32_t v = c < P.n ? mq[c] : -1;
                const bool matched = v >= 0;
                const uint32_t t = P.t_begin + c;
                const uint32_t q = P.q_offset + uint32_t(v);
                const uint32_t sgm = t / w;
                const unsigned mm = __ballot_sync(kFull, matched);
                const unsigned below = mm & below_mask;
                const int p = below ? 31 - __clz(below) : 0;
                const uint32_t p_sgm = __shfl_sync(kFull, sgm, p);
                const uint32_t p_t = __shfl_sync(kFull, t, p);
                const uint32_t p_q = __shfl_sync(kFull, q, p);
                const uint32_t prev_sgm = below ? p_sgm : carry_sgm;
                const bool first = matched && sgm != prev_sgm;
                const unsigned fm = __ballot_sync(kFull, first);
                if (first) {
                    const uint32_t idx = segs + __popc(fm & below_mask);
                    out[4 * idx] = t;
                    out[4 * idx + 1] = q;
                    if (idx > 0) {
                        out[4 * (idx - 1) + 2] = (below ? p_t : carry_t) + 1;
                        out[4 * (idx - 1) + 3] = (below ? p_q : carry_q) + 1;
                    }
                }
                segs += __popc(fm);
                if (mm) {
                    const int hl = 31 - __clz(mm);
                    carry_sgm = __shfl_sync(kFull, sgm, hl);
                    carry_t = __shfl_sync(kFull, t, hl);
                    carry_q = __shfl_sync(kFull, q, hl);
                }
            }
            if (segs > 0 && lane == 0) {
                out[4 * (segs - 1) + 2] = carry_t + 1;
                out[4 * (segs - 1) + 3] = carry_q + 1;
            }
        }
        if (lane == 0) a.bp_count[i] = 4 * segs;
    }
}

__device__ int put_run(char* dst, int pos, bool write, int len, char op) {
    char tmp[12];
    int d = 0;
    while (len > 0) {
        tmp[d++] = char('0' + len % 10);
        len /= 10;
    }
    if (write)
        for (int k = 0; k < d; ++k) dst[pos + k] = tmp[d - 1 - k];
    pos += d;
    if (write) dst[pos] = op;
    return pos + 1;
}

__device__ __forceinline__ int decimal_digits(uint32_t x) {
    int d = 1;
    while (x >= 10) {
        x /= 10;
        ++d;
    }
    return d;
}

// Standard CIGAR (M/I/D runs) of each pair from its match table, one warp
// per pair over 32-position chunks; write = 0 counts the characters into
// lens, write = 1 writes them at offs. The sequential walk it restates: per
// target position an insertion run before a matched position (the query
// positions skipped since the previous match), then M, or D when unmatched;
// equal neighbouring ops merge, and trailing query positions end with I.
// An M/D run therefore starts where the op changes or an insertion comes
// first; each such position closes the previous run and emits its own I run,
// and a warp prefix sum of their text lengths gives every lane's offset.
__global__ void __launch_bounds__(256) nw_cigar_kernel(NwDevArgs a, uint64_t* lens, const uint64_t* offs, char* out,
                                                       int write) {
    const int lane = threadIdx.x & 31;
    const unsigned below_mask = (1u << lane) - 1u;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < a.npairs; i += nwarps) {
        const NwPairDev P = a.pairs[i];
        if (P.m == 0 || P.n == 0) {
            if (!write && lane == 0) lens[i] = 0;
            continue;
        }
        const int32_t* mq = a.mq + P.mq_off;
        char* dst = write ? out + offs[i] : nullptr;
        const uint32_t n = P.n;
        uint64_t pos = 0;           // characters before this chunk
        int carry_v = -1;           // last matched query position so far
        int carry_op = -1;          // op of the position before the chunk (0 = M, 1 = D)
        uint32_t run_start = 0;     // first position of the open M/D run
        int run_op = -1;            // its op (-1: none yet)
        for (uint32_t c0 = 0; c0 < n; c0 += 32) {
            const uint32_t c = c0 + lane;
            const bool valid = c < n;
            const int v = valid ? mq[c] : -1;
            const bool matched = v >= 0;
            const int op = matched ? 0 : 1;
            const unsigned mm = __ballot_sync(kFull, matched);
            const unsigned mbelow = mm & below_mask;
            const int p_v = __shfl_sync(kFull, v, mbelow ? 31 - __clz(mbelow) : 0);
            const int prev_v = mbelow ? p_v : carry_v;
            const int ins = matched ? v - prev_v - 1 : 0;
            const int up_op = __shfl_up_sync(kFull, op, 1);
            const int prev_op = lane > 0 ? up_op : carry_op;
            const bool start = valid && (c == 0 || op != prev_op || ins > 0);
            const unsigned sm = __ballot_sync(kFull, start);
            const unsigned sbelow = sm & below_mask;
            const int ps = sbelow ? 31 - __clz(sbelow) : 0;
            const int ps_op = __shfl_sync(kFull, op, ps);
            const uint32_t prev_start = sbelow ? c0 + uint32_t(ps) : run_start;
            const int prev_run_op = sbelow ? ps_op : run_op;
            const bool close_prev = start && prev_run_op >= 0;
            const uint32_t close_len = c - prev_start;
            int tl = 0;
            if (close_prev) tl += decimal_digits(close_len) + 1;
            if (start && ins > 0) tl += decimal_digits(uint32_t(ins)) + 1;
            int x = tl;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int y = __shfl_up_sync(kFull, x, d);
                if (lane >= d) x += y;
            }
            const int total = __shfl_sync(kFull, x, 31);
            if (write && tl) {
                int at = int(pos) + x - tl;
                if (close_prev) at = put_run(dst, at, true, int(close_len), prev_run_op ? 'D' : 'M');
                if (ins > 0) put_run(dst, at, true, ins, 'I');
            }
            pos += uint64_t(total);
            if (sm) {
                const int hs = 31 - __clz(sm);
                run_start = c0 + uint32_t(hs);
                run_op = __shfl_sync(kFull, op, hs);
            }
            const int last_lane = int(min(31u, n - 1 - c0));
            carry_op = __shfl_sync(kFull, op, last_lane);
            if (mm) carry_v = __shfl_sync(kFull, v, 31 - __clz(mm));
        }
        // the open run, then the query positions after the last match
        const uint32_t last_len = n - run_start;
        const int tail = int(P.m) - 1 - carry_v;
        uint64_t end = pos + decimal_digits(last_len) + 1;
        if (tail > 0) end += decimal_digits(uint32_t(tail)) + 1;
        if (lane == 0) {
            if (write) {
                const int at = put_run(dst, int(pos), true, int(last_len), run_op ? 'D' : 'M');
                if (tail > 0) put_run(dst, at, true, tail, 'I');
            } else {
                lens[i] = end;
            }
        }
    }
}

__global__ void __launch_bounds__(256) exclusive_scan_kernel(const uint64_t* in, uint64_t* out, uint32_t n) {
    // single block of 256 threads (small enough to fit beside the serving
    // loop's resident consensus kernel); n up to a few million
    __shared__ uint64_t part[1024];
    const uint32_t tid = threadIdx.x;
    const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
    const uint32_t b = tid * per, e = min(n, b + per);
    uint64_t s = 0;
    for (uint32_t i = b; i < e; ++i) s += in[i];
    part[tid] = s;
    __syncthreads();
    if (tid == 0) {
        uint64_t acc = 0;
        for (uint32_t k = 0; k < blockDim.x; ++k) {
            const uint64_t v = part[k];
            part[k] = acc;
            acc += v;
        }
        out[n] = acc;
    }
    __syncthreads();
    uint64_t acc = part[tid];
    for (uint32_t i = b; i < e; ++i) {
        out[i] = acc;
        acc += in[i];
    }
}


// Breaking points walked from a SAM CIGAR, one thread per overlap, following
// src/overlap.cpp:226-292 step by step (window ends at every multiple of w
// inside (t_begin, t_end), plus t_end - 1).
struct CigarOvlDev {
    uint64_t cigar_off;
    uint64_t bp_off;
    uint32_t cigar_len, q_offset, t_begin, t_end;
};

__global__ void cigar_breakpoints_kernel(const char* cig, const CigarOvlDev* ov, uint32_t n,
                                         uint32_t w, uint32_t* bp, uint32_t* bp_count,
                                         unsigned int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const CigarOvlDev o = ov[i];
    const char* c = cig + o.cigar_off;
    uint32_t* out = bp + o.bp_off;
    uint32_t cnt = 0;
    // window ends in order: first multiple of w above t_begin, minus one ...
    const uint32_t first_mult = (o.t_begin / w + 1) * w;
    const uint32_t nmult = first_mult < o.t_end ? (o.t_end - 1 - first_mult) / w + 1 : 0;
    uint32_t wi = 0;
    auto window_end = [&](uint32_t k) -> int64_t {
        return k < nmult ? int64_t(first_mult) + int64_t(k) * w - 1 : int64_t(o.t_end) - 1;
    };
    const uint32_t nends = nmult + 1;
    bool found = false;
    uint32_t ft = 0, fq = 0, lt = 0, lq = 0;
    int64_t q_ptr = int64_t(o.q_offset) - 1;
    int64_t t_ptr = int64_t(o.t_begin) - 1;
    uint32_t num = 0;
    for (uint32_t k = 0; k < o.cigar_len; ++k) {
        const char ch = c[k];
        if (ch >= '0' && ch <= '9') {
            num = num * 10 + uint32_t(ch - '0');
            continue;
        }
        if (ch == 'M' || ch == '=' || ch == 'X') {
            for (uint32_t r = 0; r < num; ++r) {
                ++q_ptr;
                ++t_ptr;
                if (!found) {
                    found = true;
                    ft = uint32_t(t_ptr);
                    fq = uint32_t(q_ptr);
                }
                lt = uint32_t(t_ptr + 1);
                lq = uint32_t(q_ptr + 1);
                if (wi < nends && t_ptr == window_end(wi)) {
                    out[cnt++] = ft;
                    out[cnt++] = fq;
                    out[cnt++] = lt;
                    out[cnt++] = lq;
                    found = false;
                    ++wi;
                }
            }
        } else if (ch == 'I') {
            q_ptr += num;
        } else if (ch == 'D' || ch == 'N') {
            for (uint32_t r = 0; r < num; ++r) {
                ++t_ptr;
                if (wi < nends && t_ptr == window_end(wi)) {
                    if (found) {
                        out[cnt++] = ft;
                        out[cnt++] = fq;
                        out[cnt++] = lt;
                        out[cnt++] = lq;
                    }
                    found = false;
                    ++wi;
                }
            }
        }
        num = 0;  // S, H, P and the ops above all restart the number
        if (t_ptr >= int64_t(o.t_end)) {
            atomicCAS(status, 0u, 5u);
            break;
        }
    }
    bp_count[i] = cnt;
}


// ---------------------------------------------------------------------------
// Allocation-free edit distance (rb_nw_distance_noalloc). Same banded block
// sweep and k doubling as nw_distance_kernel, for one pair, with every byte of
// scratch (symbol-coded sequences, the two strip carry buffers) in one
// file-scope device array instead of cudaMalloc'd memory. Every call on a
// device uses the same array: it keeps the last call's contents, nothing in it
// has to start at zero (each call writes every byte it later reads), and two
// calls whose kernels overlap in time race on it.
constexpr uint32_t kNoAllocMaxLen = 1u << 17;  // per sequence
constexpr size_t kNoAllocCarry = size_t(kNoAllocMaxLen) + 64;
constexpr size_t kNoAllocScratchBytes =
    2 * size_t(kNoAllocMaxLen) + 2 * kNoAllocCarry + 2 * 4 * kNoAllocCarry + 4096;
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

__global__ void __launch_bounds__(32) nw_distance_noalloc_kernel(const char* q, uint32_t m, const char* t,
                                                                 uint32_t n, int32_t* out, uint8_t* scratch) {
    __shared__ u64 peq[kMaxSym * 32];
    __shared__ int present[256];
    const int lane = threadIdx.x;
    if (m == 0 || n == 0) {
        if (lane == 0) *out = int32_t(max(m, n));
        return;
    }
    uint8_t* qc = scratch;
    uint8_t* tc = scratch + kNoAllocMaxLen;
    WarpScratch ws;
    uint8_t* p = scratch + 2 * size_t(kNoAllocMaxLen);
    ws.carry_h[0] = reinterpret_cast<int8_t*>(p);
    ws.carry_h[1] = reinterpret_cast<int8_t*>(p + kNoAllocCarry);
    p += 2 * kNoAllocCarry;
    p = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 255) & ~uintptr_t(255));
    ws.carry_s[0] = reinterpret_cast<int32_t*>(p);
    ws.carry_s[1] = reinterpret_cast<int32_t*>(p + 4 * kNoAllocCarry);
    ws.capl_pv = ws.capl_mv = ws.capr_pv = ws.capr_mv = nullptr;
    ws.capl_sc = ws.capr_sc = nullptr;
    ws.leaf = nullptr;
    ws.block_peq = nullptr;  // strip sweeps only
    // symbols present, numbered by byte value (the distance does not depend
    // on the numbering); more than 32 distinct symbols is reported as -1
    for (int c = lane; c < 256; c += 32) present[c] = 0;
    __syncwarp();
    for (uint32_t i = lane; i < m; i += 32) present[uint8_t(q[i])] = 1;
    for (uint32_t i = lane; i < n; i += 32) present[uint8_t(t[i])] = 1;
    __syncwarp();
    int nsym = 0;
    for (int c = 0; c < 256; ++c) nsym += present[c];
    __syncwarp();
    if (nsym > kMaxSym) {
        if (lane == 0) *out = -1;
        return;
    }
    // present[c] := code of c (exclusive prefix over byte values)
    if (lane == 0) {
        int acc = 0;
        for (int c = 0; c < 256; ++c) {
            const int pr = present[c];
            present[c] = acc;
            acc += pr;
        }
    }
    __syncwarp();
    for (uint32_t i = lane; i < m; i += 32) qc[i] = uint8_t(present[uint8_t(q[i])]);
    for (uint32_t i = lane; i < n; i += 32) tc[i] = uint8_t(present[uint8_t(t[i])]);
    __syncwarp();
    SweepIO io;
    io.q = qc;
    io.t = tc;
    io.rev = false;
    io.ncols = int(n);
    io.nsym = max(nsym, 1);
    io.peq = peq;
    io.cap_pv = io.cap_mv = nullptr;
    io.cap_sc = nullptr;
    io.leaf = nullptr;
    io.bw = 0;
    int k = max(64, abs(int(m) - int(n)));
    int d;
    while (true) {
        const Band B = make_band(int(m), int(n), k);
        SweepFail f;
        d = warp_sweep<kDistance>(io, B, ws, lane, nullptr, &f);
        if (d <= k) break;
        k = next_k(k, f, int(m), int(n));
    }
    if (lane == 0) *out = d;
}

// Store offsets of one pair's query and target spans (rb_align_stage_overlaps).
struct NwStoreSrc {
    uint64_t q_src, t_src;
};

// Symbol codes of pairs cut from the staged sequence table: bytes are
// numbered by first appearance in the query, then the target (the numbering
// NwEngine::stage gives on the host), one warp per pair. First appearances
// come from one pass over 32-byte chunks in order: the lowest lane holding a
// byte value not seen before records its position. A pair with more than
// kMaxSymWide distinct bytes (impossible for bytes) sets status[0] = 1.
__global__ void __launch_bounds__(256) nw_encode_kernel(const uint8_t* store, const NwStoreSrc* src,
                                                        NwPairDev* pairs, uint8_t* codes, uint32_t n,
                                                        unsigned int* status) {
    __shared__ uint32_t first_pos[8][256];
    __shared__ uint8_t code[8][256];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    uint32_t* fp = first_pos[wib];
    uint8_t* cd = code[wib];
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
        const NwStoreSrc sp = src[i];
        const uint32_t m = pairs[i].m, nt = pairs[i].n;
        const uint64_t q_off = pairs[i].q_off, t_off = pairs[i].t_off;
        for (int v = lane; v < 256; v += 32) fp[v] = 0xFFFFFFFFu;
        __syncwarp();
        const uint32_t total = m + nt;
        for (uint32_t k0 = 0; k0 < total; k0 += 32) {
            const uint32_t k = k0 + lane;
            uint32_t c = 0x100u + uint32_t(lane);  // matches no byte value
            if (k < total) c = k < m ? store[sp.q_src + k] : store[sp.t_src + (k - m)];
            const unsigned same = __match_any_sync(0xffffffffu, c);
            if (c < 0x100u && __ffs(same) - 1 == lane && fp[c] == 0xFFFFFFFFu) fp[c] = k;
            __syncwarp();
        }
        int present = 0;
        for (int v = lane; v < 256; v += 32) {
            const uint32_t p = fp[v];
            if (p == 0xFFFFFFFFu) continue;
            int r = 0;
            for (int u = 0; u < 256; ++u) r += fp[u] < p ? 1 : 0;
            cd[v] = uint8_t(r);
            ++present;
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) present += __shfl_xor_sync(0xffffffffu, present, d);
        __syncwarp();
        if (present > kMaxSymWide) {  // cannot happen for byte symbols; kept as a guard
            if (lane == 0) status[0] = 1u;
            continue;
        }
        for (uint32_t k = lane; k < m; k += 32) codes[q_off + k] = cd[store[sp.q_src + k]];
        for (uint32_t k = lane; k < nt; k += 32) codes[t_off + k] = cd[store[sp.t_src + k]];
        if (lane == 0) pairs[i].nsym = uint32_t(max(present, 1));
        __syncwarp();
    }
}

}  // namespace

NwEngine::NwEngine(const DeviceInfo& dev, cudaStream_t stream) : dev_(dev), stream_(stream) {
    check_cuda(cudaEventCreate(&ev0_), "cudaEventCreate");
    check_cuda(cudaEventCreate(&ev1_), "cudaEventCreate");
    check_cuda(cudaEventCreate(&ev2_), "cudaEventCreate");
    check_cuda(cudaEventCreate(&ev3_), "cudaEventCreate");
    check_cuda(cudaFuncSetAttribute(nw_distance_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    kWarpsPerBlock * kMaxSym * 32 * 8),
               "cudaFuncSetAttribute");
    check_cuda(cudaFuncSetAttribute(nw_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    kWarpsPerBlock * kMaxSym * 32 * 8),
               "cudaFuncSetAttribute");
    const void* kernels[] = {reinterpret_cast<const void*>(nw_distance_kernel),
                             reinterpret_cast<const void*>(nw_level_kernel),
                             reinterpret_cast<const void*>(nw_breakpoints_kernel),
                             reinterpret_cast<const void*>(nw_cigar_kernel),
                             reinterpret_cast<const void*>(exclusive_scan_kernel),
                             reinterpret_cast<const void*>(cigar_breakpoints_kernel),
                             reinterpret_cast<const void*>(nw_encode_kernel)};
    for (const void* k : kernels) prefer_max_shared(k);
}

NwEngine::~NwEngine() {
    cudaEventDestroy(ev0_);
    cudaEventDestroy(ev1_);
    cudaEventDestroy(ev2_);
    cudaEventDestroy(ev3_);
}

void NwEngine::stage(const rb_pair* pairs, size_t n, int want_cigar, uint32_t window_length) {
    if (n > 0 && !pairs) throw Error{RB_ERR_ARG, "rb_align: pairs is NULL"};
    if (window_length == 0) throw Error{RB_ERR_ARG, "rb_align: window length is 0"};
    npairs_ = 0;
    want_cigar_ = want_cigar;
    window_length_ = window_length;
    // sizes and offsets (16-byte aligned per sequence)
    uint64_t bytes = 0, mq_len = 0, bp_slots = 0;
    max_m_ = max_n_ = 0;
    for (size_t i = 0; i < n; ++i) {
        const rb_pair& p = pairs[i];
        if (p.query_length > (1u << 24) || p.target_length > (1u << 24))
            throw Error{RB_ERR_ARG, "rb_align: span longer than 2^24 bases"};
        if ((p.query_length && !p.query) || (p.target_length && !p.target))
            throw Error{RB_ERR_ARG, "rb_align: NULL sequence with nonzero length"};
        bytes += ((p.query_length + 15) & ~15u) + ((p.target_length + 15) & ~15u);
        mq_len += p.target_length;
        if (p.target_length > 0) {
            const uint64_t segs = (uint64_t(p.t_begin) + p.target_length - 1) / window_length -
                                  p.t_begin / window_length + 1;
            bp_slots += 4 * segs;
        }
        max_m_ = std::max(max_m_, p.query_length);
        max_n_ = std::max(max_n_, p.target_length);
    }
    code_bytes_ = bytes;
    mq_len_ = mq_len;
    bp_slots_ = bp_slots;
    h_codes_.reserve(std::max<uint64_t>(bytes, 16));
    h_pairs_.reserve(std::max<size_t>(n, 1) * sizeof(NwPairDev));
    h_order_.reserve(std::max<size_t>(n, 1) * sizeof(uint32_t));
    h_src_.reserve(std::max<size_t>(n, 1) * sizeof(NwStoreSrc));
    uint8_t* codes = h_codes_.as<uint8_t>();
    NwPairDev* pd = h_pairs_.as<NwPairDev>();
    NwStoreSrc* src = h_src_.as<NwStoreSrc>();
    // raw bytes go to the device as they are; nw_encode_kernel numbers each
    // pair's symbols there, in place
    uint64_t off = 0, mqo = 0, bpo = 0;
    for (size_t i = 0; i < n; ++i) {
        const rb_pair& p = pairs[i];
        NwPairDev& d = pd[i];
        d.q_off = off;
        off += (p.query_length + 15) & ~15u;
        d.t_off = off;
        off += (p.target_length + 15) & ~15u;
        src[i].q_src = d.q_off;
        src[i].t_src = d.t_off;
        d.nsym = 1;
        d.m = p.query_length;
        d.n = p.target_length;
        d.mq_off = mqo;
        mqo += p.target_length;
        d.bp_off = bpo;
        if (p.target_length > 0) {
            const uint64_t segs = (uint64_t(p.t_begin) + p.target_length - 1) / window_length -
                                  p.t_begin / window_length + 1;
            bpo += 4 * segs;
        }
        d.q_offset = p.q_offset;
        d.t_begin = p.t_begin;
    }
    auto copy_range = [&](size_t b, size_t e) {
        for (size_t i = b; i < e; ++i) {
            if (pairs[i].query_length) memcpy(codes + pd[i].q_off, pairs[i].query, pairs[i].query_length);
            if (pairs[i].target_length) memcpy(codes + pd[i].t_off, pairs[i].target, pairs[i].target_length);
        }
    };
    const unsigned nth = bytes > (uint64_t(64) << 20) ? std::max(1u, std::min(8u, std::thread::hardware_concurrency())) : 1u;
    if (nth == 1) {
        copy_range(0, n);
    } else {
        std::vector<std::thread> pool;
        for (unsigned k = 0; k < nth; ++k) pool.emplace_back(copy_range, n * k / nth, n * (k + 1) / nth);
        for (auto& th : pool) th.join();
    }
    // size-sorted work order: largest banded work first
    uint32_t* order = h_order_.as<uint32_t>();
    std::iota(order, order + n, 0u);
    std::sort(order, order + n, [&](uint32_t x, uint32_t y) {
        const uint64_t wx = uint64_t(pd[x].m + 64) * pd[x].n, wy = uint64_t(pd[y].m + 64) * pd[y].n;
        return wx != wy ? wx > wy : x < y;
    });
    d_codes_.reserve(std::max<uint64_t>(bytes, 16));
    d_pairs_.reserve(std::max<size_t>(n, 1) * sizeof(NwPairDev));
    d_order_.reserve(std::max<size_t>(n, 1) * sizeof(uint32_t));
    d_dist_.reserve(std::max<size_t>(n, 1) * sizeof(int32_t));
    d_mq_.reserve(std::max<uint64_t>(mq_len, 1) * sizeof(int32_t));
    d_bp_.reserve(std::max<uint64_t>(bp_slots, 1) * sizeof(uint32_t));
    d_bpcnt_.reserve(std::max<size_t>(n, 1) * sizeof(uint32_t));
    d_misc_.reserve(64);
    d_src_.reserve(std::max<size_t>(n, 1) * sizeof(NwStoreSrc));
    check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    check_cuda(cudaMemcpyAsync(d_codes_.ptr, codes, bytes, cudaMemcpyHostToDevice, stream_), "H2D sequences");
    check_cuda(cudaMemcpyAsync(d_pairs_.ptr, pd, n * sizeof(NwPairDev), cudaMemcpyHostToDevice, stream_),
               "H2D pairs");
    check_cuda(cudaMemcpyAsync(d_order_.ptr, order, n * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_),
               "H2D order");
    unsigned int status = 0;
    if (n) {
        check_cuda(cudaMemcpyAsync(d_src_.ptr, src, n * sizeof(NwStoreSrc), cudaMemcpyHostToDevice, stream_),
                   "H2D pair sources");
        check_cuda(cudaMemsetAsync(d_misc_.ptr, 0, 64, stream_), "memset status");
        const int grid = int(std::max<size_t>(1, std::min<size_t>((n + 7) / 8, size_t(dev_.sm_count) * 8)));
        nw_encode_kernel<<<grid, 256, 0, stream_>>>(d_codes_.as<uint8_t>(), d_src_.as<NwStoreSrc>(),
                                                    d_pairs_.as<NwPairDev>(), d_codes_.as<uint8_t>(), uint32_t(n),
                                                    d_misc_.as<unsigned int>());
        check_cuda(cudaGetLastError(), "nw_encode_kernel");
        check_cuda(cudaMemcpyAsync(&status, d_misc_.ptr, 4, cudaMemcpyDeviceToHost, stream_), "D2H status");
    }
    check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    check_cuda(cudaStreamSynchronize(stream_), "stage sync");
    if (status) throw Error{RB_ERR_ARG, "rb_align: symbol coding failed"};
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    stats_.h2d_ms = ms;
    stats_.h2d_bytes = bytes + n * (sizeof(NwPairDev) + sizeof(NwStoreSrc) + sizeof(uint32_t));
    npairs_ = n;
}

void NwEngine::stage_store(const rb_store_pair* pairs, size_t n, int want_cigar, uint32_t window_length,
                           const SeqStore& st) {
    if (n > 0 && !pairs) throw Error{RB_ERR_ARG, "rb_align: pairs is NULL"};
    if (window_length == 0) throw Error{RB_ERR_ARG, "rb_align: window length is 0"};
    npairs_ = 0;
    want_cigar_ = want_cigar;
    window_length_ = window_length;
    uint64_t bytes = 0, mq_len = 0, bp_slots = 0;
    max_m_ = max_n_ = 0;
    h_pairs_.reserve(std::max<size_t>(n, 1) * sizeof(NwPairDev));
    h_order_.reserve(std::max<size_t>(n, 1) * sizeof(uint32_t));
    h_src_.reserve(std::max<size_t>(n, 1) * sizeof(NwStoreSrc));
    NwPairDev* pd = h_pairs_.as<NwPairDev>();
    NwStoreSrc* src = h_src_.as<NwStoreSrc>();
    for (size_t i = 0; i < n; ++i) {
        const rb_store_pair& p = pairs[i];
        if (p.q_id >= st.n || p.t_id >= st.n) throw Error{RB_ERR_ARG, "rb_align: sequence id out of range"};
        const SeqDev& q = st.host[p.q_id];
        const SeqDev& t = st.host[p.t_id];
        if (p.q_begin > p.q_end || p.q_end > q.len || p.t_begin > p.t_end || p.t_end > t.len)
            throw Error{RB_ERR_ARG, "rb_align: span outside its sequence"};
        const uint64_t qbase = p.strand ? q.rev : q.fwd;
        if (qbase == kNotStaged || t.fwd == kNotStaged)
            throw Error{RB_ERR_ARG, "rb_align: sequence strand not staged"};
        const uint32_t m = p.q_end - p.q_begin, tn = p.t_end - p.t_begin;
        if (m > (1u << 24) || tn > (1u << 24)) throw Error{RB_ERR_ARG, "rb_align: span longer than 2^24 bases"};
        // query = read span, reverse-complemented for '-' (src/overlap.cpp:193-197)
        const uint32_t q_offset = p.strand ? q.len - p.q_end : p.q_begin;
        src[i].q_src = qbase + q_offset;
        src[i].t_src = t.fwd + p.t_begin;
        NwPairDev& d = pd[i];
        d.q_off = bytes;
        bytes += (m + 15) & ~15u;
        d.t_off = bytes;
        bytes += (tn + 15) & ~15u;
        d.nsym = 1;
        d.m = m;
        d.n = tn;
        d.mq_off = mq_len;
        mq_len += tn;
        d.bp_off = bp_slots;
        if (tn > 0) bp_slots += 4 * ((uint64_t(p.t_begin) + tn - 1) / window_length - p.t_begin / window_length + 1);
        d.q_offset = q_offset;
        d.t_begin = p.t_begin;
        max_m_ = std::max(max_m_, m);
        max_n_ = std::max(max_n_, tn);
    }
    code_bytes_ = bytes;
    mq_len_ = mq_len;
    bp_slots_ = bp_slots;
    uint32_t* order = h_order_.as<uint32_t>();
    std::iota(order, order + n, 0u);
    std::sort(order, order + n, [&](uint32_t x, uint32_t y) {
        const uint64_t wx = uint64_t(pd[x].m + 64) * pd[x].n, wy = uint64_t(pd[y].m + 64) * pd[y].n;
        return wx != wy ? wx > wy : x < y;
    });
    d_codes_.reserve(std::max<uint64_t>(bytes, 16));
    d_pairs_.reserve(std::max<size_t>(n, 1) * sizeof(NwPairDev));
    d_src_.reserve(std::max<size_t>(n, 1) * sizeof(NwStoreSrc));
    d_order_.reserve(std::max<size_t>(n, 1) * sizeof(uint32_t));
    d_dist_.reserve(std::max<size_t>(n, 1) * sizeof(int32_t));
    d_mq_.reserve(std::max<uint64_t>(mq_len, 1) * sizeof(int32_t));
    d_bp_.reserve(std::max<uint64_t>(bp_slots, 1) * sizeof(uint32_t));
    d_bpcnt_.reserve(std::max<size_t>(n, 1) * sizeof(uint32_t));
    d_misc_.reserve(64);
    check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    if (n) {
        check_cuda(cudaMemcpyAsync(d_pairs_.ptr, pd, n * sizeof(NwPairDev), cudaMemcpyHostToDevice, stream_),
                   "H2D pairs");
        check_cuda(cudaMemcpyAsync(d_src_.ptr, src, n * sizeof(NwStoreSrc), cudaMemcpyHostToDevice, stream_),
                   "H2D pair sources");
        check_cuda(cudaMemcpyAsync(d_order_.ptr, order, n * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_),
                   "H2D order");
        check_cuda(cudaMemsetAsync(d_misc_.ptr, 0, 64, stream_), "memset status");
        const int grid = int(std::max<size_t>(1, std::min<size_t>((n + 7) / 8, size_t(dev_.sm_count) * 8)));
        nw_encode_kernel<<<grid, 256, 0, stream_>>>(st.bytes, d_src_.as<NwStoreSrc>(), d_pairs_.as<NwPairDev>(),
                                                    d_codes_.as<uint8_t>(), uint32_t(n), d_misc_.as<unsigned int>());
        check_cuda(cudaGetLastError(), "nw_encode_kernel");
    }
    check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    unsigned int status = 0;
    if (n) check_cuda(cudaMemcpyAsync(&status, d_misc_.ptr, 4, cudaMemcpyDeviceToHost, stream_), "D2H status");
    check_cuda(cudaStreamSynchronize(stream_), "stage sync");
    if (status) throw Error{RB_ERR_ARG, "rb_align: symbol coding failed"};
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    stats_.h2d_ms = ms;
    stats_.h2d_bytes = n * (sizeof(NwPairDev) + sizeof(NwStoreSrc) + sizeof(uint32_t));
    npairs_ = n;
}

void NwEngine::reserve_scratch(uint32_t max_m, uint32_t max_n) {
    const size_t nb = (size_t(max_m) + 63) / 64 + 1;
    const size_t ncols = size_t(max_n) + 64;
    scratch_stride_ = warp_scratch_bytes(ncols, nb);
    // warps: the device's tuned warps per SM on the context's share of the
    // SMs (all by default), bounded by a scratch budget of 4 GiB
    const size_t per_sm = tuning_get(dev_.device).alignment_warps_per_sm;
    size_t warps = std::max<size_t>(kWarpsPerBlock, size_t(dev_.sm_count) * per_sm * sm_share_pct_ / 100);
    const size_t budget = size_t(4) << 30;
    while (warps > size_t(kWarpsPerBlock) && warps * scratch_stride_ > budget) warps /= 2;
    warps = (warps / kWarpsPerBlock) * kWarpsPerBlock;
    if (warps == 0) warps = kWarpsPerBlock;
    scratch_warps_ = warps;
    d_scratch_.reserve(warps * scratch_stride_);
}

void NwEngine::run() {
    if (svc_ && npairs_ > 0 && svc_->fits(max_m_, max_n_)) {
        run_shared();
    } else {
        run_own();
    }
}

namespace {
// Arguments of the staged batch common to the engine's own kernels and the
// shared service (scratch and queue fields are set by the caller).
NwDevArgs batch_args(const DevBuf& codes, const DevBuf& pairs, const DevBuf& order, size_t n, const DevBuf& dist,
                     const DevBuf& mq, const DevBuf& bp, const DevBuf& bpcnt, uint32_t window_length,
                     const DevBuf& misc) {
    NwDevArgs a;
    memset(&a, 0, sizeof(a));
    a.codes = codes.as<uint8_t>();
    a.pairs = pairs.as<NwPairDev>();
    a.order = order.as<uint32_t>();
    a.npairs = uint32_t(n);
    a.dist = dist.as<int32_t>();
    a.mq = mq.as<int32_t>();
    a.bp = bp.as<uint32_t>();
    a.bp_count = bpcnt.as<uint32_t>();
    a.window_length = window_length;
    a.counters = misc.as<unsigned int>();
    return a;
}
}  // namespace

void NwEngine::run_own() {
    const size_t n = npairs_;
    stats_.launches = 0;
    stats_.items = n;
    stats_.cells = 0;
    if (n == 0) {
        stats_.kernel_ms = 0;
        return;
    }
    reserve_scratch(max_m_, max_n_);
    size_t task_cap = std::max<size_t>(n, 1) * 2 + 64;
    d_tasks_[0].reserve(task_cap * sizeof(NwTask));
    d_tasks_[1].reserve(task_cap * sizeof(NwTask));
    NwDevArgs a = batch_args(d_codes_, d_pairs_, d_order_, n, d_dist_, d_mq_, d_bp_, d_bpcnt_, window_length_,
                             d_misc_);
    a.scratch = d_scratch_.as<uint8_t>();
    a.scratch_stride = scratch_stride_;
    a.scratch_warps = uint32_t(scratch_warps_);
    a.max_n = max_n_ + 64;
    a.max_nb = (max_m_ + 63) / 64 + 1;
    // the distance pass appends each pair's root task (level 0)
    a.tasks_out = d_tasks_[0].as<NwTask>();
    a.tasks_out_cap = uint32_t(task_cap);
    const int grid = int(scratch_warps_ / kWarpsPerBlock);
    const size_t smem = kWarpsPerBlock * kMaxSym * 32 * 8;
    check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    check_cuda(cudaMemsetAsync(a.counters, 0, 64, stream_), "memset counters");
    // persistent by default; with a per-warp cap, enough launches back to
    // back that every pair (task) is taken
    a.per_warp_cap = yield_items_;
    auto launches_for = [&](size_t items) {
        return yield_items_ ? (items + scratch_warps_ * yield_items_ - 1) / (scratch_warps_ * yield_items_)
                            : size_t(1);
    };
    for (size_t l = launches_for(n); l > 0; --l) {
        nw_distance_kernel<<<grid, 32 * kWarpsPerBlock, smem, stream_>>>(a);
        ++stats_.launches;
    }
    unsigned int h_cnt[4];
    check_cuda(cudaMemcpyAsync(h_cnt, a.counters, 16, cudaMemcpyDeviceToHost, stream_), "D2H count");
    check_cuda(cudaStreamSynchronize(stream_), "sync level");
    if (h_cnt[2] != 0) throw Error{RB_ERR_DEVICE, "nw: distance kernel status " + std::to_string(h_cnt[2])};
    uint32_t ntasks = h_cnt[1];
    int cur = 0;
    while (ntasks > 0) {
        const size_t need = size_t(ntasks) * 2 + 64;
        d_tasks_[cur ^ 1].reserve(need * sizeof(NwTask));
        task_cap = d_tasks_[cur ^ 1].bytes / sizeof(NwTask);
        a.tasks_in = d_tasks_[cur].as<NwTask>();
        a.ntasks_in = ntasks;
        a.tasks_out = d_tasks_[cur ^ 1].as<NwTask>();
        a.tasks_out_cap = uint32_t(task_cap);
        check_cuda(cudaMemsetAsync(a.counters, 0, 8, stream_), "memset counters");
        for (size_t l = launches_for(ntasks); l > 0; --l) {
            nw_level_kernel<<<grid, 32 * kWarpsPerBlock, smem, stream_>>>(a);
            ++stats_.launches;
        }
        check_cuda(cudaMemcpyAsync(h_cnt, a.counters, 16, cudaMemcpyDeviceToHost, stream_), "D2H count");
        check_cuda(cudaStreamSynchronize(stream_), "sync level");
        if (h_cnt[2] != 0) throw Error{RB_ERR_DEVICE, "nw: level kernel status " + std::to_string(h_cnt[2])};
        ntasks = h_cnt[1];
        cur ^= 1;
    }
    finish_outputs(&a);
    check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    check_cuda(cudaStreamSynchronize(stream_), "sync run");
    check_cuda(cudaGetLastError(), "nw kernels");
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    stats_.kernel_ms = ms;
}

// The distance pass and every recursion level as batches of the shared
// service (each waits for the previous one: a level's tasks come from the
// one before), then the breaking points (and CIGARs) on this engine's stream.
void NwEngine::run_shared() {
    const size_t n = npairs_;
    stats_.launches = 0;
    stats_.items = n;
    stats_.cells = 0;
    const auto t0 = std::chrono::steady_clock::now();
    size_t task_cap = std::max<size_t>(n, 1) * 2 + 64;
    d_tasks_[0].reserve(task_cap * sizeof(NwTask));
    d_tasks_[1].reserve(task_cap * sizeof(NwTask));
    NwDevArgs a = batch_args(d_codes_, d_pairs_, d_order_, n, d_dist_, d_mq_, d_bp_, d_bpcnt_, window_length_,
                             d_misc_);
    check_cuda(cudaMemsetAsync(a.counters, 0, 64, stream_), "memset counters");
    // the staged pairs and the counters are in place before any item is published
    check_cuda(cudaStreamSynchronize(stream_), "nw stage sync");
    NwJobDev job;
    memset(&job, 0, sizeof(job));
    job.mode = kJobDistance;
    job.codes = a.codes;
    job.pairs = a.pairs;
    job.dist = a.dist;
    job.mq = a.mq;
    job.counters = a.counters;
    job.tasks_out = d_tasks_[0].ptr;
    job.tasks_out_cap = uint32_t(task_cap);
    // size class: ring 0 up to svc_priority_ pairs, then x4 per ring
    const uint64_t p = std::max<uint32_t>(1, svc_priority_);
    const int queue = n <= p ? 0 : n <= 4 * p ? 1 : n <= 16 * p ? 2 : 3;
    svc_->run_batch(job, h_order_.as<uint32_t>(), n, queue);
    ++stats_.launches;
    unsigned int h_cnt[4];
    check_cuda(cudaMemcpyAsync(h_cnt, a.counters, 16, cudaMemcpyDeviceToHost, stream_), "D2H count");
    check_cuda(cudaStreamSynchronize(stream_), "sync level");
    if (h_cnt[2] != 0) throw Error{RB_ERR_DEVICE, "nw: distance pass status " + std::to_string(h_cnt[2])};
    uint32_t ntasks = h_cnt[1];
    std::vector<uint32_t> idx;
    int cur = 0;
    while (ntasks > 0) {
        const size_t need = size_t(ntasks) * 2 + 64;
        d_tasks_[cur ^ 1].reserve(need * sizeof(NwTask));
        task_cap = d_tasks_[cur ^ 1].bytes / sizeof(NwTask);
        check_cuda(cudaMemsetAsync(a.counters, 0, 8, stream_), "memset counters");
        check_cuda(cudaStreamSynchronize(stream_), "nw level sync");
        job.mode = kJobLevel;
        job.tasks_in = d_tasks_[cur].ptr;
        job.ntasks_in = ntasks;
        job.tasks_out = d_tasks_[cur ^ 1].ptr;
        job.tasks_out_cap = uint32_t(task_cap);
        idx.resize(ntasks);
        std::iota(idx.begin(), idx.end(), 0u);
        svc_->run_batch(job, idx.data(), ntasks, queue);
        ++stats_.launches;
        check_cuda(cudaMemcpyAsync(h_cnt, a.counters, 16, cudaMemcpyDeviceToHost, stream_), "D2H count");
        check_cuda(cudaStreamSynchronize(stream_), "sync level");
        if (h_cnt[2] != 0) throw Error{RB_ERR_DEVICE, "nw: level pass status " + std::to_string(h_cnt[2])};
        ntasks = h_cnt[1];
        cur ^= 1;
    }
    finish_outputs(&a);
    check_cuda(cudaStreamSynchronize(stream_), "sync run");
    check_cuda(cudaGetLastError(), "nw kernels");
    stats_.kernel_ms = float(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
}

// Breaking points, and with want_cigar the CIGAR strings, of the aligned
// pairs: warp-per-pair kernels on this engine's stream.
void NwEngine::finish_outputs(const void* args) {
    const NwDevArgs& a = *static_cast<const NwDevArgs*>(args);
    const size_t n = npairs_;
    const int warp_grid = int(std::max<size_t>(1, std::min<size_t>((n + 7) / 8, size_t(dev_.sm_count) * 16)));
    nw_breakpoints_kernel<<<warp_grid, 256, 0, stream_>>>(a);
    ++stats_.launches;
    if (want_cigar_) {
        d_ciglen_.reserve((n + 1) * sizeof(uint64_t));
        d_cigoff_.reserve((n + 1) * sizeof(uint64_t));
        nw_cigar_kernel<<<warp_grid, 256, 0, stream_>>>(a, d_ciglen_.as<uint64_t>(), nullptr,
                                                                   nullptr, 0);
        exclusive_scan_kernel<<<1, 256, 0, stream_>>>(d_ciglen_.as<uint64_t>(), d_cigoff_.as<uint64_t>(),
                                                       uint32_t(n));
        uint64_t total = 0;
        check_cuda(cudaMemcpyAsync(&total, d_cigoff_.as<uint64_t>() + n, 8, cudaMemcpyDeviceToHost, stream_),
                   "D2H cigar total");
        check_cuda(cudaStreamSynchronize(stream_), "sync cigar");
        d_cig_.reserve(std::max<uint64_t>(total, 1));
        nw_cigar_kernel<<<warp_grid, 256, 0, stream_>>>(a, d_ciglen_.as<uint64_t>(),
                                                                   d_cigoff_.as<uint64_t>(), d_cig_.as<char>(), 1);
        stats_.launches += 3;
    }
}

void NwEngine::cigar_breakpoints(const rb_cigar_overlap* ovl, size_t n, uint32_t w, rb_aln_result* out) {
    if (n > 0 && !ovl) throw Error{RB_ERR_ARG, "rb_cigar_breakpoints: overlaps is NULL"};
    if (w == 0) throw Error{RB_ERR_ARG, "rb_cigar_breakpoints: window length is 0"};
    uint64_t cbytes = 0, slots = 0;
    for (size_t i = 0; i < n; ++i) {
        if (ovl[i].t_end < ovl[i].t_begin || (ovl[i].cigar_length && !ovl[i].cigar))
            throw Error{RB_ERR_ARG, "rb_cigar_breakpoints: invalid overlap"};
        cbytes += ovl[i].cigar_length + 1;
        const uint64_t segs = ovl[i].t_end > ovl[i].t_begin
                                  ? (uint64_t(ovl[i].t_end) - 1) / w - ovl[i].t_begin / w + 1
                                  : 1;
        slots += 4 * segs;
    }
    h_codes_.reserve(std::max<uint64_t>(cbytes, 16));
    h_pairs_.reserve(std::max<size_t>(n, 1) * sizeof(CigarOvlDev));
    char* cb = h_codes_.as<char>();
    CigarOvlDev* od = h_pairs_.as<CigarOvlDev>();
    uint64_t off = 0, bo = 0;
    for (size_t i = 0; i < n; ++i) {
        od[i].cigar_off = off;
        od[i].cigar_len = ovl[i].cigar_length;
        od[i].q_offset = ovl[i].q_offset;
        od[i].t_begin = ovl[i].t_begin;
        od[i].t_end = ovl[i].t_end;
        od[i].bp_off = bo;
        if (ovl[i].cigar_length) memcpy(cb + off, ovl[i].cigar, ovl[i].cigar_length);
        cb[off + ovl[i].cigar_length] = 0;
        off += ovl[i].cigar_length + 1;
        const uint64_t segs = ovl[i].t_end > ovl[i].t_begin
                                  ? (uint64_t(ovl[i].t_end) - 1) / w - ovl[i].t_begin / w + 1
                                  : 1;
        bo += 4 * segs;
    }
    d_codes_.reserve(std::max<uint64_t>(off, 16));
    d_pairs_.reserve(std::max<size_t>(n, 1) * sizeof(CigarOvlDev));
    d_bp_.reserve(std::max<uint64_t>(slots, 1) * 4);
    d_bpcnt_.reserve(std::max<size_t>(n, 1) * 4);
    d_misc_.reserve(64);
    check_cuda(cudaMemsetAsync(d_misc_.ptr, 0, 64, stream_), "memset status");
    check_cuda(cudaMemcpyAsync(d_codes_.ptr, cb, off, cudaMemcpyHostToDevice, stream_), "H2D cigars");
    check_cuda(cudaMemcpyAsync(d_pairs_.ptr, od, n * sizeof(CigarOvlDev), cudaMemcpyHostToDevice, stream_),
               "H2D overlaps");
    check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    if (n)
        cigar_breakpoints_kernel<<<int((n + 127) / 128), 128, 0, stream_>>>(
            d_codes_.as<char>(), d_pairs_.as<CigarOvlDev>(), uint32_t(n), w, d_bp_.as<uint32_t>(),
            d_bpcnt_.as<uint32_t>(), d_misc_.as<unsigned int>());
    check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    std::vector<uint32_t> cnt(n), raw(slots);
    unsigned int status = 0;
    if (n) {
        check_cuda(cudaMemcpyAsync(cnt.data(), d_bpcnt_.ptr, n * 4, cudaMemcpyDeviceToHost, stream_), "D2H");
        check_cuda(cudaMemcpyAsync(raw.data(), d_bp_.ptr, slots * 4, cudaMemcpyDeviceToHost, stream_), "D2H");
    }
    check_cuda(cudaMemcpyAsync(&status, d_misc_.ptr, 4, cudaMemcpyDeviceToHost, stream_), "D2H");
    check_cuda(cudaStreamSynchronize(stream_), "sync cigar breakpoints");
    check_cuda(cudaGetLastError(), "cigar breakpoints kernel");
    if (status) throw Error{RB_ERR_ARG, "rb_cigar_breakpoints: CIGAR runs past the target span"};
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    stats_.kernel_ms = ms;
    stats_.launches = n ? 1 : 0;
    stats_.items = n;
    npairs_ = 0;
    dist_.assign(n, -1);
    bp_offsets_.assign(n + 1, 0);
    bp_.clear();
    for (size_t i = 0; i < n; ++i) {
        bp_offsets_[i] = bp_.size();
        bp_.insert(bp_.end(), raw.begin() + od[i].bp_off, raw.begin() + od[i].bp_off + cnt[i]);
    }
    bp_offsets_[n] = bp_.size();
    out->edit_distance = dist_.data();
    out->breakpoints = bp_.data();
    out->bp_offsets = bp_offsets_.data();
    out->cigars = nullptr;
    out->cigar_offsets = nullptr;
}

void NwEngine::fetch(rb_aln_result* out) {
    const size_t n = npairs_;
    check_cuda(cudaEventRecord(ev2_, stream_), "cudaEventRecord");
    dist_.resize(n);
    // pinned staging: the breakpoint slots and counts, and the CIGAR text,
    // which the result points into directly
    h_bpcnt_.reserve(std::max<size_t>(n, 1) * 4);
    h_bp_.reserve(std::max<uint64_t>(bp_slots_, 1) * 4);
    const uint32_t* cnt = h_bpcnt_.as<uint32_t>();
    const uint32_t* raw = h_bp_.as<uint32_t>();
    if (n) {
        check_cuda(cudaMemcpyAsync(dist_.data(), d_dist_.ptr, n * 4, cudaMemcpyDeviceToHost, stream_), "D2H dist");
        check_cuda(cudaMemcpyAsync(h_bpcnt_.ptr, d_bpcnt_.ptr, n * 4, cudaMemcpyDeviceToHost, stream_), "D2H bpcnt");
        if (bp_slots_)
            check_cuda(cudaMemcpyAsync(h_bp_.ptr, d_bp_.ptr, bp_slots_ * 4, cudaMemcpyDeviceToHost, stream_),
                       "D2H bp");
    }
    uint64_t d2h = n * 8 + bp_slots_ * 4;
    std::vector<uint64_t> cigoff;
    if (want_cigar_ && n) {
        cigoff.resize(n + 1);
        check_cuda(cudaMemcpyAsync(cigoff.data(), d_cigoff_.ptr, (n + 1) * 8, cudaMemcpyDeviceToHost, stream_),
                   "D2H cigoff");
        check_cuda(cudaStreamSynchronize(stream_), "sync fetch");
        h_cig_.reserve(std::max<uint64_t>(cigoff[n], 1));
        if (cigoff[n])
            check_cuda(cudaMemcpyAsync(h_cig_.ptr, d_cig_.ptr, cigoff[n], cudaMemcpyDeviceToHost, stream_),
                       "D2H cigars");
        d2h += (n + 1) * 8 + cigoff[n];
    }
    check_cuda(cudaEventRecord(ev3_, stream_), "cudaEventRecord");
    check_cuda(cudaStreamSynchronize(stream_), "sync fetch");
    float ms = 0;
    cudaEventElapsedTime(&ms, ev2_, ev3_);
    stats_.d2h_ms = ms;
    stats_.d2h_bytes = d2h;
    // compact breakpoints
    const NwPairDev* pd = h_pairs_.as<NwPairDev>();
    bp_offsets_.assign(n + 1, 0);
    bp_.clear();
    for (size_t i = 0; i < n; ++i) {
        bp_offsets_[i] = bp_.size();
        bp_.insert(bp_.end(), raw + pd[i].bp_off, raw + pd[i].bp_off + cnt[i]);
    }
    bp_offsets_[n] = bp_.size();
    out->edit_distance = dist_.data();
    out->breakpoints = bp_.data();
    out->bp_offsets = bp_offsets_.data();
    if (want_cigar_) {
        cig_offsets_ = cigoff.empty() ? std::vector<uint64_t>(n + 1, 0) : cigoff;
        if (cigoff.empty()) h_cig_.reserve(1);
        out->cigars = h_cig_.as<char>();
        out->cigar_offsets = cig_offsets_.data();
    } else {
        out->cigars = nullptr;
        out->cigar_offsets = nullptr;
    }
}

// ---------------------------------------------------------------------------
// Shared overlap-alignment service (continuous batching for the serving loop)

struct NwSvcState {
    explicit NwSvcState(int device) : ring(device, sizeof(NwJobDev), "rb_align service") {}
    RingService ring;
    void* d_scratch = nullptr;  // one scratch slot per resident warp
    NwSvcArgs args{};
    uint32_t slots = 0, grid = 0, max_span = 0;
};

namespace {
cudaError_t launch_nw_service(cudaStream_t stream, void* user) {
    const NwSvcState* S = static_cast<const NwSvcState*>(user);
    nw_service_kernel<<<S->grid, 32 * kWarpsPerBlock, kWarpsPerBlock * kMaxSym * 32 * 8, stream>>>(S->args);
    return cudaGetLastError();
}
}  // namespace

NwService::NwService(int device, uint32_t max_span, size_t scratch_budget, uint32_t ctas_per_sm,
                     uint32_t large_first_every)
    : st_(nullptr) {
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    int sm_count = 148;
    check_cuda(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device), "sm count");
    std::unique_ptr<NwSvcState> S(new NwSvcState(device));
    max_span = std::max<uint32_t>(max_span, 64);
    // the same layout the engine's own kernels use for spans up to max_span
    const size_t nb = (size_t(max_span) + 63) / 64 + 1, ncols = size_t(max_span) + 64;
    const size_t stride = warp_scratch_bytes(ncols, nb);
    size_t warps = size_t(sm_count) * std::max<uint32_t>(1, ctas_per_sm) * kWarpsPerBlock;
    while (warps > size_t(kWarpsPerBlock) && warps * stride > scratch_budget) warps -= kWarpsPerBlock;
    S->slots = uint32_t(warps);
    S->grid = uint32_t(warps / kWarpsPerBlock);
    S->max_span = max_span;
    check_cuda(cudaMalloc(&S->d_scratch, warps * stride), "cudaMalloc alignment service scratch");
    NwSvcArgs& A = S->args;
    memset(&A, 0, sizeof(A));
    A.base.scratch = static_cast<uint8_t*>(S->d_scratch);
    A.base.scratch_stride = stride;
    A.base.scratch_warps = uint32_t(warps);
    A.base.max_n = uint32_t(ncols);
    A.base.max_nb = uint32_t(nb);
    S->ring.set_large_first_every(large_first_every);
    A.jobs = static_cast<const NwJobDev*>(S->ring.records());
    A.q = S->ring.queue();
    check_cuda(cudaFuncSetAttribute(nw_service_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    kWarpsPerBlock * kMaxSym * 32 * 8),
               "cudaFuncSetAttribute");
    prefer_max_shared(reinterpret_cast<const void*>(nw_service_kernel));
    st_ = S.release();
    st_->ring.start(launch_nw_service, st_);
}

NwService::~NwService() {
    st_->ring.stop();
    cudaFree(st_->d_scratch);
    delete st_;
}

bool NwService::fits(uint32_t max_m, uint32_t max_n) const {
    return max_m <= st_->max_span && max_n <= st_->max_span;
}
uint32_t NwService::slots() const { return st_->slots; }
uint32_t NwService::launches() const { return st_->ring.launches(); }

void NwService::run_batch(const NwJobDev& job, const uint32_t* index, size_t n, int queue) {
    const size_t cap = st_->ring.max_batch();
    for (size_t b = 0; b < n; b += cap) st_->ring.run_batch(&job, index + b, std::min(cap, n - b), queue);
}

}  // namespace rb

// ---------------------------------------------------------------------------
// rb_nw_distance_noalloc: C entry point of the allocation-free variant.
namespace {

constexpr int kNoAllocMaxDevices = 64;

int noalloc_fail(char* err, uint32_t cap, int code, const char* fmt, ...) {
    if (err && cap) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(err, cap, fmt, ap);
        va_end(ap);
    }
    return code;
}

}  // namespace

extern "C" int rb_nw_distance_noalloc(const char* query, uint32_t query_length, const char* target,
                                      uint32_t target_length, int32_t* distance, void* stream, char* err,
                                      uint32_t err_capacity) {
    if (err && err_capacity) err[0] = '\0';
    if (!distance || (query_length && !query) || (target_length && !target))
        return noalloc_fail(err, err_capacity, RB_ERR_ARG, "rb_nw_distance_noalloc: null pointer argument");
    if (query_length > rb::kNoAllocMaxLen || target_length > rb::kNoAllocMaxLen)
        return noalloc_fail(err, err_capacity, RB_ERR_ARG,
                            "rb_nw_distance_noalloc: sequence length %llu exceeds the static scratch limit of %llu bytes",
                            (unsigned long long)std::max(query_length, target_length),
                            (unsigned long long)rb::kNoAllocMaxLen);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices)
        return noalloc_fail(err, err_capacity, RB_ERR_CUDA, "rb_nw_distance_noalloc: no usable current device (CUDA error %d, device %d)",
                            int(e), dev);
    // The scratch array's device address, looked up on every call: host code
    // cannot take the address of a __device__ variable directly, and after a
    // cudaDeviceReset (a new primary context) the module is loaded again and
    // the array can move, so a cached address could be stale. The lookup
    // allocates nothing. The device's first call also loads the module.
    void* scratch = nullptr;
    e = cudaGetSymbolAddress(&scratch, rb::g_noalloc_scratch);
    if (e != cudaSuccess || !scratch)
        return noalloc_fail(err, err_capacity, RB_ERR_CUDA, "rb_nw_distance_noalloc: scratch address lookup failed: %s",
                            cudaGetErrorString(e));
    rb::nw_distance_noalloc_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(
        query, query_length, target, target_length, distance, static_cast<uint8_t*>(scratch));
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return noalloc_fail(err, err_capacity, RB_ERR_CUDA, "rb_nw_distance_noalloc: launch failed: %s",
                            cudaGetErrorString(e));
    return RB_OK;
}
