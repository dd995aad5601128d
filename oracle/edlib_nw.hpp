// ORACLE — test infrastructure only. Never linked into, or called by, the
// racon_b200 product path. Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg may use it, and only as the checker.
//
// CPU restatement of the edit-distance aligner racon calls for every overlap
// without a CIGAR:
//   src/overlap.cpp:205-224  edlibAlign(q, |q|, t, |t|,
//       edlibNewAlignConfig(-1, EDLIB_MODE_NW, EDLIB_TASK_PATH, nullptr, 0))
//       followed by edlibAlignmentToCigar(..., EDLIB_CIGAR_STANDARD)
//   test/racon_test.cpp:16-25  edlibAlign(..., edlibDefaultAlignConfig())
//       (NW, distance only) as the golden-test metric.
// edlib itself (github.com/martinsos/edlib, API 1.2.x; the submodule pin is
// not recoverable from the reference tree) is absent. This file restates its
// published algorithm (Myers 1999 bit-vector, Hyyro's block/band extension,
// Sosic & Sikic 2017): 64-bit blocks, Ukkonen band with k doubling from 64,
// traceback from stored blocks when the stored data is below 1 MiB, else a
// Hirschberg split at the middle target column.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace oracle {

// Edit operations in alignment order, same codes as edlib's EDLIB_EDOP_*.
enum EditOp : uint8_t { kMatch = 0, kInsert = 1, kDelete = 2, kMismatch = 3 };

struct NwResult {
    int edit_distance = -1;
    std::vector<uint8_t> ops;  // empty when task is distance only
    bool ok = false;
};

// Global (NW) alignment. with_path=false returns only the distance.
NwResult nw_align(const char* query, int query_length, const char* target,
                  int target_length, bool with_path);

// Standard CIGAR (M/I/D run lengths) of an op string, as edlibAlignmentToCigar
// with EDLIB_CIGAR_STANDARD produces it.
std::string ops_to_cigar(const std::vector<uint8_t>& ops);

}  // namespace oracle
