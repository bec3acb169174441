// Checkpoint schedule of the Born adjoint / FWI gradient (host arithmetic only).
//
// A record of `blocks` coarse blocks is cut into nseg = ceil(blocks / L)
// segments aligned to the END of the record: segment s covers blocks
// [start(s), start(s+1)), every segment has L blocks except the first, which
// holds the remainder.  The forward pass decimates the velocity of the last
// segment into the velocity slots as it goes; the adjoint pass recomputes each
// earlier segment s from the state saved at the start of block start(s)-1
// (none for s = 0, which starts from rest) through block
// min(start(s+1)+1, blocks-1), so that V[start(s) .. min(start(s+1)+1, blocks)]
// is complete for the imaging condition of its adjoint blocks.
#pragma once

#include <algorithm>

namespace e3d {
namespace schedule {

inline int segments(int blocks, int L) { return (blocks + L - 1) / L; }

inline int segStart(int blocks, int L, int nseg, int s) { return std::max(0, blocks - (nseg - s) * L); }

// Source blocks the adjoint pass recomputes: every segment but the last, each
// from the block before it (none before the first) to two blocks past its end.
inline int recomputedBlocks(int blocks, int L) {
  const int nseg = segments(blocks, L);
  int r = 0;
  for (int s = 0; s + 1 < nseg; s++) {
    const int b0 = s == 0 ? 0 : segStart(blocks, L, nseg, s) - 1;
    r += std::min(segStart(blocks, L, nseg, s + 1) + 1, blocks - 1) - b0 + 1;
  }
  return r;
}

}  // namespace schedule
}  // namespace e3d
