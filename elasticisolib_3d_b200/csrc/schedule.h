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
#include <cstddef>

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

// ---------------------------------------------------------------------------
// Memory plan.  Storage types: states 0 fp32, 1 fp16, 2 bf16 (-1 automatic);
// velocity slots 0 fp32, 1 fp16 (-1 automatic).  n = cells of the padded grid,
// ny = its y slices (one scale per field and y slice for 16-bit storage).
// ---------------------------------------------------------------------------
constexpr int kStateF32 = 0, kStateF16 = 1, kSlotF32 = 0, kSlotF16 = 1;

// One checkpoint: 18 fields (both leapfrog levels), plus scales when 16-bit.
inline double stateBytes(long long n, int ny, int type) {
  double b = 18.0 * (double)n * (type == kStateF32 ? 4 : 2);
  if (type != kStateF32) b += 18.0 * ny * sizeof(float) + 256;
  return b;
}

// FP16 velocity slot: three fields of n halves, padded to 256 B, then 3*ny scales.
inline size_t halfSlotValuesBytes(long long n) { return ((size_t)3 * n * 2 + 255) / 256 * 256; }
inline size_t halfSlotBytes(long long n, int ny) { return halfSlotValuesBytes(n) + (size_t)3 * ny * sizeof(float); }
inline double slotBytes(long long n, int ny, int vt) {
  return vt == kSlotF32 ? 3.0 * (double)n * sizeof(float) : (double)halfSlotBytes(n, ny);
}

// Checkpoints plus velocity slots of a plan with segment length L.  FP32 slots
// hold V[b .. b+L+2] of a segment starting at block b (the last one partial,
// from the recompute's final block); FP16 slots hold V[b .. b+L+1] plus four
// FP32 working slots (two accumulators while recomputing, a four-deep window
// V(t-1..t+2) for the imaging condition of a block).
inline double planBytes(long long n, int ny, int nts, int ck, int vt, int L) {
  const int nseg = segments(nts - 1, L);
  double b = (double)(nseg - 1) * stateBytes(n, ny, ck);
  if (vt == kSlotF32) b += (L + 3) * slotBytes(n, ny, kSlotF32);
  else b += (L + 2) * slotBytes(n, ny, kSlotF16) + 4 * slotBytes(n, ny, kSlotF32);
  return b;
}

struct Plan {
  int ck, vt, L;
};

// The plan for `budget` bytes.  Candidates: fp32 states + fp32 slots, fp16
// states + fp32 slots, fp16 states + fp16 slots (automatic states), or the
// given state type with fp32 then fp16 slots; a fixed slot type keeps only
// its candidates.  An explicit segment length takes the first candidate that
// fits it, else the last one.  Otherwise each candidate takes the longest
// segment that fits, and the plan that recomputes the fewest source blocks
// wins once a lower-precision plan is charged a margin (5% of the blocks for
// 16-bit states, 5% for 16-bit slots).  False when nothing fits.
inline bool choosePlan(long long n, int ny, int nts, double budget, int ckptType, int vType, int segment,
                       Plan& out) {
  const int blocks = nts - 1;
  const Plan autoList[3] = {{kStateF32, kSlotF32, 0}, {kStateF16, kSlotF32, 0}, {kStateF16, kSlotF16, 0}};
  const Plan typedList[2] = {{ckptType, kSlotF32, 0}, {ckptType, kSlotF16, 0}};
  const Plan* all = ckptType < 0 ? autoList : typedList;
  const int nAll = ckptType < 0 ? 3 : 2;
  Plan cands[3];
  int nc = 0;
  for (int i = 0; i < nAll; i++)
    if (vType < 0 || all[i].vt == vType) cands[nc++] = all[i];
  if (segment > 0) {
    const int l = std::min(segment, blocks);
    for (int i = 0; i < nc; i++)
      if (planBytes(n, ny, nts, cands[i].ck, cands[i].vt, l) <= budget || i + 1 == nc) {
        out = {cands[i].ck, cands[i].vt, l};
        return true;
      }
  }
  int best = -1;
  double bestCost = 0;
  for (int i = 0; i < nc; i++) {
    int l = blocks;
    while (l >= 1 && planBytes(n, ny, nts, cands[i].ck, cands[i].vt, l) > budget) l--;
    if (l < 1) continue;
    const double cost = recomputedBlocks(blocks, l) +
                        blocks * ((cands[i].ck != kStateF32 ? 0.05 : 0.0) + (cands[i].vt == kSlotF16 ? 0.05 : 0.0));
    if (best < 0 || cost < bestCost) {
      best = i;
      bestCost = cost;
      out = {cands[i].ck, cands[i].vt, l};
    }
  }
  return best >= 0;
}

}  // namespace schedule
}  // namespace e3d
