// CUDA kernels of the elastic 3D propagation engine (sm_100a).
//
// Stepper: one launch advances all nine components of one shot by one fine
// time step.  2.5D y-marching: a CTA owns a 32(z) x TX(x) column tile and
// walks a chunk of y-planes.  Per plane the eight fields that need z/x
// neighbours are staged in shared memory (tile plus a 4-cell halo, loaded
// cooperatively with 128-byte z rows); the six fields that need y neighbours
// keep an 8-deep register window.  The cosine sponge is fused: the reference
// damps both time levels after every step (dampCosineEdge_3D); here the new
// level is damped when written and the other level is damped when it is next
// read as the "old" level, which gives the same recursion without a second
// pass over 18 arrays.
#pragma once
#include <cuda.h>
#include "common.cuh"

namespace e3d {

constexpr int TZ = 32;
constexpr int HALO = 4;
constexpr int SZ = TZ + 2 * HALO;  // shared tile row length (z)

struct StepPtrs {
  float* o[NCOMP];        // old level in; new level out when nw is null (in place)
  float* nw[NCOMP];       // new level out (null: written over the old level)
  const float* c[NCOMP];  // current level
  const float* m[NMED];   // medium planes
  // optional Born secondary source injected inside the step (may be null)
  const float* ssL[NCOMP];
  const float* ssR[NCOMP];
  float ssWl, ssWr;
  // optional decimation of the new level into coarse accumulators (may be null)
  float* accL[NCOMP];
  float* accR[NCOMP];
  float accWl, accWr;
  int nAcc;               // number of leading components accumulated (3 or 9)
  int accInitL;           // 1: accL is written (v*accWl) rather than accumulated; TMA stepper only
  // mode 2 with a dual state: c[] holds the medium-premultiplied current level
  // and the step also writes the premultiplied new level here (may be null)
  float* oP[NCOMP];
};

// A "device set" concatenates the regular-grid points of the nine
// components: component k owns entries [off[k], off[k+1]) of pos.
struct SparseSet {
  const long long* pos;
  int off[NCOMP + 1];
};

// Medium-premultiplied wavefield at one cell (stepAdjGpuBorn_3D, kernelsElaGpu_3D.cu:864-920).
__device__ __forceinline__ void premultiply(const float* v, float rhox, float rhoy, float rhoz, float l2m, float lam,
                                            float muxz, float muxy, float muyz, float* q) {
  q[VX] = v[VX] * rhox;
  q[VY] = v[VY] * rhoy;
  q[VZ] = v[VZ] * rhoz;
  q[SXX] = v[SXX] * l2m + (v[SYY] + v[SZZ]) * lam;
  q[SYY] = v[SYY] * l2m + (v[SXX] + v[SZZ]) * lam;
  q[SZZ] = v[SZZ] * l2m + (v[SXX] + v[SYY]) * lam;
  q[SXZ] = v[SXZ] * muxz;
  q[SXY] = v[SXY] * muxy;
  q[SYZ] = v[SYZ] * muyz;
}

// Shared tiles: fields needing a z or x halo.
enum Tile { T_VX = 0, T_VY, T_VZ, T_SXX, T_SZZ, T_SXY, T_SXZ, T_SYZ, NTILE };
// Register windows: fields needing y neighbours.  Window k holds plane y+base+k
// with base -4 for backward (minus) and -3 for forward (plus) derivatives.
enum Queue { Q_VX = 0, Q_VY, Q_VZ, Q_SYY, Q_SXY, Q_SYZ, NQUEUE };
__device__ constexpr int qBase(int q) { return (q == Q_VY || q == Q_SXY || q == Q_SYZ) ? -3 : -4; }

// Field value entering the derivative: raw (modes 0/1) or medium-premultiplied
// (mode 2, stepAdjGpuBorn_3D kernelsElaGpu_3D.cu:864-920).
template <int MODE>
__device__ __forceinline__ float tileValue(const StepPtrs& p, int t, long long i) {
  if (MODE != STEP_ADJ_EXACT) {
    const int comp = (t == T_VX) ? VX : (t == T_VY) ? VY : (t == T_VZ) ? VZ : (t == T_SXX) ? SXX
                   : (t == T_SZZ) ? SZZ : (t == T_SXY) ? SXY : (t == T_SXZ) ? SXZ : SYZ;
    return __ldg(p.c[comp] + i);
  } else {
    switch (t) {
      case T_VX: return __ldg(p.c[VX] + i) * __ldg(p.m[RHOX] + i);
      case T_VY: return __ldg(p.c[VY] + i) * __ldg(p.m[RHOY] + i);
      case T_VZ: return __ldg(p.c[VZ] + i) * __ldg(p.m[RHOZ] + i);
      case T_SXX: return __ldg(p.c[SXX] + i) * __ldg(p.m[L2M] + i) +
                         (__ldg(p.c[SYY] + i) + __ldg(p.c[SZZ] + i)) * __ldg(p.m[LAM] + i);
      case T_SZZ: return __ldg(p.c[SZZ] + i) * __ldg(p.m[L2M] + i) +
                         (__ldg(p.c[SXX] + i) + __ldg(p.c[SYY] + i)) * __ldg(p.m[LAM] + i);
      case T_SXY: return __ldg(p.c[SXY] + i) * __ldg(p.m[MUXY] + i);
      case T_SXZ: return __ldg(p.c[SXZ] + i) * __ldg(p.m[MUXZ] + i);
      default: return __ldg(p.c[SYZ] + i) * __ldg(p.m[MUYZ] + i);
    }
  }
}

template <int MODE>
__device__ __forceinline__ float queueValue(const StepPtrs& p, int q, long long i) {
  if (MODE != STEP_ADJ_EXACT) {
    const int comp = (q == Q_VX) ? VX : (q == Q_VY) ? VY : (q == Q_VZ) ? VZ : (q == Q_SYY) ? SYY
                   : (q == Q_SXY) ? SXY : SYZ;
    return __ldg(p.c[comp] + i);
  } else {
    switch (q) {
      case Q_VX: return __ldg(p.c[VX] + i) * __ldg(p.m[RHOX] + i);
      case Q_VY: return __ldg(p.c[VY] + i) * __ldg(p.m[RHOY] + i);
      case Q_VZ: return __ldg(p.c[VZ] + i) * __ldg(p.m[RHOZ] + i);
      case Q_SYY: return __ldg(p.c[SYY] + i) * __ldg(p.m[L2M] + i) +
                         (__ldg(p.c[SXX] + i) + __ldg(p.c[SZZ] + i)) * __ldg(p.m[LAM] + i);
      case Q_SXY: return __ldg(p.c[SXY] + i) * __ldg(p.m[MUXY] + i);
      default: return __ldg(p.c[SYZ] + i) * __ldg(p.m[MUYZ] + i);
    }
  }
}

__device__ __forceinline__ float dWin(const float* w, const float* c) {
  return c[0] * (w[4] - w[3]) + c[1] * (w[5] - w[2]) + c[2] * (w[6] - w[1]) + c[3] * (w[7] - w[0]);
}
// forward (+) / backward (-) 8th-order staggered derivatives along a shared-tile axis of stride s
__device__ __forceinline__ float dPlus(const float* t, int i, int s, const float* c) {
  return c[0] * (t[i + s] - t[i]) + c[1] * (t[i + 2 * s] - t[i - s]) + c[2] * (t[i + 3 * s] - t[i - 2 * s]) +
         c[3] * (t[i + 4 * s] - t[i - 3 * s]);
}
__device__ __forceinline__ float dMinus(const float* t, int i, int s, const float* c) {
  return c[0] * (t[i] - t[i - s]) + c[1] * (t[i + s] - t[i - 2 * s]) + c[2] * (t[i + 2 * s] - t[i - 3 * s]) +
         c[3] * (t[i + 3 * s] - t[i - 4 * s]);
}

// One fine time step for a y-chunk of one (z,x) tile.
//   MODE 0: new = G*(G*old + M D(cur))              (stepFwdGpu_3D)
//   MODE 1: new = G*(G*old - M D(cur))              (stepAdjGpu_3D)
//   MODE 2: new = G*(G*old - D(M cur))              (stepAdjGpuBorn_3D)
// G is the sponge taper at the cell.  Optional extras: a Born secondary source
// added before damping, and decimation of the damped new level.
template <int MODE, int TX>
__global__ void __launch_bounds__(TZ * TX) kStep(StepPtrs p, GridConst g, int yChunk) {
  constexpr int SX = TX + 2 * HALO;
  constexpr int TILE = SZ * SX;
  __shared__ float tile[NTILE][TILE];

  const int tz = threadIdx.x, tx = threadIdx.y;
  const int tid = tx * TZ + tz;
  const int z0 = FAT + blockIdx.x * TZ, x0 = FAT + blockIdx.y * TX;
  const int iz = z0 + tz, ix = x0 + tx;
  const bool active = (iz < g.nz - FAT) && (ix < g.nx - FAT);
  const int yBeg = FAT + blockIdx.z * yChunk;
  const int yEnd = min(yBeg + yChunk, g.ny - FAT);
  const long long ys = g.yStride;
  const long long col = (long long)ix * g.nz + iz;

  float w[NQUEUE][8];
  if (active) {
#pragma unroll
    for (int q = 0; q < NQUEUE; q++) {
#pragma unroll
      for (int k = 0; k < 7; k++) w[q][k] = queueValue<MODE>(p, q, (long long)(yBeg + qBase(q) + k) * ys + col);
    }
  }

  const int lc = (tx + HALO) * SZ + (tz + HALO);  // this thread's centre in the tile
  for (int y = yBeg; y < yEnd; y++) {
    const long long ic = (long long)y * ys + col;
    float ov[NCOMP], mv[NMED];
    if (active) {
#pragma unroll
      for (int q = 0; q < NQUEUE; q++) w[q][7] = queueValue<MODE>(p, q, ic + (long long)(qBase(q) + 7) * ys);
#pragma unroll
      for (int k = 0; k < NCOMP; k++) ov[k] = p.o[k][ic];
      if (MODE != STEP_ADJ_EXACT) {
#pragma unroll
        for (int k = 0; k < NMED; k++) mv[k] = __ldg(p.m[k] + ic);
      }
    }
    __syncthreads();  // previous plane's tile reads are complete
    {
      const long long plane = (long long)y * ys;
      for (int s = tid; s < TILE; s += TZ * TX) {
        const int lz = s % SZ, lx = s / SZ;
        const int gz = z0 - HALO + lz, gx = x0 - HALO + lx;
        const bool in = (gz < g.nz) && (gx < g.nx);
        const long long gi = plane + (long long)gx * g.nz + gz;
#pragma unroll
        for (int t = 0; t < NTILE; t++) tile[t][s] = in ? tileValue<MODE>(p, t, gi) : 0.0f;
      }
    }
    __syncthreads();
    if (active) {
      const float* cz = g.cz;
      const float* cx = g.cx;
      const float* cy = g.cy;
      const float dvx_dx = dPlus(tile[T_VX], lc, SZ, cx);
      const float dvy_dy = dWin(w[Q_VY], cy);
      const float dvz_dz = dPlus(tile[T_VZ], lc, 1, cz);
      const float fvx = dMinus(tile[T_SXX], lc, SZ, cx) + dWin(w[Q_SXY], cy) + dPlus(tile[T_SXZ], lc, 1, cz);
      const float fvy = dPlus(tile[T_SXY], lc, SZ, cx) + dWin(w[Q_SYY], cy) + dPlus(tile[T_SYZ], lc, 1, cz);
      const float fvz = dPlus(tile[T_SXZ], lc, SZ, cx) + dWin(w[Q_SYZ], cy) + dMinus(tile[T_SZZ], lc, 1, cz);
      const float fxy = dWin(w[Q_VX], cy) + dMinus(tile[T_VY], lc, SZ, cx);
      const float fxz = dMinus(tile[T_VX], lc, 1, cz) + dMinus(tile[T_VZ], lc, SZ, cx);
      const float fyz = dWin(w[Q_VZ], cy) + dMinus(tile[T_VY], lc, 1, cz);

      float up[NCOMP];
      if (MODE == STEP_ADJ_EXACT) {
        up[VX] = -fvx; up[VY] = -fvy; up[VZ] = -fvz;
        up[SXX] = -dvx_dx; up[SYY] = -dvy_dy; up[SZZ] = -dvz_dz;
        up[SXZ] = -fxz; up[SXY] = -fxy; up[SYZ] = -fyz;
      } else {
        const float sgn = (MODE == STEP_FWD) ? 1.0f : -1.0f;
        up[VX] = sgn * (mv[RHOX] * fvx);
        up[VY] = sgn * (mv[RHOY] * fvy);
        up[VZ] = sgn * (mv[RHOZ] * fvz);
        up[SXX] = sgn * (mv[L2M] * dvx_dx + mv[LAM] * (dvy_dy + dvz_dz));
        up[SYY] = sgn * (mv[L2M] * dvy_dy + mv[LAM] * (dvx_dx + dvz_dz));
        up[SZZ] = sgn * (mv[L2M] * dvz_dz + mv[LAM] * (dvx_dx + dvy_dy));
        up[SXZ] = sgn * (mv[MUXZ] * fxz);
        up[SXY] = sgn * (mv[MUXY] * fxy);
        up[SYZ] = sgn * (mv[MUYZ] * fyz);
      }
      const float G = taperAt(g, iz, ix, y);
      const bool hasSS = p.ssL[0] != nullptr;
      const bool hasAcc = p.accL[0] != nullptr;
#pragma unroll
      for (int k = 0; k < NCOMP; k++) {
        float v = G * ov[k] + up[k];
        if (hasSS) v += __ldg(p.ssL[k] + ic) * p.ssWl + __ldg(p.ssR[k] + ic) * p.ssWr;
        v *= G;
        (p.nw[0] ? p.nw[k] : p.o[k])[ic] = v;
        if (hasAcc && k < p.nAcc) {
          p.accL[k][ic] += v * p.accWl;
          if (p.accR[0] != nullptr) p.accR[k][ic] += v * p.accWr;
        }
      }
#pragma unroll
      for (int q = 0; q < NQUEUE; q++) {
#pragma unroll
        for (int k = 0; k < 7; k++) w[q][k] = w[q][k + 1];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Pipelined stepper (modes 0/1).  Same arithmetic as kStep; every per-plane
// global read (the eight halo tiles, the six y-window leads, the old level and
// the medium) is issued as 16-byte cp.async copies into a STAGES-deep ring of
// shared-memory stages, so plane y+1.. are in flight while plane y computes,
// with one barrier per plane.  Requires nz % 4 == 0 (16-byte rows), which the
// reference's block-size rule guarantees.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cpAsync16(float* smem, const float* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpAsyncWait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int TX>
struct PipeLayout {
  static constexpr int SX = TX + 2 * HALO;
  static constexpr int HALO_F = SZ * SX;       // floats per halo tile
  static constexpr int INT_F = TZ * TX;        // floats per interior tile
  static constexpr int HALO_CH = HALO_F / 4;   // 16-byte chunks per halo tile
  static constexpr int INT_CH = INT_F / 4;
  static constexpr int N_INT = NQUEUE + NCOMP + NMED;  // leads, old level, medium
  static constexpr int STAGE_F = NTILE * HALO_F + N_INT * INT_F;
  static constexpr int LEAD_OFF = NTILE * HALO_F;
  static constexpr int OLD_OFF = LEAD_OFF + NQUEUE * INT_F;
  static constexpr int MED_OFF = OLD_OFF + NCOMP * INT_F;
};

__device__ __forceinline__ int tileComp(int t) {
  return t == T_VX ? VX : t == T_VY ? VY : t == T_VZ ? VZ : t == T_SXX ? SXX : t == T_SZZ ? SZZ
         : t == T_SXY ? SXY : t == T_SXZ ? SXZ : SYZ;
}
__device__ __forceinline__ int queueComp(int q) {
  return q == Q_VX ? VX : q == Q_VY ? VY : q == Q_VZ ? VZ : q == Q_SYY ? SYY : q == Q_SXY ? SXY : SYZ;
}

template <int TX>
__device__ __forceinline__ void issuePlane(const StepPtrs& p, const GridConst& g, float* st, int y, int z0, int x0,
                                           int tid) {
  using L = PipeLayout<TX>;
  constexpr int NT = TZ * TX;
  const long long ys = g.yStride;
  const long long plane = (long long)y * ys;
  // halo tiles: rows of 40 floats starting at z0-4 (16-byte aligned when nz % 4 == 0)
  for (int c = tid; c < NTILE * L::HALO_CH; c += NT) {
    const int t = c / L::HALO_CH;
    const int r = c - t * L::HALO_CH;
    const int lx = r / (SZ / 4), q = r - lx * (SZ / 4);
    const int gz = z0 - HALO + 4 * q, gx = x0 - HALO + lx;
    const bool ok = (gz < g.nz) && (gx < g.nx);
    const float* src = p.c[tileComp(t)];
    cpAsync16(st + t * L::HALO_F + lx * SZ + 4 * q, ok ? src + plane + (long long)gx * g.nz + gz : src, ok);
  }
  // interior tiles: y-window leads, old level, medium
  for (int c = tid; c < L::N_INT * L::INT_CH; c += NT) {
    const int f = c / L::INT_CH;
    const int r = c - f * L::INT_CH;
    const int lx = r / (TZ / 4), q = r - lx * (TZ / 4);
    const int gz = z0 + 4 * q, gx = x0 + lx;
    const bool ok = (gz < g.nz) && (gx < g.nx);
    const float* src;
    long long off = (long long)gx * g.nz + gz;
    if (f < NQUEUE) {
      src = p.c[queueComp(f)];
      off += (long long)(y + qBase(f) + 7) * ys;
    } else if (f < NQUEUE + NCOMP) {
      src = p.o[f - NQUEUE];
      off += plane;
    } else {
      src = p.m[f - NQUEUE - NCOMP];
      off += plane;
    }
    cpAsync16(st + L::LEAD_OFF + f * L::INT_F + lx * TZ + 4 * q, ok ? src + off : src, ok);
  }
}

template <int MODE, int TX, int STAGES>
__global__ void __launch_bounds__(TZ * TX) kStepPipe(StepPtrs p, GridConst g, int yChunk) {
  using L = PipeLayout<TX>;
  extern __shared__ __align__(1024) float smem[];
  const int tz = threadIdx.x, tx = threadIdx.y;
  const int tid = tx * TZ + tz;
  const int z0 = FAT + blockIdx.x * TZ, x0 = FAT + blockIdx.y * TX;
  const int iz = z0 + tz, ix = x0 + tx;
  const bool active = (iz < g.nz - FAT) && (ix < g.nx - FAT);
  const int yBeg = FAT + blockIdx.z * yChunk;
  const int yEnd = min(yBeg + yChunk, g.ny - FAT);
  const long long ys = g.yStride;
  const long long col = (long long)ix * g.nz + iz;

  // prologue: planes yBeg .. yBeg+STAGES-2 in flight
#pragma unroll
  for (int s = 0; s < STAGES - 1; s++) {
    if (yBeg + s < yEnd) issuePlane<TX>(p, g, smem + s * L::STAGE_F, yBeg + s, z0, x0, tid);
    cpAsyncCommit();
  }
  float w[NQUEUE][8];
  if (active) {
#pragma unroll
    for (int q = 0; q < NQUEUE; q++) {
#pragma unroll
      for (int k = 0; k < 7; k++) w[q][k] = __ldg(p.c[queueComp(q)] + (long long)(yBeg + qBase(q) + k) * ys + col);
    }
  }
  const int lc = (tx + HALO) * SZ + (tz + HALO);
  const int li = tx * TZ + tz;
  int slot = 0;
  for (int y = yBeg; y < yEnd; y++) {
    cpAsyncWait<STAGES - 2>();
    __syncthreads();  // plane y visible to all; the stage read at y-1 is free again
    {
      const int yn = y + STAGES - 1;
      int ns = slot + STAGES - 1;
      if (ns >= STAGES) ns -= STAGES;
      if (yn < yEnd) issuePlane<TX>(p, g, smem + ns * L::STAGE_F, yn, z0, x0, tid);
      cpAsyncCommit();
    }
    const float* st = smem + slot * L::STAGE_F;
    if (active) {
#pragma unroll
      for (int q = 0; q < NQUEUE; q++) w[q][7] = st[L::LEAD_OFF + q * L::INT_F + li];
      const float* tl[NTILE];
#pragma unroll
      for (int t = 0; t < NTILE; t++) tl[t] = st + t * L::HALO_F;
      const float* cz = g.cz;
      const float* cx = g.cx;
      const float* cy = g.cy;
      const float dvx_dx = dPlus(tl[T_VX], lc, SZ, cx);
      const float dvy_dy = dWin(w[Q_VY], cy);
      const float dvz_dz = dPlus(tl[T_VZ], lc, 1, cz);
      const float fvx = dMinus(tl[T_SXX], lc, SZ, cx) + dWin(w[Q_SXY], cy) + dPlus(tl[T_SXZ], lc, 1, cz);
      const float fvy = dPlus(tl[T_SXY], lc, SZ, cx) + dWin(w[Q_SYY], cy) + dPlus(tl[T_SYZ], lc, 1, cz);
      const float fvz = dPlus(tl[T_SXZ], lc, SZ, cx) + dWin(w[Q_SYZ], cy) + dMinus(tl[T_SZZ], lc, 1, cz);
      const float fxy = dWin(w[Q_VX], cy) + dMinus(tl[T_VY], lc, SZ, cx);
      const float fxz = dMinus(tl[T_VX], lc, 1, cz) + dMinus(tl[T_VZ], lc, SZ, cx);
      const float fyz = dWin(w[Q_VZ], cy) + dMinus(tl[T_VY], lc, 1, cz);
      const float* mv = st + L::MED_OFF + li;
      const float* ov = st + L::OLD_OFF + li;
      const float sgn = (MODE == STEP_FWD) ? 1.0f : -1.0f;
      float up[NCOMP];
      up[VX] = sgn * (mv[RHOX * L::INT_F] * fvx);
      up[VY] = sgn * (mv[RHOY * L::INT_F] * fvy);
      up[VZ] = sgn * (mv[RHOZ * L::INT_F] * fvz);
      const float l2m = mv[L2M * L::INT_F], lam = mv[LAM * L::INT_F];
      up[SXX] = sgn * (l2m * dvx_dx + lam * (dvy_dy + dvz_dz));
      up[SYY] = sgn * (l2m * dvy_dy + lam * (dvx_dx + dvz_dz));
      up[SZZ] = sgn * (l2m * dvz_dz + lam * (dvx_dx + dvy_dy));
      up[SXZ] = sgn * (mv[MUXZ * L::INT_F] * fxz);
      up[SXY] = sgn * (mv[MUXY * L::INT_F] * fxy);
      up[SYZ] = sgn * (mv[MUYZ * L::INT_F] * fyz);
      const float G = taperAt(g, iz, ix, y);
      const long long ic = (long long)y * ys + col;
      const bool hasSS = p.ssL[0] != nullptr;
      const bool hasAcc = p.accL[0] != nullptr;
#pragma unroll
      for (int k = 0; k < NCOMP; k++) {
        float v = G * ov[k * L::INT_F] + up[k];
        if (hasSS) v += __ldg(p.ssL[k] + ic) * p.ssWl + __ldg(p.ssR[k] + ic) * p.ssWr;
        v *= G;
        (p.nw[0] ? p.nw[k] : p.o[k])[ic] = v;
        if (hasAcc && k < p.nAcc) {
          p.accL[k][ic] += v * p.accWl;
          if (p.accR[0] != nullptr) p.accR[k][ic] += v * p.accWr;
        }
      }
#pragma unroll
      for (int q = 0; q < NQUEUE; q++) {
#pragma unroll
        for (int k = 0; k < 7; k++) w[q][k] = w[q][k + 1];
      }
    }
    slot = (slot + 1 == STAGES) ? 0 : slot + 1;
  }
  cpAsyncWait<0>();
}

// ---------------------------------------------------------------------------
// TMA stepper.  One elected thread per CTA issues, for every plane, the 31
// tile copies of that plane (eight halo boxes 40 x (TX+8), six y-window lead
// boxes, nine old-level and eight medium boxes 32 x TX) as
// cp.async.bulk.tensor loads completing on one mbarrier per stage; the other
// threads only compute.  Boxes start at z0-4 or z0, multiples of 4 floats, so
// the innermost TMA coordinate is 16-byte aligned; boxes reaching past nz/nx
// are zero-filled by the hardware.  Every mbarrier wait is bounded: on
// expiry the CTA records the failure in g_e3dPipeError, waits (bounded) for
// its own copies in flight and returns.
// ---------------------------------------------------------------------------
struct TmaMaps {
  CUtensorMap halo[NTILE];   // current level, halo box
  CUtensorMap lead[NQUEUE];  // current level, interior box (y-window leads)
  CUtensorMap old[NCOMP];    // old level, interior box
  CUtensorMap med[NMED];     // medium, interior box
};

__device__ unsigned int g_e3dPipeError;

__device__ __forceinline__ unsigned smemAddr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbarInit(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbarExpectTx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smemAddr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbarTryWait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smemAddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: false when the iteration budget is exhausted
__device__ __forceinline__ bool mbarWaitBounded(unsigned long long* bar, unsigned parity) {
  for (int i = 0; i < (1 << 22); i++)
    if (mbarTryWait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tmaLoad3d(float* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                          unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smemAddr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smemAddr(bar))
      : "memory");
}

// 4D form: a (z, x, y, shot) map over the fields of several shots stacked per field.
__device__ __forceinline__ void tmaLoad4d(float* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                          unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];\n" ::"r"(smemAddr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smemAddr(bar))
      : "memory");
}

template <int TX>
__device__ __forceinline__ void tmaIssuePlane(const TmaMaps& mp, float* st, unsigned long long* bar, int y, int z0,
                                              int x0) {
  using L = PipeLayout<TX>;
  constexpr unsigned bytes = (unsigned)L::STAGE_F * 4u;
  mbarExpectTx(bar, bytes);
#pragma unroll
  for (int t = 0; t < NTILE; t++) tmaLoad3d(st + t * L::HALO_F, &mp.halo[t], z0 - HALO, x0 - HALO, y, bar);
#pragma unroll
  for (int q = 0; q < NQUEUE; q++)
    tmaLoad3d(st + L::LEAD_OFF + q * L::INT_F, &mp.lead[q], z0, x0, y + qBase(q) + 7, bar);
#pragma unroll
  for (int k = 0; k < NCOMP; k++) tmaLoad3d(st + L::OLD_OFF + k * L::INT_F, &mp.old[k], z0, x0, y, bar);
#pragma unroll
  for (int k = 0; k < NMED; k++) tmaLoad3d(st + L::MED_OFF + k * L::INT_F, &mp.med[k], z0, x0, y, bar);
}

template <int MODE, int TX, int STAGES>
__global__ void __launch_bounds__(TZ * TX) kStepTma(const __grid_constant__ TmaMaps mp, StepPtrs p, GridConst g,
                                                     int yChunk) {
  using L = PipeLayout<TX>;
  extern __shared__ __align__(1024) float smem[];
  __shared__ __align__(8) unsigned long long bars[STAGES];
  const int tz = threadIdx.x, tx = threadIdx.y;
  const int tid = tx * TZ + tz;
  const int z0 = FAT + blockIdx.x * TZ, x0 = FAT + blockIdx.y * TX;
  const int iz = z0 + tz, ix = x0 + tx;
  const bool active = (iz < g.nz - FAT) && (ix < g.nx - FAT);
  const int yBeg = FAT + blockIdx.z * yChunk;
  const int yEnd = min(yBeg + yChunk, g.ny - FAT);
  const long long ys = g.yStride;
  const long long col = (long long)ix * g.nz + iz;

  if (tid == 0) {
    for (int s = 0; s < STAGES; s++) mbarInit(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    for (int s = 0; s < STAGES - 1; s++)
      if (yBeg + s < yEnd) tmaIssuePlane<TX>(mp, smem + s * L::STAGE_F, &bars[s], yBeg + s, z0, x0);
  }
  float w[NQUEUE][8];
  if (active) {
#pragma unroll
    for (int q = 0; q < NQUEUE; q++) {
#pragma unroll
      for (int k = 0; k < 7; k++) w[q][k] = __ldg(p.c[queueComp(q)] + (long long)(yBeg + qBase(q) + k) * ys + col);
    }
  }
  // sponge distance: the z/x part is fixed for this thread
  const int dzx = min(min(topDistance(g, iz), ix - FAT), min(g.nz - iz - 1 - FAT, g.nx - ix - 1 - FAT));
  // the taper of the (z, x) part is fixed for this thread; the y part is uniform
  // over the CTA and is fetched at the top of each plane, ahead of the wait
  const float Gzx = (active && dzx < g.minPad) ? __ldg(g.taper + dzx) : 1.0f;
  const int lc = (tx + HALO) * SZ + (tz + HALO);
  const int li = tx * TZ + tz;
  int slot = 0;
  unsigned parity = 0;  // bit s: parity of the next completion of stage s
  for (int y = yBeg; y < yEnd; y++) {
    const int dyy = yDistance(g, y);
    const float Gy = dyy < g.minPad ? __ldg(g.taper + dyy) : 1.0f;
    const bool ok = mbarWaitBounded(&bars[slot], (parity >> slot) & 1u);
    // barrier: every thread is past plane y-1, so its stage can be refilled;
    // the OR makes an expired wait a CTA-wide decision
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(&g_e3dPipeError, 1u);
        // drain the copies this CTA still has in flight (bounded), then leave
        for (int s = 0; s < STAGES; s++) mbarWaitBounded(&bars[s], (parity >> s) & 1u);
      }
      __syncthreads();
      return;
    }
    parity ^= 1u << slot;
    if (tid == 0) {
      const int yn = y + STAGES - 1;
      int ns = slot + STAGES - 1;
      if (ns >= STAGES) ns -= STAGES;
      if (yn < yEnd) tmaIssuePlane<TX>(mp, smem + ns * L::STAGE_F, &bars[ns], yn, z0, x0);
    }
    const float* st = smem + slot * L::STAGE_F;
    if (active) {
      // Secondary sources or decimation accumulators of this cell, loaded before any
      // store of the step, so that they are issued together instead of one at a
      // time behind stores that the compiler cannot move them across.
      const long long ic = (long long)y * ys + col;
      const bool hasSS = p.ssL[0] != nullptr;
      const bool hasAcc = p.accL[0] != nullptr;
      const bool hasR = hasSS || p.accR[0] != nullptr;
      float preL[NCOMP], preR[NCOMP];
#pragma unroll
      for (int k = 0; k < NCOMP; k++) {
        preL[k] = 0.f;
        preR[k] = 0.f;
        if (hasSS) {
          preL[k] = __ldg(p.ssL[k] + ic);
          preR[k] = __ldg(p.ssR[k] + ic);
        } else if (hasAcc && k < p.nAcc) {
          if (!p.accInitL) preL[k] = p.accL[k][ic];
          if (hasR) preR[k] = p.accR[k][ic];
        }
      }
#pragma unroll
      for (int q = 0; q < NQUEUE; q++) w[q][7] = st[L::LEAD_OFF + q * L::INT_F + li];
      const float* tl[NTILE];
#pragma unroll
      for (int t = 0; t < NTILE; t++) tl[t] = st + t * L::HALO_F;
      const float* cz = g.cz;
      const float* cx = g.cx;
      const float* cy = g.cy;
      const float dvx_dx = dPlus(tl[T_VX], lc, SZ, cx);
      const float dvy_dy = dWin(w[Q_VY], cy);
      const float dvz_dz = dPlus(tl[T_VZ], lc, 1, cz);
      const float fvx = dMinus(tl[T_SXX], lc, SZ, cx) + dWin(w[Q_SXY], cy) + dPlus(tl[T_SXZ], lc, 1, cz);
      const float fvy = dPlus(tl[T_SXY], lc, SZ, cx) + dWin(w[Q_SYY], cy) + dPlus(tl[T_SYZ], lc, 1, cz);
      const float fvz = dPlus(tl[T_SXZ], lc, SZ, cx) + dWin(w[Q_SYZ], cy) + dMinus(tl[T_SZZ], lc, 1, cz);
      const float fxy = dWin(w[Q_VX], cy) + dMinus(tl[T_VY], lc, SZ, cx);
      const float fxz = dMinus(tl[T_VX], lc, 1, cz) + dMinus(tl[T_VZ], lc, SZ, cx);
      const float fyz = dWin(w[Q_VZ], cy) + dMinus(tl[T_VY], lc, 1, cz);
      const float* mv = st + L::MED_OFF + li;
      const float* ov = st + L::OLD_OFF + li;
      const float rhox = mv[RHOX * L::INT_F], rhoy = mv[RHOY * L::INT_F], rhoz = mv[RHOZ * L::INT_F];
      const float l2m = mv[L2M * L::INT_F], lam = mv[LAM * L::INT_F];
      const float muxz = mv[MUXZ * L::INT_F], muxy = mv[MUXY * L::INT_F], muyz = mv[MUYZ * L::INT_F];
      float up[NCOMP];
      if (MODE == STEP_ADJ_EXACT) {
        // tiles and window hold the premultiplied current level
        up[VX] = -fvx; up[VY] = -fvy; up[VZ] = -fvz;
        up[SXX] = -dvx_dx; up[SYY] = -dvy_dy; up[SZZ] = -dvz_dz;
        up[SXZ] = -fxz; up[SXY] = -fxy; up[SYZ] = -fyz;
      } else {
        const float sgn = (MODE == STEP_FWD) ? 1.0f : -1.0f;
        up[VX] = sgn * (rhox * fvx);
        up[VY] = sgn * (rhoy * fvy);
        up[VZ] = sgn * (rhoz * fvz);
        up[SXX] = sgn * (l2m * dvx_dx + lam * (dvy_dy + dvz_dz));
        up[SYY] = sgn * (l2m * dvy_dy + lam * (dvx_dx + dvz_dz));
        up[SZZ] = sgn * (l2m * dvz_dz + lam * (dvx_dx + dvy_dy));
        up[SXZ] = sgn * (muxz * fxz);
        up[SXY] = sgn * (muxy * fxy);
        up[SYZ] = sgn * (muyz * fyz);
      }
      // = taper[min(dzx, dyy)] when that distance is below minPad, else 1
      const float G = dyy < dzx ? Gy : Gzx;
      float nv[NCOMP];
#pragma unroll
      for (int k = 0; k < NCOMP; k++) {
        float v = G * ov[k * L::INT_F] + up[k];
        if (hasSS) v += preL[k] * p.ssWl + preR[k] * p.ssWr;
        v *= G;
        nv[k] = v;
      }
#pragma unroll
      for (int k = 0; k < NCOMP; k++) {
        (p.nw[0] ? p.nw[k] : p.o[k])[ic] = nv[k];
        if (hasAcc && k < p.nAcc) {
          p.accL[k][ic] = preL[k] + nv[k] * p.accWl;
          if (hasR) p.accR[k][ic] = preR[k] + nv[k] * p.accWr;
        }
      }
      if (MODE == STEP_ADJ_EXACT) {
        float q[NCOMP];
        premultiply(nv, rhox, rhoy, rhoz, l2m, lam, muxz, muxy, muyz, q);
#pragma unroll
        for (int k = 0; k < NCOMP; k++) p.oP[k][ic] = q[k];
      }
#pragma unroll
      for (int q = 0; q < NQUEUE; q++) {
#pragma unroll
        for (int k = 0; k < 7; k++) w[q][k] = w[q][k + 1];
      }
    }
    slot = (slot + 1 == STAGES) ? 0 : slot + 1;
  }
}

// ---------------------------------------------------------------------------
// Split stepper.  Within one step the velocity update reads only the current
// stresses and the stress update only the current velocities, so a launch can
// run them as two independent CTA roles: role V (blockIdx.z < yChunksV)
// advances vx, vy, vz; role S the six stresses.  Each role stages half the
// fields (five or three halo boxes, three y-window leads, its old level and
// medium: 5504 floats either way) and keeps three y-windows instead of six,
// so a CTA holds fewer registers and STAGES-deep TMA pipelines fit at higher
// occupancy.  The bytes moved and the arithmetic of every component are those
// of kStepTma (modes 0..2, the dual state of mode 2 included); the fused
// decimation and secondary sources stay with kStepTma.
// ---------------------------------------------------------------------------
struct SplitMaps {
  CUtensorMap v[14];  // halo SXX, SXY, SXZ, SYZ, SZZ; lead SXY, SYY, SYZ; old VX, VY, VZ; med RHOX, RHOY, RHOZ
  CUtensorMap s[17];  // halo VX, VY, VZ; lead VX, VY, VZ; old SXX..SYZ; med L2M, LAM, MUXZ, MUXY, MUYZ
};
constexpr int SPL_HALO_F = SZ * (8 + 2 * HALO);
constexpr int SPL_INT_F = TZ * 8;
constexpr int SPL_STAGE_F = 5 * SPL_HALO_F + 9 * SPL_INT_F;  // = 3 * SPL_HALO_F + 14 * SPL_INT_F
static_assert(5 * SPL_HALO_F + 9 * SPL_INT_F == 3 * SPL_HALO_F + 14 * SPL_INT_F, "role stages differ");

template <bool ROLE_S>
struct SplitRole {
  static constexpr int NH = ROLE_S ? 3 : 5;      // halo boxes
  static constexpr int NO = ROLE_S ? 6 : 3;      // old-level (and new-level) components
  static constexpr int NM = ROLE_S ? 5 : 3;      // medium planes
  static constexpr int C0 = ROLE_S ? SXX : VX;   // first component of the role
  static constexpr int M0 = ROLE_S ? L2M : RHOX; // first medium plane of the role
  static constexpr int LEAD_OFF = NH * SPL_HALO_F;
  static constexpr int OLD_OFF = LEAD_OFF + 3 * SPL_INT_F;
  static constexpr int MED_OFF = OLD_OFF + NO * SPL_INT_F;
  __device__ static constexpr int lead(int q) {  // y-window fields (component, base)
    return ROLE_S ? (q == 0 ? VX : q == 1 ? VY : VZ) : (q == 0 ? SXY : q == 1 ? SYY : SYZ);
  }
  __device__ static constexpr int base(int q) {
    return ROLE_S ? (q == 1 ? -3 : -4) : (q == 1 ? -4 : -3);
  }
};

// BATCH: the field maps are (z, x, y, shot) maps over stacked shots and `shot`
// selects the shot; the medium maps stay 3D (one medium for every shot).
template <bool ROLE_S, bool BATCH>
__device__ __forceinline__ void splitIssuePlane(const CUtensorMap* mp, float* st, unsigned long long* bar, int y,
                                                int z0, int x0, int shot) {
  using R = SplitRole<ROLE_S>;
  mbarExpectTx(bar, (unsigned)SPL_STAGE_F * 4u);
#pragma unroll
  for (int t = 0; t < R::NH; t++) {
    if (BATCH) tmaLoad4d(st + t * SPL_HALO_F, &mp[t], z0 - HALO, x0 - HALO, y, shot, bar);
    else tmaLoad3d(st + t * SPL_HALO_F, &mp[t], z0 - HALO, x0 - HALO, y, bar);
  }
#pragma unroll
  for (int q = 0; q < 3; q++) {
    if (BATCH) tmaLoad4d(st + R::LEAD_OFF + q * SPL_INT_F, &mp[R::NH + q], z0, x0, y + R::base(q) + 7, shot, bar);
    else tmaLoad3d(st + R::LEAD_OFF + q * SPL_INT_F, &mp[R::NH + q], z0, x0, y + R::base(q) + 7, bar);
  }
#pragma unroll
  for (int k = 0; k < R::NO; k++) {
    if (BATCH) tmaLoad4d(st + R::OLD_OFF + k * SPL_INT_F, &mp[R::NH + 3 + k], z0, x0, y, shot, bar);
    else tmaLoad3d(st + R::OLD_OFF + k * SPL_INT_F, &mp[R::NH + 3 + k], z0, x0, y, bar);
  }
#pragma unroll
  for (int k = 0; k < R::NM; k++)
    tmaLoad3d(st + R::MED_OFF + k * SPL_INT_F, &mp[R::NH + 3 + R::NO + k], z0, x0, y, bar);
}

template <int MODE, bool ROLE_S, int STAGES, bool BATCH>
__device__ __forceinline__ void splitRole(const CUtensorMap* mp, const StepPtrs& p, const GridConst& g, int yChunk,
                                          int chunk, float* smem, unsigned long long* bars, int nshots,
                                          long long shotStride) {
  using R = SplitRole<ROLE_S>;
  constexpr int TXS = 8;
  const int tz = threadIdx.x, tx = threadIdx.y;
  const int tid = tx * TZ + tz;
  // stacked shots: consecutive CTAs take one tile for consecutive shots, so a
  // medium tile fetched for one shot is in L2 for the others
  const int shot = BATCH ? (int)(blockIdx.x % nshots) : 0;
  const int tileZ = BATCH ? (int)(blockIdx.x / nshots) : (int)blockIdx.x;
  const long long soff = BATCH ? (long long)shot * shotStride : 0;
  const int z0 = FAT + tileZ * TZ, x0 = FAT + blockIdx.y * TXS;
  const int iz = z0 + tz, ix = x0 + tx;
  const bool active = (iz < g.nz - FAT) && (ix < g.nx - FAT);
  const int yBeg = FAT + chunk * yChunk;
  const int yEnd = min(yBeg + yChunk, g.ny - FAT);
  const long long ys = g.yStride;
  const long long col = (long long)ix * g.nz + iz;
  if (tid == 0) {
    for (int s = 0; s < STAGES; s++) mbarInit(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    for (int s = 0; s < STAGES - 1; s++)
      if (yBeg + s < yEnd)
        splitIssuePlane<ROLE_S, BATCH>(mp, smem + s * SPL_STAGE_F, &bars[s], yBeg + s, z0, x0, shot);
  }
  float w[3][8];
  if (active) {
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
      for (int k = 0; k < 7; k++)
        w[q][k] = __ldg(p.c[R::lead(q)] + soff + (long long)(yBeg + R::base(q) + k) * ys + col);
  }
  const int dzx = min(min(topDistance(g, iz), ix - FAT), min(g.nz - iz - 1 - FAT, g.nx - ix - 1 - FAT));
  const float Gzx = (active && dzx < g.minPad) ? __ldg(g.taper + dzx) : 1.0f;
  const int lc = (tx + HALO) * SZ + (tz + HALO);
  const int li = tx * TZ + tz;
  float* const* dst = p.nw[0] ? p.nw : p.o;
  int slot = 0;
  unsigned parity = 0;
  for (int y = yBeg; y < yEnd; y++) {
    const int dyy = yDistance(g, y);
    const float Gy = dyy < g.minPad ? __ldg(g.taper + dyy) : 1.0f;
    const bool ok = mbarWaitBounded(&bars[slot], (parity >> slot) & 1u);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(&g_e3dPipeError, 1u);
        for (int s = 0; s < STAGES; s++) mbarWaitBounded(&bars[s], (parity >> s) & 1u);
      }
      __syncthreads();
      return;
    }
    parity ^= 1u << slot;
    if (tid == 0) {
      const int yn = y + STAGES - 1;
      int ns = slot + STAGES - 1;
      if (ns >= STAGES) ns -= STAGES;
      if (yn < yEnd) splitIssuePlane<ROLE_S, BATCH>(mp, smem + ns * SPL_STAGE_F, &bars[ns], yn, z0, x0, shot);
    }
    const float* st = smem + slot * SPL_STAGE_F;
    if (active) {
      const long long ic = (long long)y * ys + col;
      const long long icf = ic + soff;  // this shot's cell in the stacked fields
#pragma unroll
      for (int q = 0; q < 3; q++) w[q][7] = st[R::LEAD_OFF + q * SPL_INT_F + li];
      const float* cz = g.cz;
      const float* cx = g.cx;
      const float* cy = g.cy;
      const float* mv = st + R::MED_OFF + li;
      const float* ov = st + R::OLD_OFF + li;
      const float G = dyy < dzx ? Gy : Gzx;
      float up[6], nv[6];
      if (!ROLE_S) {
        const float* tSXX = st;
        const float* tSXY = st + SPL_HALO_F;
        const float* tSXZ = st + 2 * SPL_HALO_F;
        const float* tSYZ = st + 3 * SPL_HALO_F;
        const float* tSZZ = st + 4 * SPL_HALO_F;
        const float fvx = dMinus(tSXX, lc, SZ, cx) + dWin(w[0], cy) + dPlus(tSXZ, lc, 1, cz);
        const float fvy = dPlus(tSXY, lc, SZ, cx) + dWin(w[1], cy) + dPlus(tSYZ, lc, 1, cz);
        const float fvz = dPlus(tSXZ, lc, SZ, cx) + dWin(w[2], cy) + dMinus(tSZZ, lc, 1, cz);
        const float rhox = mv[0], rhoy = mv[SPL_INT_F], rhoz = mv[2 * SPL_INT_F];
        if (MODE == STEP_ADJ_EXACT) {
          up[0] = -fvx; up[1] = -fvy; up[2] = -fvz;
        } else {
          const float sgn = (MODE == STEP_FWD) ? 1.0f : -1.0f;
          up[0] = sgn * (rhox * fvx);
          up[1] = sgn * (rhoy * fvy);
          up[2] = sgn * (rhoz * fvz);
        }
#pragma unroll
        for (int k = 0; k < 3; k++) nv[k] = G * (G * ov[k * SPL_INT_F] + up[k]);
#pragma unroll
        for (int k = 0; k < 3; k++) dst[VX + k][icf] = nv[k];
        if (MODE == STEP_ADJ_EXACT && p.oP[0]) {
          p.oP[VX][icf] = nv[0] * rhox;
          p.oP[VY][icf] = nv[1] * rhoy;
          p.oP[VZ][icf] = nv[2] * rhoz;
        }
      } else {
        const float* tVX = st;
        const float* tVY = st + SPL_HALO_F;
        const float* tVZ = st + 2 * SPL_HALO_F;
        const float dvx_dx = dPlus(tVX, lc, SZ, cx);
        const float dvy_dy = dWin(w[1], cy);
        const float dvz_dz = dPlus(tVZ, lc, 1, cz);
        const float fxy = dWin(w[0], cy) + dMinus(tVY, lc, SZ, cx);
        const float fxz = dMinus(tVX, lc, 1, cz) + dMinus(tVZ, lc, SZ, cx);
        const float fyz = dWin(w[2], cy) + dMinus(tVY, lc, 1, cz);
        const float l2m = mv[0], lam = mv[SPL_INT_F];
        const float muxz = mv[2 * SPL_INT_F], muxy = mv[3 * SPL_INT_F], muyz = mv[4 * SPL_INT_F];
        // local order SXX, SYY, SZZ, SXZ, SXY, SYZ (the component order from SXX on)
        if (MODE == STEP_ADJ_EXACT) {
          up[0] = -dvx_dx; up[1] = -dvy_dy; up[2] = -dvz_dz;
          up[3] = -fxz; up[4] = -fxy; up[5] = -fyz;
        } else {
          const float sgn = (MODE == STEP_FWD) ? 1.0f : -1.0f;
          up[0] = sgn * (l2m * dvx_dx + lam * (dvy_dy + dvz_dz));
          up[1] = sgn * (l2m * dvy_dy + lam * (dvx_dx + dvz_dz));
          up[2] = sgn * (l2m * dvz_dz + lam * (dvx_dx + dvy_dy));
          up[3] = sgn * (muxz * fxz);
          up[4] = sgn * (muxy * fxy);
          up[5] = sgn * (muyz * fyz);
        }
#pragma unroll
        for (int k = 0; k < 6; k++) nv[k] = G * (G * ov[k * SPL_INT_F] + up[k]);
#pragma unroll
        for (int k = 0; k < 6; k++) dst[SXX + k][icf] = nv[k];
        if (MODE == STEP_ADJ_EXACT && p.oP[0]) {
          p.oP[SXX][icf] = nv[0] * l2m + (nv[1] + nv[2]) * lam;
          p.oP[SYY][icf] = nv[1] * l2m + (nv[0] + nv[2]) * lam;
          p.oP[SZZ][icf] = nv[2] * l2m + (nv[0] + nv[1]) * lam;
          p.oP[SXZ][icf] = nv[3] * muxz;
          p.oP[SXY][icf] = nv[4] * muxy;
          p.oP[SYZ][icf] = nv[5] * muyz;
        }
      }
#pragma unroll
      for (int q = 0; q < 3; q++)
#pragma unroll
        for (int k = 0; k < 7; k++) w[q][k] = w[q][k + 1];
    }
    slot = (slot + 1 == STAGES) ? 0 : slot + 1;
  }
}

// ---------------------------------------------------------------------------
// Paired split stepper: the same tiles, TMA boxes, stages and barriers as
// kStepSplit, with each thread updating two consecutive z cells (iz, iz+1,
// iz even) of its column.  The two cells' stencil operands are read from shared
// memory as 8-byte pairs: a z derivative of both cells takes 5 paired loads
// instead of 16 single ones, an x derivative 8 instead of 16, and the old level,
// medium and y-window planes one paired load per field; the new level is
// stored as float2.  Each cell's arithmetic is kStepSplit's, term by term.
// blockDim (TZ/2, 8); forward and time-reversed modes.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 lds2(const float* t, int i) { return *reinterpret_cast<const float2*>(t + i); }

// z derivatives of cells i and i+1 (i even) of a shared tile row: forward (+) and backward (-)
__device__ __forceinline__ void dPlusZ2(const float* t, int i, const float* c, float& r0, float& r1) {
  const float2 a = lds2(t, i - 4), b = lds2(t, i - 2), m = lds2(t, i), d = lds2(t, i + 2), e = lds2(t, i + 4);
  r0 = c[0] * (m.y - m.x) + c[1] * (d.x - b.y) + c[2] * (d.y - b.x) + c[3] * (e.x - a.y);
  r1 = c[0] * (d.x - m.y) + c[1] * (d.y - m.x) + c[2] * (e.x - b.y) + c[3] * (e.y - b.x);
}
__device__ __forceinline__ void dMinusZ2(const float* t, int i, const float* c, float& r0, float& r1) {
  const float2 a = lds2(t, i - 4), b = lds2(t, i - 2), m = lds2(t, i), d = lds2(t, i + 2), e = lds2(t, i + 4);
  r0 = c[0] * (m.x - b.y) + c[1] * (m.y - b.x) + c[2] * (d.x - a.y) + c[3] * (d.y - a.x);
  r1 = c[0] * (m.y - m.x) + c[1] * (d.x - b.y) + c[2] * (d.y - b.x) + c[3] * (e.x - a.y);
}
// derivatives of cells i and i+1 along the tile's x axis (stride s, even)
__device__ __forceinline__ void dPlusX2(const float* t, int i, int s, const float* c, float& r0, float& r1) {
  const float2 m3 = lds2(t, i - 3 * s), m2 = lds2(t, i - 2 * s), m1 = lds2(t, i - s), p0 = lds2(t, i);
  const float2 p1 = lds2(t, i + s), p2 = lds2(t, i + 2 * s), p3 = lds2(t, i + 3 * s), p4 = lds2(t, i + 4 * s);
  r0 = c[0] * (p1.x - p0.x) + c[1] * (p2.x - m1.x) + c[2] * (p3.x - m2.x) + c[3] * (p4.x - m3.x);
  r1 = c[0] * (p1.y - p0.y) + c[1] * (p2.y - m1.y) + c[2] * (p3.y - m2.y) + c[3] * (p4.y - m3.y);
}
__device__ __forceinline__ void dMinusX2(const float* t, int i, int s, const float* c, float& r0, float& r1) {
  const float2 m4 = lds2(t, i - 4 * s), m3 = lds2(t, i - 3 * s), m2 = lds2(t, i - 2 * s), m1 = lds2(t, i - s);
  const float2 p0 = lds2(t, i), p1 = lds2(t, i + s), p2 = lds2(t, i + 2 * s), p3 = lds2(t, i + 3 * s);
  r0 = c[0] * (p0.x - m1.x) + c[1] * (p1.x - m2.x) + c[2] * (p2.x - m3.x) + c[3] * (p3.x - m4.x);
  r1 = c[0] * (p0.y - m1.y) + c[1] * (p1.y - m2.y) + c[2] * (p2.y - m3.y) + c[3] * (p3.y - m4.y);
}

template <int MODE, bool ROLE_S, int STAGES>
__device__ __forceinline__ void splitRolePair(const CUtensorMap* mp, const StepPtrs& p, const GridConst& g,
                                              int yChunk, int chunk, float* smem, unsigned long long* bars) {
  static_assert(MODE != STEP_ADJ_EXACT, "the paired split stepper takes the forward and time-reversed modes");
  using R = SplitRole<ROLE_S>;
  constexpr int TXS = 8;
  const int tz2 = threadIdx.x, tx = threadIdx.y;
  const int tid = tx * (TZ / 2) + tz2;
  const int z0 = FAT + blockIdx.x * TZ, x0 = FAT + blockIdx.y * TXS;
  const int iz = z0 + 2 * tz2, ix = x0 + tx;  // cells iz and iz+1
  // nz - FAT is even (nz % 4 == 0) and iz is even, so both cells are inside or both outside
  const bool active = (iz < g.nz - FAT) && (ix < g.nx - FAT);
  const int yBeg = FAT + chunk * yChunk;
  const int yEnd = min(yBeg + yChunk, g.ny - FAT);
  const long long ys = g.yStride;
  const long long col = (long long)ix * g.nz + iz;
  if (tid == 0) {
    for (int s = 0; s < STAGES; s++) mbarInit(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    for (int s = 0; s < STAGES - 1; s++)
      if (yBeg + s < yEnd) splitIssuePlane<ROLE_S, false>(mp, smem + s * SPL_STAGE_F, &bars[s], yBeg + s, z0, x0, 0);
  }
  float w0[3][8], w1[3][8];  // y-windows of cells iz and iz+1
  if (active) {
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
      for (int k = 0; k < 7; k++) {
        const float2 v = __ldg(reinterpret_cast<const float2*>(p.c[R::lead(q)] + (long long)(yBeg + R::base(q) + k) * ys + col));
        w0[q][k] = v.x;
        w1[q][k] = v.y;
      }
  }
  int dzx[2];
  float Gzx[2];
#pragma unroll
  for (int h = 0; h < 2; h++) {
    dzx[h] = min(min(topDistance(g, iz + h), ix - FAT), min(g.nz - iz - h - 1 - FAT, g.nx - ix - 1 - FAT));
    Gzx[h] = (active && dzx[h] < g.minPad) ? __ldg(g.taper + dzx[h]) : 1.0f;
  }
  const int lc = (tx + HALO) * SZ + (2 * tz2 + HALO);
  const int li = tx * TZ + 2 * tz2;
  float* const* dst = p.nw[0] ? p.nw : p.o;
  int slot = 0;
  unsigned parity = 0;
  for (int y = yBeg; y < yEnd; y++) {
    const int dyy = yDistance(g, y);
    const float Gy = dyy < g.minPad ? __ldg(g.taper + dyy) : 1.0f;
    const bool ok = mbarWaitBounded(&bars[slot], (parity >> slot) & 1u);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(&g_e3dPipeError, 1u);
        for (int s = 0; s < STAGES; s++) mbarWaitBounded(&bars[s], (parity >> s) & 1u);
      }
      __syncthreads();
      return;
    }
    parity ^= 1u << slot;
    if (tid == 0) {
      const int yn = y + STAGES - 1;
      int ns = slot + STAGES - 1;
      if (ns >= STAGES) ns -= STAGES;
      if (yn < yEnd) splitIssuePlane<ROLE_S, false>(mp, smem + ns * SPL_STAGE_F, &bars[ns], yn, z0, x0, 0);
    }
    const float* st = smem + slot * SPL_STAGE_F;
    if (active) {
      const long long ic = (long long)y * ys + col;
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const float2 v = lds2(st, R::LEAD_OFF + q * SPL_INT_F + li);
        w0[q][7] = v.x;
        w1[q][7] = v.y;
      }
      const float* cz = g.cz;
      const float* cx = g.cx;
      const float* cy = g.cy;
      const float G[2] = {dyy < dzx[0] ? Gy : Gzx[0], dyy < dzx[1] ? Gy : Gzx[1]};
      const float sgn = (MODE == STEP_FWD) ? 1.0f : -1.0f;
      if (!ROLE_S) {
        const float* tSXX = st;
        const float* tSXY = st + SPL_HALO_F;
        const float* tSXZ = st + 2 * SPL_HALO_F;
        const float* tSYZ = st + 3 * SPL_HALO_F;
        const float* tSZZ = st + 4 * SPL_HALO_F;
        float a0, a1, b0, b1, e0, e1;
        float fv[3][2];
        dMinusX2(tSXX, lc, SZ, cx, a0, a1);
        dPlusZ2(tSXZ, lc, cz, b0, b1);
        fv[0][0] = a0 + dWin(w0[0], cy) + b0;
        fv[0][1] = a1 + dWin(w1[0], cy) + b1;
        dPlusX2(tSXY, lc, SZ, cx, a0, a1);
        dPlusZ2(tSYZ, lc, cz, b0, b1);
        fv[1][0] = a0 + dWin(w0[1], cy) + b0;
        fv[1][1] = a1 + dWin(w1[1], cy) + b1;
        dPlusX2(tSXZ, lc, SZ, cx, a0, a1);
        dMinusZ2(tSZZ, lc, cz, e0, e1);
        fv[2][0] = a0 + dWin(w0[2], cy) + e0;
        fv[2][1] = a1 + dWin(w1[2], cy) + e1;
#pragma unroll
        for (int k = 0; k < 3; k++) {
          const float2 rho = lds2(st, R::MED_OFF + k * SPL_INT_F + li);
          const float2 ov = lds2(st, R::OLD_OFF + k * SPL_INT_F + li);
          float2 nv;
          nv.x = G[0] * (G[0] * ov.x + sgn * (rho.x * fv[k][0]));
          nv.y = G[1] * (G[1] * ov.y + sgn * (rho.y * fv[k][1]));
          *reinterpret_cast<float2*>(dst[VX + k] + ic) = nv;
        }
      } else {
        const float* tVX = st;
        const float* tVY = st + SPL_HALO_F;
        const float* tVZ = st + 2 * SPL_HALO_F;
        float dxx[2], dyy_[2], dzz[2], fxy[2], fxz[2], fyz[2], a0, a1, b0, b1;
        dPlusX2(tVX, lc, SZ, cx, dxx[0], dxx[1]);
        dyy_[0] = dWin(w0[1], cy);
        dyy_[1] = dWin(w1[1], cy);
        dPlusZ2(tVZ, lc, cz, dzz[0], dzz[1]);
        dMinusX2(tVY, lc, SZ, cx, a0, a1);
        fxy[0] = dWin(w0[0], cy) + a0;
        fxy[1] = dWin(w1[0], cy) + a1;
        dMinusZ2(tVX, lc, cz, a0, a1);
        dMinusX2(tVZ, lc, SZ, cx, b0, b1);
        fxz[0] = a0 + b0;
        fxz[1] = a1 + b1;
        dMinusZ2(tVY, lc, cz, a0, a1);
        fyz[0] = dWin(w0[2], cy) + a0;
        fyz[1] = dWin(w1[2], cy) + a1;
        const float2 l2m = lds2(st, R::MED_OFF + li), lam = lds2(st, R::MED_OFF + SPL_INT_F + li);
        const float2 muxz = lds2(st, R::MED_OFF + 2 * SPL_INT_F + li);
        const float2 muxy = lds2(st, R::MED_OFF + 3 * SPL_INT_F + li);
        const float2 muyz = lds2(st, R::MED_OFF + 4 * SPL_INT_F + li);
        const float L2M_[2] = {l2m.x, l2m.y}, LAM_[2] = {lam.x, lam.y};
        const float MXZ[2] = {muxz.x, muxz.y}, MXY[2] = {muxy.x, muxy.y}, MYZ[2] = {muyz.x, muyz.y};
        float up[6][2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          up[0][h] = sgn * (L2M_[h] * dxx[h] + LAM_[h] * (dyy_[h] + dzz[h]));
          up[1][h] = sgn * (L2M_[h] * dyy_[h] + LAM_[h] * (dxx[h] + dzz[h]));
          up[2][h] = sgn * (L2M_[h] * dzz[h] + LAM_[h] * (dxx[h] + dyy_[h]));
          up[3][h] = sgn * (MXZ[h] * fxz[h]);
          up[4][h] = sgn * (MXY[h] * fxy[h]);
          up[5][h] = sgn * (MYZ[h] * fyz[h]);
        }
#pragma unroll
        for (int k = 0; k < 6; k++) {
          const float2 ov = lds2(st, R::OLD_OFF + k * SPL_INT_F + li);
          float2 nv;
          nv.x = G[0] * (G[0] * ov.x + up[k][0]);
          nv.y = G[1] * (G[1] * ov.y + up[k][1]);
          *reinterpret_cast<float2*>(dst[SXX + k] + ic) = nv;
        }
      }
#pragma unroll
      for (int q = 0; q < 3; q++)
#pragma unroll
        for (int k = 0; k < 7; k++) {
          w0[q][k] = w0[q][k + 1];
          w1[q][k] = w1[q][k + 1];
        }
    }
    slot = (slot + 1 == STAGES) ? 0 : slot + 1;
  }
}

template <int MODE, int STAGES, int MINB>
__global__ void __launch_bounds__(TZ / 2 * 8, MINB) kStepSplitPair(const __grid_constant__ SplitMaps mp, StepPtrs p,
                                                                   GridConst g, int yChunk, int chunksV) {
  extern __shared__ __align__(1024) float smem[];
  __shared__ __align__(8) unsigned long long bars[STAGES];
  if ((int)blockIdx.z < chunksV) splitRolePair<MODE, false, STAGES>(mp.v, p, g, yChunk, blockIdx.z, smem, bars);
  else splitRolePair<MODE, true, STAGES>(mp.s, p, g, yChunk, blockIdx.z - chunksV, smem, bars);
}

// BATCH: nshots shots stacked per field (shot s at offset s * shotStride), field
// maps 4D, blockIdx.x = tile * nshots + shot; forward and time-reversed modes only.
template <int MODE, int STAGES, int MINB, bool BATCH = false>
__global__ void __launch_bounds__(TZ * 8, MINB) kStepSplit(const __grid_constant__ SplitMaps mp, StepPtrs p,
                                                            GridConst g, int yChunk, int chunksV, int nshots,
                                                            long long shotStride) {
  extern __shared__ __align__(1024) float smem[];
  __shared__ __align__(8) unsigned long long bars[STAGES];
  if ((int)blockIdx.z < chunksV)
    splitRole<MODE, false, STAGES, BATCH>(mp.v, p, g, yChunk, blockIdx.z, smem, bars, nshots, shotStride);
  else
    splitRole<MODE, true, STAGES, BATCH>(mp.s, p, g, yChunk, blockIdx.z - chunksV, smem, bars, nshots, shotStride);
}

// Recompute the premultiplied level at injected points (dual-state mode 2):
// after kInject changed raw values there.  The three normal stresses share
// the center-grid positions and are refreshed together by the sxx entries.
__global__ void kRefreshPremultiplied(StepPtrs p, SparseSet s) {
  const int ntot = s.off[NCOMP];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ntot) return;
  int k = 0;
#pragma unroll
  for (int c = 1; c < NCOMP; c++) k += (j >= s.off[c]);
  if (k == SYY || k == SZZ) return;
  const long long i = s.pos[j];
  switch (k) {
    case VX: p.oP[VX][i] = p.o[VX][i] * __ldg(p.m[RHOX] + i); break;
    case VY: p.oP[VY][i] = p.o[VY][i] * __ldg(p.m[RHOY] + i); break;
    case VZ: p.oP[VZ][i] = p.o[VZ][i] * __ldg(p.m[RHOZ] + i); break;
    case SXZ: p.oP[SXZ][i] = p.o[SXZ][i] * __ldg(p.m[MUXZ] + i); break;
    case SXY: p.oP[SXY][i] = p.o[SXY][i] * __ldg(p.m[MUXY] + i); break;
    case SYZ: p.oP[SYZ][i] = p.o[SYZ][i] * __ldg(p.m[MUYZ] + i); break;
    default: {
      const float sxx = p.o[SXX][i], syy = p.o[SYY][i], szz = p.o[SZZ][i];
      const float l2m = __ldg(p.m[L2M] + i), lam = __ldg(p.m[LAM] + i);
      p.oP[SXX][i] = sxx * l2m + (syy + szz) * lam;
      p.oP[SYY][i] = syy * l2m + (sxx + szz) * lam;
      p.oP[SZZ][i] = szz * l2m + (sxx + syy) * lam;
    }
  }
}

// Injection into the raw new level and the refresh of its premultiplied copy
// at the injected points in one launch (dual-state mode 2): kInject followed by
// kRefreshPremultiplied, without decimation accumulators.  The normal stresses
// share the center-grid points (equal counts, the same order), so the thread of
// the r-th sxx entry injects sxx, syy and szz at that point before
// premultiplying the three.
__global__ void kInjectRefresh(StepPtrs p, GridConst g, SparseSet s, const float* sigL, const float* sigR, float wl,
                               float wr) {
  const int ntot = s.off[NCOMP];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ntot) return;
  int k = 0;
#pragma unroll
  for (int c = 1; c < NCOMP; c++) k += (j >= s.off[c]);
  if (k == SYY || k == SZZ) return;
  const long long i = s.pos[j];
  const int iz = (int)(i % g.nz);
  const int ix = (int)((i / g.nz) % g.nx);
  const int iy = (int)(i / g.yStride);
  const float G = taperAt(g, iz, ix, iy);
  if (k == SXX) {
    const int r = j - s.off[SXX];
    float v[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const int jj = s.off[SXX + c] + r;
      const float add = G * (sigL[jj] * wl + sigR[jj] * wr);
      v[c] = p.o[SXX + c][i] + add;
      p.o[SXX + c][i] = v[c];
    }
    const float l2m = __ldg(p.m[L2M] + i), lam = __ldg(p.m[LAM] + i);
    p.oP[SXX][i] = v[0] * l2m + (v[1] + v[2]) * lam;
    p.oP[SYY][i] = v[1] * l2m + (v[0] + v[2]) * lam;
    p.oP[SZZ][i] = v[2] * l2m + (v[0] + v[1]) * lam;
    return;
  }
  const float add = G * (sigL[j] * wl + sigR[j] * wr);
  const float v = p.o[k][i] + add;
  p.o[k][i] = v;
  const int med = k == VX ? RHOX : k == VY ? RHOY : k == VZ ? RHOZ : k == SXZ ? MUXZ : k == SXY ? MUXY : MUYZ;
  p.oP[k][i] = v * __ldg(p.m[med] + i);
}

// Injection into a premultiplied-only adjoint state: the raw
// increment G*(sigL*wl + sigR*wr) of each component enters premultiplied,
// P += M * add, the normal stresses together as in kInjectRefresh.
__global__ void kInjectPremultiplied(StepPtrs p, GridConst g, SparseSet s, const float* sigL, const float* sigR,
                                     float wl, float wr) {
  const int ntot = s.off[NCOMP];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ntot) return;
  int k = 0;
#pragma unroll
  for (int c = 1; c < NCOMP; c++) k += (j >= s.off[c]);
  if (k == SYY || k == SZZ) return;
  const long long i = s.pos[j];
  const int iz = (int)(i % g.nz);
  const int ix = (int)((i / g.nz) % g.nx);
  const int iy = (int)(i / g.yStride);
  const float G = taperAt(g, iz, ix, iy);
  if (k == SXX) {
    const int r = j - s.off[SXX];
    float a[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const int jj = s.off[SXX + c] + r;
      a[c] = G * (sigL[jj] * wl + sigR[jj] * wr);
    }
    const float l2m = __ldg(p.m[L2M] + i), lam = __ldg(p.m[LAM] + i);
    p.o[SXX][i] += a[0] * l2m + (a[1] + a[2]) * lam;
    p.o[SYY][i] += a[1] * l2m + (a[0] + a[2]) * lam;
    p.o[SZZ][i] += a[2] * l2m + (a[0] + a[1]) * lam;
    return;
  }
  const float add = G * (sigL[j] * wl + sigR[j] * wr);
  const int med = k == VX ? RHOX : k == VY ? RHOY : k == VZ ? RHOZ : k == SXZ ? MUXZ : k == SXY ? MUXY : MUYZ;
  p.o[k][i] += add * __ldg(p.m[med] + i);
}

// Largest condition number of the normal-stress block of the premultiplication
// over the updated cells, as the bits of a non-negative float (for atomicMax);
// a cell whose block or shear, density planes are not positive counts as +inf.
__global__ void kPremultiplyCondition(StepPtrs p, GridConst g, unsigned* out) {
  const float* const* m = p.m;
  const long long ncell = g.n;
  float worst = 0.0f;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ncell;
       i += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(i % g.nz);
    const int ix = (int)((i / g.nz) % g.nx);
    const int iy = (int)(i / g.yStride);
    if (iz < FAT || iz >= g.nz - FAT || ix < FAT || ix >= g.nx - FAT || iy < FAT || iy >= g.ny - FAT) continue;
    const float a = __ldg(m[L2M] + i), b = __ldg(m[LAM] + i);
    const float e1 = a - b, e2 = a + 2.0f * b;
    float c = (e1 > 0.0f && e2 > 0.0f) ? fmaxf(e1, e2) / fminf(e1, e2) : INFINITY;
    if (!(__ldg(m[RHOX] + i) > 0.0f && __ldg(m[RHOY] + i) > 0.0f && __ldg(m[RHOZ] + i) > 0.0f &&
          __ldg(m[MUXZ] + i) > 0.0f && __ldg(m[MUXY] + i) > 0.0f && __ldg(m[MUYZ] + i) > 0.0f))
      c = INFINITY;
    worst = fmaxf(worst, c);
  }
  for (int o = 16; o > 0; o >>= 1) worst = fmaxf(worst, __shfl_xor_sync(0xffffffffu, worst, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(worst));
}

// ---------------------------------------------------------------------------
// TMA stepper, second form.  Differences from kStepTma:
//  * the y-window is a ring of 8 registers addressed by (k + R) & 7 with the
//    plane loop unrolled by 8, so no register moves per plane;
//  * OM_SMEM = false: the old level and the medium are read with plain
//    coalesced loads (issued right after the barrier), which shrinks a stage
//    to the eight halo boxes and six lead boxes so more CTAs fit per SM.
// ---------------------------------------------------------------------------
template <int TX, bool OM_SMEM>
struct Tma2Layout {
  using B = PipeLayout<TX>;
  static constexpr int HALO_F = B::HALO_F;
  static constexpr int INT_F = B::INT_F;
  static constexpr int LEAD_OFF = NTILE * HALO_F;
  static constexpr int OLD_OFF = LEAD_OFF + NQUEUE * INT_F;
  static constexpr int MED_OFF = OLD_OFF + NCOMP * INT_F;
  static constexpr int STAGE_F = OM_SMEM ? B::STAGE_F : LEAD_OFF + NQUEUE * INT_F;
};

template <int TX, bool OM_SMEM>
__device__ __forceinline__ void tma2IssuePlane(const TmaMaps& mp, float* st, unsigned long long* bar, int y, int z0,
                                               int x0) {
  using L = Tma2Layout<TX, OM_SMEM>;
  constexpr unsigned bytes = (unsigned)L::STAGE_F * 4u;
  mbarExpectTx(bar, bytes);
#pragma unroll
  for (int t = 0; t < NTILE; t++) tmaLoad3d(st + t * L::HALO_F, &mp.halo[t], z0 - HALO, x0 - HALO, y, bar);
#pragma unroll
  for (int q = 0; q < NQUEUE; q++)
    tmaLoad3d(st + L::LEAD_OFF + q * L::INT_F, &mp.lead[q], z0, x0, y + qBase(q) + 7, bar);
  if (OM_SMEM) {
#pragma unroll
    for (int k = 0; k < NCOMP; k++) tmaLoad3d(st + L::OLD_OFF + k * L::INT_F, &mp.old[k], z0, x0, y, bar);
#pragma unroll
    for (int k = 0; k < NMED; k++) tmaLoad3d(st + L::MED_OFF + k * L::INT_F, &mp.med[k], z0, x0, y, bar);
  }
}

template <int R>
__device__ __forceinline__ float dRing(const float* w, const float* c) {
  return c[0] * (w[(4 + R) & 7] - w[(3 + R) & 7]) + c[1] * (w[(5 + R) & 7] - w[(2 + R) & 7]) +
         c[2] * (w[(6 + R) & 7] - w[(1 + R) & 7]) + c[3] * (w[(7 + R) & 7] - w[(0 + R) & 7]);
}

template <int MODE, int TX, int STAGES, bool OM_SMEM>
struct Tma2State {
  const TmaMaps* mp;
  const StepPtrs* p;
  const GridConst* g;
  float* smem;
  unsigned long long* bars;
  int tid, z0, x0, iz, ix, yEnd, dzx, lc, li;
  bool active;
  long long col;
  int slot;
  unsigned parity;
  float w[NQUEUE][8];
};

// One plane with window rotation R.  Returns false if the CTA must stop.
template <int MODE, int TX, int STAGES, bool OM_SMEM, int R>
__device__ __forceinline__ bool tma2Plane(Tma2State<MODE, TX, STAGES, OM_SMEM>& S, int y) {
  using L = Tma2Layout<TX, OM_SMEM>;
  const StepPtrs& p = *S.p;
  const GridConst& g = *S.g;
  const bool ok = mbarWaitBounded(&S.bars[S.slot], (S.parity >> S.slot) & 1u);
  if (__syncthreads_or(!ok)) {
    if (S.tid == 0) {
      atomicExch(&g_e3dPipeError, 1u);
      for (int s = 0; s < STAGES; s++) mbarWaitBounded(&S.bars[s], (S.parity >> s) & 1u);
    }
    __syncthreads();
    return false;
  }
  S.parity ^= 1u << S.slot;
  if (S.tid == 0) {
    const int yn = y + STAGES - 1;
    int ns = S.slot + STAGES - 1;
    if (ns >= STAGES) ns -= STAGES;
    if (yn < S.yEnd) tma2IssuePlane<TX, OM_SMEM>(*S.mp, S.smem + ns * L::STAGE_F, &S.bars[ns], yn, S.z0, S.x0);
  }
  const float* st = S.smem + S.slot * L::STAGE_F;
  if (S.active) {
    const long long ic = (long long)y * g.yStride + S.col;
    float ovr[NCOMP], mvr[NMED];
    if (!OM_SMEM) {
#pragma unroll
      for (int k = 0; k < NCOMP; k++) ovr[k] = p.o[k][ic];
#pragma unroll
      for (int k = 0; k < NMED; k++) mvr[k] = __ldg(p.m[k] + ic);
    } else {
#pragma unroll
      for (int k = 0; k < NCOMP; k++) ovr[k] = st[L::OLD_OFF + k * L::INT_F + S.li];
#pragma unroll
      for (int k = 0; k < NMED; k++) mvr[k] = st[L::MED_OFF + k * L::INT_F + S.li];
    }
#pragma unroll
    for (int q = 0; q < NQUEUE; q++) S.w[q][(7 + R) & 7] = st[L::LEAD_OFF + q * L::INT_F + S.li];
    const float* tl[NTILE];
#pragma unroll
    for (int t = 0; t < NTILE; t++) tl[t] = st + t * L::HALO_F;
    const int lc = S.lc;
    const float* cz = g.cz;
    const float* cx = g.cx;
    const float* cy = g.cy;
    const float dvx_dx = dPlus(tl[T_VX], lc, SZ, cx);
    const float dvy_dy = dRing<R>(S.w[Q_VY], cy);
    const float dvz_dz = dPlus(tl[T_VZ], lc, 1, cz);
    const float fvx = dMinus(tl[T_SXX], lc, SZ, cx) + dRing<R>(S.w[Q_SXY], cy) + dPlus(tl[T_SXZ], lc, 1, cz);
    const float fvy = dPlus(tl[T_SXY], lc, SZ, cx) + dRing<R>(S.w[Q_SYY], cy) + dPlus(tl[T_SYZ], lc, 1, cz);
    const float fvz = dPlus(tl[T_SXZ], lc, SZ, cx) + dRing<R>(S.w[Q_SYZ], cy) + dMinus(tl[T_SZZ], lc, 1, cz);
    const float fxy = dRing<R>(S.w[Q_VX], cy) + dMinus(tl[T_VY], lc, SZ, cx);
    const float fxz = dMinus(tl[T_VX], lc, 1, cz) + dMinus(tl[T_VZ], lc, SZ, cx);
    const float fyz = dRing<R>(S.w[Q_VZ], cy) + dMinus(tl[T_VY], lc, 1, cz);
    const float sgn = (MODE == STEP_FWD) ? 1.0f : -1.0f;
    float up[NCOMP];
    up[VX] = sgn * (mvr[RHOX] * fvx);
    up[VY] = sgn * (mvr[RHOY] * fvy);
    up[VZ] = sgn * (mvr[RHOZ] * fvz);
    up[SXX] = sgn * (mvr[L2M] * dvx_dx + mvr[LAM] * (dvy_dy + dvz_dz));
    up[SYY] = sgn * (mvr[L2M] * dvy_dy + mvr[LAM] * (dvx_dx + dvz_dz));
    up[SZZ] = sgn * (mvr[L2M] * dvz_dz + mvr[LAM] * (dvx_dx + dvy_dy));
    up[SXZ] = sgn * (mvr[MUXZ] * fxz);
    up[SXY] = sgn * (mvr[MUXY] * fxy);
    up[SYZ] = sgn * (mvr[MUYZ] * fyz);
    const int d = min(S.dzx, yDistance(g, y));
    const float G = d < g.minPad ? __ldg(g.taper + d) : 1.0f;
    const bool hasSS = p.ssL[0] != nullptr;
    const bool hasAcc = p.accL[0] != nullptr;
#pragma unroll
    for (int k = 0; k < NCOMP; k++) {
      float v = G * ovr[k] + up[k];
      if (hasSS) v += __ldg(p.ssL[k] + ic) * p.ssWl + __ldg(p.ssR[k] + ic) * p.ssWr;
      v *= G;
      (p.nw[0] ? p.nw[k] : p.o[k])[ic] = v;
      if (hasAcc && k < p.nAcc) {
        p.accL[k][ic] += v * p.accWl;
        if (p.accR[0] != nullptr) p.accR[k][ic] += v * p.accWr;
      }
    }
  }
  S.slot = (S.slot + 1 == STAGES) ? 0 : S.slot + 1;
  return true;
}

template <int MODE, int TX, int STAGES, bool OM_SMEM, int MINB>
__global__ void __launch_bounds__(TZ * TX, MINB) kStepTma2(const __grid_constant__ TmaMaps mp, StepPtrs p,
                                                            GridConst g, int yChunk) {
  using L = Tma2Layout<TX, OM_SMEM>;
  extern __shared__ __align__(1024) float smem[];
  __shared__ __align__(8) unsigned long long bars[STAGES];
  Tma2State<MODE, TX, STAGES, OM_SMEM> S;
  S.mp = &mp;
  S.p = &p;
  S.g = &g;
  S.smem = smem;
  S.bars = bars;
  const int tz = threadIdx.x, tx = threadIdx.y;
  S.tid = tx * TZ + tz;
  S.z0 = FAT + blockIdx.x * TZ;
  S.x0 = FAT + blockIdx.y * TX;
  S.iz = S.z0 + tz;
  S.ix = S.x0 + tx;
  S.active = (S.iz < g.nz - FAT) && (S.ix < g.nx - FAT);
  const int yBeg = FAT + blockIdx.z * yChunk;
  S.yEnd = min(yBeg + yChunk, g.ny - FAT);
  S.col = (long long)S.ix * g.nz + S.iz;
  S.dzx = min(min(topDistance(g, S.iz), S.ix - FAT), min(g.nz - S.iz - 1 - FAT, g.nx - S.ix - 1 - FAT));
  S.lc = (tx + HALO) * SZ + (tz + HALO);
  S.li = tx * TZ + tz;
  S.slot = 0;
  S.parity = 0;
  if (S.tid == 0) {
    for (int s = 0; s < STAGES; s++) mbarInit(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (S.tid == 0) {
    for (int s = 0; s < STAGES - 1; s++)
      if (yBeg + s < S.yEnd) tma2IssuePlane<TX, OM_SMEM>(mp, smem + s * L::STAGE_F, &bars[s], yBeg + s, S.z0, S.x0);
  }
  if (S.active) {
#pragma unroll
    for (int q = 0; q < NQUEUE; q++) {
#pragma unroll
      for (int k = 0; k < 7; k++)
        S.w[q][k] = __ldg(p.c[queueComp(q)] + (long long)(yBeg + qBase(q) + k) * g.yStride + S.col);
    }
  }
  int y = yBeg;
  for (; y + 8 <= S.yEnd; y += 8) {
    if (!tma2Plane<MODE, TX, STAGES, OM_SMEM, 0>(S, y)) return;
    if (!tma2Plane<MODE, TX, STAGES, OM_SMEM, 1>(S, y + 1)) return;
    if (!tma2Plane<MODE, TX, STAGES, OM_SMEM, 2>(S, y + 2)) return;
    if (!tma2Plane<MODE, TX, STAGES, OM_SMEM, 3>(S, y + 3)) return;
    if (!tma2Plane<MODE, TX, STAGES, OM_SMEM, 4>(S, y + 4)) return;
    if (!tma2Plane<MODE, TX, STAGES, OM_SMEM, 5>(S, y + 5)) return;
    if (!tma2Plane<MODE, TX, STAGES, OM_SMEM, 6>(S, y + 6)) return;
    if (!tma2Plane<MODE, TX, STAGES, OM_SMEM, 7>(S, y + 7)) return;
  }
  // tail: fewer than 8 planes; rotation continues from 0
  const int r = S.yEnd - y;
  if (r > 0 && !tma2Plane<MODE, TX, STAGES, OM_SMEM, 0>(S, y)) return;
  if (r > 1 && !tma2Plane<MODE, TX, STAGES, OM_SMEM, 1>(S, y + 1)) return;
  if (r > 2 && !tma2Plane<MODE, TX, STAGES, OM_SMEM, 2>(S, y + 2)) return;
  if (r > 3 && !tma2Plane<MODE, TX, STAGES, OM_SMEM, 3>(S, y + 3)) return;
  if (r > 4 && !tma2Plane<MODE, TX, STAGES, OM_SMEM, 4>(S, y + 4)) return;
  if (r > 5 && !tma2Plane<MODE, TX, STAGES, OM_SMEM, 5>(S, y + 5)) return;
  if (r > 6 && !tma2Plane<MODE, TX, STAGES, OM_SMEM, 6>(S, y + 6)) return;
}

// ---------------------------------------------------------------------------
// Sparse signal kernels.  A "device set" concatenates the regular-grid points
// of the nine components: component k owns entries [off[k], off[k+1]) of pos.
// Signals are time-major on the device: sig[t*ntot + j].
// ---------------------------------------------------------------------------

// field[pos] += G(pos) * (sig[its]*wl + sig[its+1]*wr)
// (ker_inject_source_* / ker_inject_data_*, kernelsElaGpu_3D.cu:11-52; the
// source enters before the sponge, hence the taper at the point.)
__device__ __forceinline__ void injectAt(const StepPtrs& p, const GridConst& g, const SparseSet& s,
                                         const float* sigL, const float* sigR, float wl, float wr) {
  const int ntot = s.off[NCOMP];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ntot) return;
  int k = 0;
#pragma unroll
  for (int c = 1; c < NCOMP; c++) k += (j >= s.off[c]);
  const long long pos = s.pos[j];
  const float v = sigL[j] * wl + sigR[j] * wr;
  const int iz = (int)(pos % g.nz);
  const int ix = (int)((pos / g.nz) % g.nx);
  const int iy = (int)((pos / g.yStride) % g.ny);  // positions of stacked shots carry shot * n
  const float add = taperAt(g, iz, ix, iy) * v;
  p.o[k][pos] += add;
  // keep a decimation that the stepper fused in consistent with the injected value
  if (p.accL[0] != nullptr && k < p.nAcc) {
    p.accL[k][pos] += add * p.accWl;
    if (p.accR[0] != nullptr) p.accR[k][pos] += add * p.accWr;
  }
}

// Check of a device position table before any injection or recording: every
// entry must be an updated cell (not in the FAT ring, not outside the grid), as
// the host path requires of host tables.  Reads the table only; a bad entry
// sets *bad, which the host reads back.  With shots > 1 the table indexes that
// many grids stacked one after another (shot s at offset s * nz*nx*ny).
__global__ void kCheckPositions(const long long* pos, int n, int nz, int nx, int ny, int shots, unsigned* bad) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const long long p = pos[j];
  const long long ys = (long long)nz * nx;
  bool ok = p >= 0 && p < ys * ny * shots;
  if (ok) {
    const long long iz = p % nz, ix = (p / nz) % nx, iy = (p / ys) % ny;
    ok = iz >= FAT && iz < nz - FAT && ix >= FAT && ix < nx - FAT && iy >= FAT && iy < ny - FAT;
  }
  if (!ok) atomicOr(bad, 1u);
}

// The sponge taper written from kernel arguments (no host buffer involved).
struct TaperArg {
  float v[PAD_MAX];
};
__global__ void kWriteTaper(TaperArg t, float* out) {
  for (int i = threadIdx.x; i < PAD_MAX; i += blockDim.x) out[i] = t.v[i];
}

__global__ void kInject(StepPtrs p, GridConst g, SparseSet s, const float* sigL, const float* sigR, float wl,
                        float wr) {
  injectAt(p, g, s, sigL, sigR, wl, wr);
}

// The same with the coarse time index read on the device (time-major signals
// [nts][ntot], slices its and its+1): the form a replayed CUDA graph uses.
__global__ void kInjectIdx(StepPtrs p, GridConst g, SparseSet s, const float* sig, const int* its, float wl,
                           float wr) {
  const long long t = *its, ntot = s.off[NCOMP];
  injectAt(p, g, s, sig + t * ntot, sig + (t + 1) * ntot, wl, wr);
}

// Advance the device-side coarse time index of a replayed coarse block.
__global__ void kAdvanceIndex(int* its, int delta) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *its += delta;
}

// ---------------------------------------------------------------------------
// Free surface at the first interior row zs = FAT, the row of the normal
// stresses.  The reference parses freeSurface but applies it nowhere
// (fdParamElastic_3D.cpp:19, 44-45); this is new physics: stress imaging with
// the horizontal normal stresses re-derived at the surface.
//   * sxx, syy at zs: the step's lambda*d(vz)/dz term is replaced by the
//     stress-free relation d(vz)/dz = -lambda/(lambda+2mu) (d(vx)/dx + d(vy)/dy),
//     i.e. new += sgn*G*(-lam*dvz - lam^2/l2m*(dvx + dvy)) with the derivatives
//     of the current level (the ones the step used) and the 2dtw-scaled planes;
//   * szz = 0 at zs and odd about it: szz[zs-k] = -szz[zs+k], k = 1..FAT;
//   * sxz, syz (rows r at depth r-1/2) odd about zs: row r = -row 2*FAT+1-r,
//     r = 0..FAT (row FAT lies half a cell above the surface);
//   * vz rows 0..FAT (at or above zs-1/2) are ghosts held at zero.
// One thread per interior (x, y) column; sgn = +1 forward, -1 time-reversed.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float dPlusG(const float* a, long long i, long long s, const float* c) {
  return c[0] * (__ldg(a + i + s) - __ldg(a + i)) + c[1] * (__ldg(a + i + 2 * s) - __ldg(a + i - s)) +
         c[2] * (__ldg(a + i + 3 * s) - __ldg(a + i - 2 * s)) + c[3] * (__ldg(a + i + 4 * s) - __ldg(a + i - 3 * s));
}

__global__ void kFreeSurface(StepPtrs p, GridConst g, float sgn) {
  const int ix = FAT + blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = FAT + blockIdx.y;
  if (ix >= g.nx - FAT || iy >= g.ny - FAT) return;
  const long long ys = g.yStride;
  const long long col = (long long)iy * ys + (long long)ix * g.nz;
  const long long i = col + FAT;
  const float dvx = dPlusG(p.c[VX], i, g.nz, g.cx);
  const float dvy = dPlusG(p.c[VY], i, ys, g.cy);
  const float dvz = dPlusG(p.c[VZ], i, 1, g.cz);
  const float l2m = __ldg(p.m[L2M] + i), lam = __ldg(p.m[LAM] + i);
  const float G = taperAt(g, FAT, ix, iy);
  const float corr = sgn * G * (-lam * dvz - (lam * lam / l2m) * (dvx + dvy));
  p.o[SXX][i] += corr;
  p.o[SYY][i] += corr;
  p.o[SZZ][i] = 0.0f;
#pragma unroll
  for (int k = 1; k <= FAT; k++) p.o[SZZ][i - k] = -p.o[SZZ][i + k];
#pragma unroll
  for (int r = 0; r <= FAT; r++) {
    p.o[SXZ][col + r] = -p.o[SXZ][col + 2 * FAT + 1 - r];
    p.o[SYZ][col + r] = -p.o[SYZ][col + 2 * FAT + 1 - r];
    p.o[VZ][col + r] = 0.0f;
  }
}

// outL[j] += field[pos]*wl; outR[j] += field[pos]*wr, with outL/outR the
// time slices its and its+1 (ker_record_*, kernelsElaGpu_3D.cu:61-104)
__device__ __forceinline__ void recordAt(const StepPtrs& p, const SparseSet& s, float* outL, float* outR, float wl,
                                         float wr) {
  const int ntot = s.off[NCOMP];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ntot) return;
  int k = 0;
#pragma unroll
  for (int c = 1; c < NCOMP; c++) k += (j >= s.off[c]);
  const float v = p.o[k][s.pos[j]];
  outL[j] += v * wl;
  outR[j] += v * wr;
}

__global__ void kRecord(StepPtrs p, SparseSet s, float* outL, float* outR, float wl, float wr) {
  recordAt(p, s, outL, outR, wl, wr);
}

// Transpose of kInject: outL[j] += G(pos)*field[pos]*wl, outR[j] += G(pos)*field[pos]*wr, the
// taper G being the factor the injection applied at the point.
__global__ void kExtractSource(StepPtrs p, GridConst g, SparseSet s, float* outL, float* outR, float wl, float wr) {
  const int ntot = s.off[NCOMP];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ntot) return;
  int k = 0;
#pragma unroll
  for (int c = 1; c < NCOMP; c++) k += (j >= s.off[c]);
  const long long pos = s.pos[j];
  const int iz = (int)(pos % g.nz);
  const int ix = (int)((pos / g.nz) % g.nx);
  const int iy = (int)((pos / g.yStride) % g.ny);  // positions of stacked shots carry shot * n
  const float v = taperAt(g, iz, ix, iy) * p.o[k][pos];
  outL[j] += v * wl;
  outR[j] += v * wr;
}

__global__ void kRecordIdx(StepPtrs p, SparseSet s, float* out, const int* its, float wl, float wr) {
  const long long t = *its, ntot = s.off[NCOMP];
  recordAt(p, s, out + t * ntot, out + (t + 1) * ntot, wl, wr);
}

// ---------------------------------------------------------------------------
// Receiver traces between the regular acquisition points and the irregular
// receivers, one coarse time slice at a time (spaceInterpGpu_3D::forward /
// ::adjoint, spaceInterpGpu_3D.cpp:140-175).
// Gather: irr[r] = sum_f w[r*nf+f] * reg[slot[r*nf+f]], f ascending from 0,
//   r = k*nIrreg + i over the nine components.
// Spread: reg[j] = sum over the entries e of row j (ordered by receiver, then
//   tap) of w[e] * irr[idx[e]] -- the accumulation order of the reference's
//   device loop, without atomics.
// Table entries outside the slice (a slot >= nReg, a receiver row >= nRows)
// contribute nothing.
// ---------------------------------------------------------------------------
__global__ void kTraceGather(const float* __restrict__ reg, float* __restrict__ irr, int nRows, int nf,
                             const int* __restrict__ slot, const float* __restrict__ w, int nReg) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nRows) return;
  float acc = 0.f;
  for (int f = 0; f < nf; f++) {
    const int j = __ldg(slot + (long long)r * nf + f);
    if ((unsigned)j < (unsigned)nReg) acc += __ldg(w + (long long)r * nf + f) * __ldg(reg + j);
  }
  irr[r] = acc;
}

__global__ void kTraceSpread(const float* __restrict__ irr, float* __restrict__ reg, int nReg,
                             const int* __restrict__ rowPtr, const int* __restrict__ idx,
                             const float* __restrict__ w, int nRows) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nReg) return;
  float acc = 0.f;
  for (int e = __ldg(rowPtr + j); e < __ldg(rowPtr + j + 1); e++) {
    const int r = __ldg(idx + e);
    if ((unsigned)r < (unsigned)nRows) acc += __ldg(w + e) * __ldg(irr + r);
  }
  reg[j] = acc;
}

// ---------------------------------------------------------------------------
// Born scattering (imagingElaFwdGpu_3D, kernelsElaGpu_3D.cu:1232-1438) and
// imaging (imagingElaAdjGpu_3D, :1440-1641) at one coarse time t.
// V* are the decimated source velocities at t-1, t, t+1 (null outside [0,nts)).
// pert: drhox, drhoy, drhoz, dlame, dmu, dmuxz, dmuxy, dmuyz.
// ---------------------------------------------------------------------------
struct ImagingPtrs {
  const float* vPrev[3];
  const float* vCur[3];
  const float* vNext[3];
  float* ss[NCOMP];        // forward: secondary sources written; adjoint: decimated adjoint field read
  float* pert[NMED];       // forward: read; adjoint: accumulated
  float dtsInv;            // 1/(2 dts)
  int q3compat;
};

__device__ __forceinline__ float gPlus(const float* a, long long i, long long s, const float* c) {
  return c[0] * (__ldg(a + i + s) - __ldg(a + i)) + c[1] * (__ldg(a + i + 2 * s) - __ldg(a + i - s)) +
         c[2] * (__ldg(a + i + 3 * s) - __ldg(a + i - 2 * s)) + c[3] * (__ldg(a + i + 4 * s) - __ldg(a + i - 3 * s));
}
__device__ __forceinline__ float gMinus(const float* a, long long i, long long s, const float* c) {
  return c[0] * (__ldg(a + i) - __ldg(a + i - s)) + c[1] * (__ldg(a + i + s) - __ldg(a + i - 2 * s)) +
         c[2] * (__ldg(a + i + 2 * s) - __ldg(a + i - 3 * s)) + c[3] * (__ldg(a + i + 3 * s) - __ldg(a + i - 4 * s));
}

template <bool ADJ>
__global__ void kImaging(ImagingPtrs q, GridConst g) {
  const int iz = FAT + blockIdx.x * blockDim.x + threadIdx.x;
  const int ix = FAT + blockIdx.y * blockDim.y + threadIdx.y;
  const int iy = FAT + blockIdx.z;
  if (iz >= g.nz - FAT || ix >= g.nx - FAT) return;
  const long long i = (long long)iy * g.yStride + (long long)ix * g.nz + iz;
  const long long xs = g.nz, ys = g.yStride;
  const float* vx = q.vCur[0];
  const float* vy = q.vCur[1];
  const float* vz = q.vCur[2];
  const float dvx_dx = gPlus(vx, i, xs, g.cx);
  const float dvy_dy = gPlus(vy, i, ys, g.cy);
  const float dvz_dz = gPlus(vz, i, 1, g.cz);
  const float exz = gMinus(vx, i, 1, g.cz) + gMinus(vz, i, xs, g.cx);
  const float exy = gMinus(vx, i, ys, g.cy) + gMinus(vy, i, xs, g.cx);
  const float eyz = q.q3compat ? exz : (gMinus(vz, i, ys, g.cy) + gMinus(vy, i, 1, g.cz));
  float tder[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const float a = q.vPrev[k] ? __ldg(q.vPrev[k] + i) : 0.0f;
    const float b = q.vNext[k] ? __ldg(q.vNext[k] + i) : 0.0f;
    tder[k] = (a - b) * q.dtsInv;
  }
  const float div = dvx_dx + dvy_dy + dvz_dz;
  if (!ADJ) {
    q.ss[VX][i] = __ldg(q.pert[0] + i) * tder[0];
    q.ss[VY][i] = __ldg(q.pert[1] + i) * tder[1];
    q.ss[VZ][i] = __ldg(q.pert[2] + i) * tder[2];
    const float dl = __ldg(q.pert[3] + i), dm = __ldg(q.pert[4] + i);
    q.ss[SXX][i] = dl * div + 2.0f * dm * dvx_dx;
    q.ss[SYY][i] = dl * div + 2.0f * dm * dvy_dy;
    q.ss[SZZ][i] = dl * div + 2.0f * dm * dvz_dz;
    q.ss[SXZ][i] = __ldg(q.pert[5] + i) * exz;
    q.ss[SXY][i] = __ldg(q.pert[6] + i) * exy;
    q.ss[SYZ][i] = __ldg(q.pert[7] + i) * eyz;
  } else {
    const float axx = q.ss[SXX][i], ayy = q.ss[SYY][i], azz = q.ss[SZZ][i];
    q.pert[0][i] += q.ss[VX][i] * tder[0];
    q.pert[1][i] += q.ss[VY][i] * tder[1];
    q.pert[2][i] += q.ss[VZ][i] * tder[2];
    q.pert[3][i] += (axx + ayy + azz) * div;
    q.pert[4][i] += 2.0f * (dvx_dx * axx + dvy_dy * ayy + dvz_dz * azz);
    q.pert[5][i] += q.ss[SXZ][i] * exz;
    q.pert[6][i] += q.ss[SXY][i] * exy;
    q.pert[7][i] += q.ss[SYZ][i] * eyz;
  }
}

// ---------------------------------------------------------------------------
// Decimation from a ring of fine levels.  The gradient's passes keep the
// fine time levels of one coarse block in a ring of buffers (the stepper
// writes each new level beside the old one instead of over it) and decimate
// once per block, so that the steppers carry no accumulators: the reference's
// interpWavefieldVxVyVz_3D / extractInterpAdjointWavefield_3D
// (kernelsElaGpu_3D.cu:1646-1672, 1694-1714) weight every fine level of block
// b by the time-interpolation filter into the coarse samples b (left weight)
// and b+1 (right weight).
// ---------------------------------------------------------------------------
constexpr int RING_SUB_MAX = 8;  // longest block (internal sub) decimated from a ring

// Source velocity (3 fields): V[b] (left) and V[b+1] (right) from the levels of block b.
//   vl: 3 fields at vl + k*n; vlMode 0 skip, 1 accumulate onto V[b] (which holds
//   the right part of block b-1), 2 write; vr: written (the first part of V[b+1]).
struct DecimatePtrs {
  const float* lev[RING_SUB_MAX][3];
  float wl[RING_SUB_MAX], wr[RING_SUB_MAX];
  int nlev;
  float* vl;
  float* vr;
  int vlMode;
  long long n;
};

template <bool VEC>
__global__ void __launch_bounds__(256) kDecimateVelocity(DecimatePtrs d) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long start = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;  // velocity component
  if (VEC) {
    const long long nv = d.n / 4;
    for (long long j = start; j < nv; j += stride) {
      float4 l = make_float4(0.f, 0.f, 0.f, 0.f), r = l;
      if (d.vl && d.vlMode == 1) l = reinterpret_cast<const float4*>(d.vl + k * d.n)[j];
      for (int t = 0; t < d.nlev; t++) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(d.lev[t][k]) + j);
        l.x = fmaf(v.x, d.wl[t], l.x); l.y = fmaf(v.y, d.wl[t], l.y);
        l.z = fmaf(v.z, d.wl[t], l.z); l.w = fmaf(v.w, d.wl[t], l.w);
        r.x = fmaf(v.x, d.wr[t], r.x); r.y = fmaf(v.y, d.wr[t], r.y);
        r.z = fmaf(v.z, d.wr[t], r.z); r.w = fmaf(v.w, d.wr[t], r.w);
      }
      if (d.vl && d.vlMode) reinterpret_cast<float4*>(d.vl + k * d.n)[j] = l;
      if (d.vr) reinterpret_cast<float4*>(d.vr + k * d.n)[j] = r;
    }
  } else {
    for (long long j = start; j < d.n; j += stride) {
      float l = (d.vl && d.vlMode == 1) ? d.vl[k * d.n + j] : 0.f, r = 0.f;
      for (int t = 0; t < d.nlev; t++) {
        const float v = __ldg(d.lev[t][k] + j);
        l = fmaf(v, d.wl[t], l);
        r = fmaf(v, d.wr[t], r);
      }
      if (d.vl && d.vlMode) d.vl[k * d.n + j] = l;
      if (d.vr) d.vr[k * d.n + j] = r;
    }
  }
}

// Velocity terms of the Born imaging condition at one coarse time (the
// derivatives of imagingElaAdjGpu_3D, kernelsElaGpu_3D.cu:1440-1641, as kImaging).
struct VelTerms {
  float dvx_dx, dvy_dy, dvz_dz, exz, exy, eyz, tder[3];
};
__device__ __forceinline__ VelTerms velTerms(const float* const* vPrev, const float* const* vCur,
                                             const float* const* vNext, long long i, const GridConst& g,
                                             float dtsInv, int q3compat) {
  const long long xs = g.nz, ys = g.yStride;
  const float* vx = vCur[0];
  const float* vy = vCur[1];
  const float* vz = vCur[2];
  VelTerms t;
  t.dvx_dx = gPlus(vx, i, xs, g.cx);
  t.dvy_dy = gPlus(vy, i, ys, g.cy);
  t.dvz_dz = gPlus(vz, i, 1, g.cz);
  t.exz = gMinus(vx, i, 1, g.cz) + gMinus(vz, i, xs, g.cx);
  t.exy = gMinus(vx, i, ys, g.cy) + gMinus(vy, i, xs, g.cx);
  t.eyz = q3compat ? t.exz : (gMinus(vz, i, ys, g.cy) + gMinus(vy, i, 1, g.cz));
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const float a = vPrev[k] ? __ldg(vPrev[k] + i) : 0.0f;
    const float b = vNext[k] ? __ldg(vNext[k] + i) : 0.0f;
    t.tder[k] = (a - b) * dtsInv;
  }
  return t;
}

// Imaging contributions of the decimated adjoint field a (9 components) at one coarse time.
__device__ __forceinline__ void imagingTerms(const VelTerms& t, const float* a, float* out) {
  const float div = t.dvx_dx + t.dvy_dy + t.dvz_dz;
  out[0] = a[VX] * t.tder[0];
  out[1] = a[VY] * t.tder[1];
  out[2] = a[VZ] * t.tder[2];
  out[3] = (a[SXX] + a[SYY] + a[SZZ]) * div;
  out[4] = 2.0f * (t.dvx_dx * a[SXX] + t.dvy_dy * a[SYY] + t.dvz_dz * a[SZZ]);
  out[5] = a[SXZ] * t.exz;
  out[6] = a[SXY] * t.exy;
  out[7] = a[SYZ] * t.eyz;
}

// Adjoint imaging of one coarse block `its` from the ring of its fine adjoint
// levels (9 fields each, after injection): R = sum_t wr[t] lev[t] belongs to
// the coarse sample its+1, L = sum_t wl[t] lev[t] to its.
//   pert += I(V at its+1, R [+ carry when carryIn])      v[1..3] = V(its..its+2)
//   leftImage: pert += I(V at its, L)                     v[0..2] = V(its-1..its+1)
//   else:      carry = L (imaged with the block before, whose right part completes it)
struct ImagingBlockPtrs {
  const float* lev[RING_SUB_MAX][NCOMP];
  float wl[RING_SUB_MAX], wr[RING_SUB_MAX];
  int nlev;
  const float* v[4][3];  // V(its-1), V(its), V(its+1), V(its+2); null outside the record
  float* carry[NCOMP];
  int carryIn, leftImage;
  float* pert[NMED];
  float dtsInv;
  int q3compat;
  int prem;                // the levels are premultiplied: the sums are converted back to raw values
  const float* med[NMED];  // medium planes (prem)
};

// Both decimated sums of premultiplied levels back to raw values: the inverse of premultiply.
// The normal stresses invert the block [[a,b,b],[b,a,b],[b,b,a]] (a = lambda+2mu, b = lambda,
// scaled), whose inverse is [[a+b,-b,-b],[-b,a+b,-b],[-b,-b,a+b]] / ((a-b)(a+2b)); the other
// components divide by their own plane.  The reciprocals are taken once for both sums.
__device__ __forceinline__ void premSumsToRaw(const float* md, float* L, float* R) {
  const float r[6] = {__frcp_rn(md[RHOX]), __frcp_rn(md[RHOY]), __frcp_rn(md[RHOZ]),
                      __frcp_rn(md[MUXZ]), __frcp_rn(md[MUXY]), __frcp_rn(md[MUYZ])};
  const float det = __frcp_rn((md[L2M] - md[LAM]) * (md[L2M] + 2.0f * md[LAM]));
  const float apb = md[L2M] + md[LAM], lam = md[LAM];
  float* const sums[2] = {L, R};
#pragma unroll
  for (int s = 0; s < 2; s++) {
    float* v = sums[s];
    const float xx = v[SXX], yy = v[SYY], zz = v[SZZ];
    v[VX] *= r[0];
    v[VY] *= r[1];
    v[VZ] *= r[2];
    v[SXX] = (apb * xx - lam * (yy + zz)) * det;
    v[SYY] = (apb * yy - lam * (xx + zz)) * det;
    v[SZZ] = (apb * zz - lam * (xx + yy)) * det;
    v[SXZ] *= r[3];
    v[SXY] *= r[4];
    v[SYZ] *= r[5];
  }
}

// Decimated sums of one block from its levels: L (coarse sample its) and R (its+1), raw values,
// R including the carried left part of the block after it when carryIn.
__device__ __forceinline__ void blockSums(const ImagingBlockPtrs& q, long long ic, float* L, float* R) {
#pragma unroll
  for (int k = 0; k < NCOMP; k++) {
    L[k] = 0.f;
    R[k] = 0.f;
  }
  // a runtime loop over the levels: measured faster on B200 than the loads unrolled for a
  // compile-time level count (1.51 against 1.71 ms per block in the 288^3 gradient)
  for (int j = 0; j < q.nlev; j++) {
    const float wl = q.wl[j], wr = q.wr[j];
#pragma unroll
    for (int k = 0; k < NCOMP; k++) {
      const float a = __ldg(q.lev[j][k] + ic);
      L[k] = fmaf(a, wl, L[k]);
      R[k] = fmaf(a, wr, R[k]);
    }
  }
  if (q.prem) {
    float md[NMED];
#pragma unroll
    for (int k = 0; k < NMED; k++) md[k] = __ldg(q.med[k] + ic);
    premSumsToRaw(md, L, R);
  }
  if (q.carryIn) {
#pragma unroll
    for (int k = 0; k < NCOMP; k++) R[k] += q.carry[k][ic];
  }
}

__global__ void __launch_bounds__(256) kImagingBlock(ImagingBlockPtrs q, GridConst g) {
  const int iz = FAT + blockIdx.x * blockDim.x + threadIdx.x;
  const int ix = FAT + blockIdx.y * blockDim.y + threadIdx.y;
  const int iy = FAT + blockIdx.z;
  if (iz >= g.nz - FAT || ix >= g.nx - FAT) return;
  const long long i = (long long)iy * g.yStride + (long long)ix * g.nz + iz;
  float L[NCOMP], R[NCOMP];
  blockSums(q, i, L, R);
  float acc[NMED];
  {
    const VelTerms t1 = velTerms(q.v[1], q.v[2], q.v[3], i, g, q.dtsInv, q.q3compat);
    imagingTerms(t1, R, acc);
  }
  if (q.leftImage) {
    const VelTerms t0 = velTerms(q.v[0], q.v[1], q.v[2], i, g, q.dtsInv, q.q3compat);
    float accL[NMED];
    imagingTerms(t0, L, accL);
#pragma unroll
    for (int k = 0; k < NMED; k++) acc[k] += accL[k];
  } else {
#pragma unroll
    for (int k = 0; k < NCOMP; k++) q.carry[k][i] = L[k];
  }
#pragma unroll
  for (int k = 0; k < NMED; k++) q.pert[k][i] += acc[k];
}

// ---------------------------------------------------------------------------
// kImagingBlock as a 2.5D y-march: a CTA owns a 32(z) x 8(x) tile column and
// walks a chunk of y planes.  Per plane one elected thread issues TMA box
// copies of the three source velocities of the two coarse times the block
// images (halo boxes for the z/x derivatives, lead boxes for 8-deep register
// y-windows) into a 2-stage mbarrier pipeline; the adjoint levels, the time-
// derivative neighbours and the image planes are read with coalesced loads
// issued before the wait.  Same arithmetic, term by term, as kImagingBlock.
// Time index 1 = V(its+1) (right part), 0 = V(its) (left part, leftImage).
// Every wait is bounded as in kStepTma.
// ---------------------------------------------------------------------------
struct ImagingMaps {
  CUtensorMap halo[2][3];  // [time][vx, vy, vz], halo box
  CUtensorMap lead[2][3];  // [time][vx, vy, vz], interior box
};
constexpr int IMG_TX = 8;
constexpr int IMG_HALO_F = SZ * (IMG_TX + 2 * HALO);  // floats per halo box
constexpr int IMG_INT_F = TZ * IMG_TX;                // floats per interior box
constexpr int IMG_STAGE_F = 6 * IMG_HALO_F + 6 * IMG_INT_F;
// y-window bases: vy enters a forward y derivative (dvy/dy), vx and vz backward ones (exy, eyz)
__device__ constexpr int imgBase(int f) { return f == 1 ? -3 : -4; }

__device__ __forceinline__ void imgIssuePlane(const ImagingMaps& mp, float* st, unsigned long long* bar, int y,
                                              int z0, int x0, int ntimes) {
  const unsigned bytes = (unsigned)(ntimes * 3 * (IMG_HALO_F + IMG_INT_F)) * 4u;
  mbarExpectTx(bar, bytes);
  for (int t = 2 - ntimes; t < 2; t++)
#pragma unroll
    for (int f = 0; f < 3; f++) {
      tmaLoad3d(st + (t * 3 + f) * IMG_HALO_F, &mp.halo[t][f], z0 - HALO, x0 - HALO, y, bar);
      tmaLoad3d(st + 6 * IMG_HALO_F + (t * 3 + f) * IMG_INT_F, &mp.lead[t][f], z0, x0, y + imgBase(f) + 7, bar);
    }
}

// Velocity terms at one cell from the shared tiles (halo boxes of vx, vy, vz) and the y-windows
__device__ __forceinline__ VelTerms tileVelTerms(const float* tx_, const float* ty_, const float* tz_,
                                                 const float* wx, const float* wy, const float* wz, int lc,
                                                 const GridConst& g, float prev[3], float next[3], float dtsInv,
                                                 int q3compat) {
  VelTerms t;
  t.dvx_dx = dPlus(tx_, lc, SZ, g.cx);
  t.dvy_dy = dWin(wy, g.cy);
  t.dvz_dz = dPlus(tz_, lc, 1, g.cz);
  t.exz = dMinus(tx_, lc, 1, g.cz) + dMinus(tz_, lc, SZ, g.cx);
  t.exy = dWin(wx, g.cy) + dMinus(ty_, lc, SZ, g.cx);
  t.eyz = q3compat ? t.exz : (dWin(wz, g.cy) + dMinus(ty_, lc, 1, g.cz));
#pragma unroll
  for (int k = 0; k < 3; k++) t.tder[k] = (prev[k] - next[k]) * dtsInv;
  return t;
}

__global__ void __launch_bounds__(TZ * IMG_TX) kImagingTma(const __grid_constant__ ImagingMaps mp,
                                                           ImagingBlockPtrs q, GridConst g, int yChunk) {
  extern __shared__ __align__(1024) float smem[];
  __shared__ __align__(8) unsigned long long bars[2];
  const int tz = threadIdx.x, tx = threadIdx.y;
  const int tid = tx * TZ + tz;
  const int z0 = FAT + blockIdx.x * TZ, x0 = FAT + blockIdx.y * IMG_TX;
  const int iz = z0 + tz, ix = x0 + tx;
  const bool active = (iz < g.nz - FAT) && (ix < g.nx - FAT);
  const int yBeg = FAT + blockIdx.z * yChunk;
  const int yEnd = min(yBeg + yChunk, g.ny - FAT);
  const long long ys = g.yStride;
  const long long col = (long long)ix * g.nz + iz;
  const int ntimes = q.leftImage ? 2 : 1;
  const int t0 = 2 - ntimes;  // first time index present

  if (tid == 0) {
    for (int s = 0; s < 2; s++) mbarInit(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (tid == 0 && yBeg < yEnd) imgIssuePlane(mp, smem, &bars[0], yBeg, z0, x0, ntimes);
  // y-windows: w[t][f][k] holds plane y + imgBase(f) + k of field f at time t
  float w[2][3][8];
  if (active) {
#pragma unroll
    for (int t = 0; t < 2; t++)
#pragma unroll
      for (int f = 0; f < 3; f++)
#pragma unroll
        for (int k = 0; k < 7; k++)
          w[t][f][k] = (t >= t0) ? __ldg(q.v[t + 1][f] + (long long)(yBeg + imgBase(f) + k) * ys + col) : 0.f;
  }
  const int lc = (tx + HALO) * SZ + (tz + HALO);
  const int li = tx * TZ + tz;
  int slot = 0;
  unsigned parity = 0;
  for (int y = yBeg; y < yEnd; y++) {
    const long long ic = (long long)y * ys + col;
    // coalesced per-cell loads, issued ahead of the wait
    float L[NCOMP], R[NCOMP], pv[NMED], nxt[3], prv[3], cur0[3];
    if (active) {
      blockSums(q, ic, L, R);
#pragma unroll
      for (int k = 0; k < 3; k++) {
        nxt[k] = q.v[3][k] ? __ldg(q.v[3][k] + ic) : 0.f;                        // V(its+2)
        prv[k] = (q.leftImage && q.v[0][k]) ? __ldg(q.v[0][k] + ic) : 0.f;       // V(its-1)
        cur0[k] = q.leftImage ? 0.f : __ldg(q.v[1][k] + ic);                     // V(its) without its tile
      }
#pragma unroll
      for (int k = 0; k < NMED; k++) pv[k] = q.pert[k][ic];
    }
    const bool ok = mbarWaitBounded(&bars[slot], (parity >> slot) & 1u);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(&g_e3dPipeError, 1u);
        for (int s = 0; s < 2; s++) mbarWaitBounded(&bars[s], (parity >> s) & 1u);
      }
      __syncthreads();
      return;
    }
    parity ^= 1u << slot;
    if (tid == 0 && y + 1 < yEnd) imgIssuePlane(mp, smem + (slot ^ 1) * IMG_STAGE_F, &bars[slot ^ 1], y + 1, z0, x0, ntimes);
    const float* st = smem + slot * IMG_STAGE_F;
    if (active) {
#pragma unroll
      for (int t = 0; t < 2; t++)
#pragma unroll
        for (int f = 0; f < 3; f++)
          if (t >= t0) w[t][f][7] = st[6 * IMG_HALO_F + (t * 3 + f) * IMG_INT_F + li];
      const float* h1x = st + 3 * IMG_HALO_F;
      const float* h1y = st + 4 * IMG_HALO_F;
      const float* h1z = st + 5 * IMG_HALO_F;
      // right part: V(its+1); prev = V(its) (its tile when present), next = V(its+2)
      float prevR[3];
      if (q.leftImage) {
        prevR[0] = st[0 * IMG_HALO_F + lc];
        prevR[1] = st[1 * IMG_HALO_F + lc];
        prevR[2] = st[2 * IMG_HALO_F + lc];
      } else {
        prevR[0] = cur0[0];
        prevR[1] = cur0[1];
        prevR[2] = cur0[2];
      }
      float acc[NMED];
      {
        const VelTerms t1 = tileVelTerms(h1x, h1y, h1z, w[1][0], w[1][1], w[1][2], lc, g, prevR, nxt, q.dtsInv,
                                         q.q3compat);
        imagingTerms(t1, R, acc);
      }
      if (q.leftImage) {
        float nextL[3] = {h1x[lc], h1y[lc], h1z[lc]};  // V(its+1)
        const VelTerms tl = tileVelTerms(st, st + IMG_HALO_F, st + 2 * IMG_HALO_F, w[0][0], w[0][1], w[0][2], lc,
                                         g, prv, nextL, q.dtsInv, q.q3compat);
        float accL[NMED];
        imagingTerms(tl, L, accL);
#pragma unroll
        for (int k = 0; k < NMED; k++) acc[k] += accL[k];
      } else {
#pragma unroll
        for (int k = 0; k < NCOMP; k++) q.carry[k][ic] = L[k];
      }
#pragma unroll
      for (int k = 0; k < NMED; k++) q.pert[k][ic] = pv[k] + acc[k];
#pragma unroll
      for (int t = 0; t < 2; t++)
#pragma unroll
        for (int f = 0; f < 3; f++)
#pragma unroll
          for (int k = 0; k < 7; k++) w[t][f][k] = w[t][f][k + 1];
    }
    slot ^= 1;
  }
}

// ---------------------------------------------------------------------------
// kImagingTma with every per-cell operand of the block sums staged by TMA as
// well: per plane the elected thread also issues one interior box per level
// component (NLEV levels x 9) and, for premultiplied levels, per medium plane,
// so the sums read shared memory instead of waiting on NLEV rounds of
// dependent global loads.  The image planes, the carried part and the
// time-derivative neighbours stay coalesced loads issued before the wait.
// STAGES-deep pipeline; one CTA per SM (the stages take most of its shared
// memory).  Same arithmetic, in the same order, as kImagingTma.
// ---------------------------------------------------------------------------
template <int NLEV>
struct ImagingLevMaps {
  CUtensorMap halo[2][3];
  CUtensorMap lead[2][3];
  CUtensorMap lev[NLEV][NCOMP];
  CUtensorMap med[NMED];
};
// ITX-wide tiles (8: one CTA per SM; 4: three CTAs per SM with two stages)
__host__ __device__ constexpr int imgHaloF(int itx) { return SZ * (itx + 2 * HALO); }
__host__ __device__ constexpr int imgIntF(int itx) { return TZ * itx; }
__host__ __device__ constexpr int imgLevOff(int itx) { return 6 * imgHaloF(itx) + 6 * imgIntF(itx); }  // first level box
__host__ __device__ constexpr int imgLevStageF(int nlev, int itx) {
  return imgLevOff(itx) + (nlev * NCOMP + NMED) * imgIntF(itx);
}
// 8-wide tiles: three stages where they fit in 227 KB of shared memory, else two; 4-wide: two
__host__ __device__ constexpr int imgLevStages(int nlev, int itx) {
  return itx == 8 && 3 * imgLevStageF(nlev, itx) * 4 <= 227 * 1024 ? 3 : 2;
}

template <int NLEV, int ITX>
__device__ __forceinline__ void imgLevIssuePlane(const ImagingLevMaps<NLEV>& mp, float* st, unsigned long long* bar,
                                                 int y, int z0, int x0, int ntimes, bool prem) {
  constexpr int IMG_HALO_F = imgHaloF(ITX), IMG_INT_F = imgIntF(ITX), IMG_LEV_OFF = imgLevOff(ITX);
  const unsigned floats = (unsigned)(ntimes * 3 * (IMG_HALO_F + IMG_INT_F) + (NLEV * NCOMP + (prem ? NMED : 0)) * IMG_INT_F);
  mbarExpectTx(bar, floats * 4u);
  for (int t = 2 - ntimes; t < 2; t++)
#pragma unroll
    for (int f = 0; f < 3; f++) {
      tmaLoad3d(st + (t * 3 + f) * IMG_HALO_F, &mp.halo[t][f], z0 - HALO, x0 - HALO, y, bar);
      tmaLoad3d(st + 6 * IMG_HALO_F + (t * 3 + f) * IMG_INT_F, &mp.lead[t][f], z0, x0, y + imgBase(f) + 7, bar);
    }
#pragma unroll
  for (int j = 0; j < NLEV; j++)
#pragma unroll
    for (int k = 0; k < NCOMP; k++)
      tmaLoad3d(st + IMG_LEV_OFF + (j * NCOMP + k) * IMG_INT_F, &mp.lev[j][k], z0, x0, y, bar);
  if (prem)
#pragma unroll
    for (int k = 0; k < NMED; k++)
      tmaLoad3d(st + IMG_LEV_OFF + (NLEV * NCOMP + k) * IMG_INT_F, &mp.med[k], z0, x0, y, bar);
}

template <int NLEV, int STAGES, int ITX>
__global__ void __launch_bounds__(TZ * ITX, ITX == 4 ? 3 : 1) kImagingLev(const __grid_constant__ ImagingLevMaps<NLEV> mp,
                                                                          ImagingBlockPtrs q, GridConst g, int yChunk) {
  constexpr int SF = imgLevStageF(NLEV, ITX);
  constexpr int IMG_TX = ITX, IMG_HALO_F = imgHaloF(ITX), IMG_INT_F = imgIntF(ITX), IMG_LEV_OFF = imgLevOff(ITX);
  extern __shared__ __align__(1024) float smem[];
  __shared__ __align__(8) unsigned long long bars[STAGES];
  const int tz = threadIdx.x, tx = threadIdx.y;
  const int tid = tx * TZ + tz;
  const int z0 = FAT + blockIdx.x * TZ, x0 = FAT + blockIdx.y * IMG_TX;
  const int iz = z0 + tz, ix = x0 + tx;
  const bool active = (iz < g.nz - FAT) && (ix < g.nx - FAT);
  const int yBeg = FAT + blockIdx.z * yChunk;
  const int yEnd = min(yBeg + yChunk, g.ny - FAT);
  const long long ys = g.yStride;
  const long long col = (long long)ix * g.nz + iz;
  const int ntimes = q.leftImage ? 2 : 1;
  const int t0 = 2 - ntimes;
  const bool prem = q.prem != 0;

  if (tid == 0) {
    for (int s = 0; s < STAGES; s++) mbarInit(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (tid == 0)
    for (int s = 0; s < STAGES - 1; s++)
      if (yBeg + s < yEnd) imgLevIssuePlane<NLEV, ITX>(mp, smem + s * SF, &bars[s], yBeg + s, z0, x0, ntimes, prem);
  float w[2][3][8];
  if (active) {
#pragma unroll
    for (int t = 0; t < 2; t++)
#pragma unroll
      for (int f = 0; f < 3; f++)
#pragma unroll
        for (int k = 0; k < 7; k++)
          w[t][f][k] = (t >= t0) ? __ldg(q.v[t + 1][f] + (long long)(yBeg + imgBase(f) + k) * ys + col) : 0.f;
  }
  const int lc = (tx + HALO) * SZ + (tz + HALO);
  const int li = tx * TZ + tz;
  int slot = 0;
  unsigned parity = 0;
  for (int y = yBeg; y < yEnd; y++) {
    const long long ic = (long long)y * ys + col;
    float pv[NMED], nxt[3], prv[3], cur0[3], cin[NCOMP];
    if (active) {
#pragma unroll
      for (int k = 0; k < 3; k++) {
        nxt[k] = q.v[3][k] ? __ldg(q.v[3][k] + ic) : 0.f;                   // V(its+2)
        prv[k] = (q.leftImage && q.v[0][k]) ? __ldg(q.v[0][k] + ic) : 0.f;  // V(its-1)
        cur0[k] = q.leftImage ? 0.f : __ldg(q.v[1][k] + ic);                // V(its) without its tile
      }
#pragma unroll
      for (int k = 0; k < NCOMP; k++) cin[k] = q.carryIn ? q.carry[k][ic] : 0.f;
#pragma unroll
      for (int k = 0; k < NMED; k++) pv[k] = q.pert[k][ic];
    }
    const bool ok = mbarWaitBounded(&bars[slot], (parity >> slot) & 1u);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(&g_e3dPipeError, 1u);
        for (int s = 0; s < STAGES; s++) mbarWaitBounded(&bars[s], (parity >> s) & 1u);
      }
      __syncthreads();
      return;
    }
    parity ^= 1u << slot;
    if (tid == 0) {
      const int yn = y + STAGES - 1;
      int ns = slot + STAGES - 1;
      if (ns >= STAGES) ns -= STAGES;
      if (yn < yEnd) imgLevIssuePlane<NLEV, ITX>(mp, smem + ns * SF, &bars[ns], yn, z0, x0, ntimes, prem);
    }
    const float* st = smem + slot * SF;
    if (active) {
      // block sums from the staged levels, in blockSums' order
      float L[NCOMP], R[NCOMP];
#pragma unroll
      for (int k = 0; k < NCOMP; k++) {
        L[k] = 0.f;
        R[k] = 0.f;
      }
#pragma unroll
      for (int j = 0; j < NLEV; j++) {
        const float wl = q.wl[j], wr = q.wr[j];
#pragma unroll
        for (int k = 0; k < NCOMP; k++) {
          const float a = st[IMG_LEV_OFF + (j * NCOMP + k) * IMG_INT_F + li];
          L[k] = fmaf(a, wl, L[k]);
          R[k] = fmaf(a, wr, R[k]);
        }
      }
      if (prem) {
        float md[NMED];
#pragma unroll
        for (int k = 0; k < NMED; k++) md[k] = st[IMG_LEV_OFF + (NLEV * NCOMP + k) * IMG_INT_F + li];
        premSumsToRaw(md, L, R);
      }
      if (q.carryIn) {
#pragma unroll
        for (int k = 0; k < NCOMP; k++) R[k] += cin[k];
      }
#pragma unroll
      for (int t = 0; t < 2; t++)
#pragma unroll
        for (int f = 0; f < 3; f++)
          if (t >= t0) w[t][f][7] = st[6 * IMG_HALO_F + (t * 3 + f) * IMG_INT_F + li];
      const float* h1x = st + 3 * IMG_HALO_F;
      const float* h1y = st + 4 * IMG_HALO_F;
      const float* h1z = st + 5 * IMG_HALO_F;
      float prevR[3];
      if (q.leftImage) {
        prevR[0] = st[0 * IMG_HALO_F + lc];
        prevR[1] = st[1 * IMG_HALO_F + lc];
        prevR[2] = st[2 * IMG_HALO_F + lc];
      } else {
        prevR[0] = cur0[0];
        prevR[1] = cur0[1];
        prevR[2] = cur0[2];
      }
      float acc[NMED];
      {
        const VelTerms t1 = tileVelTerms(h1x, h1y, h1z, w[1][0], w[1][1], w[1][2], lc, g, prevR, nxt, q.dtsInv,
                                         q.q3compat);
        imagingTerms(t1, R, acc);
      }
      if (q.leftImage) {
        float nextL[3] = {h1x[lc], h1y[lc], h1z[lc]};
        const VelTerms tl = tileVelTerms(st, st + IMG_HALO_F, st + 2 * IMG_HALO_F, w[0][0], w[0][1], w[0][2], lc,
                                         g, prv, nextL, q.dtsInv, q.q3compat);
        float accL[NMED];
        imagingTerms(tl, L, accL);
#pragma unroll
        for (int k = 0; k < NMED; k++) acc[k] += accL[k];
      } else {
#pragma unroll
        for (int k = 0; k < NCOMP; k++) q.carry[k][ic] = L[k];
      }
#pragma unroll
      for (int k = 0; k < NMED; k++) q.pert[k][ic] = pv[k] + acc[k];
#pragma unroll
      for (int t = 0; t < 2; t++)
#pragma unroll
        for (int f = 0; f < 3; f++)
#pragma unroll
          for (int k = 0; k < 7; k++) w[t][f][k] = w[t][f][k + 1];
    }
    slot = (slot + 1 == STAGES) ? 0 : slot + 1;
  }
}

// ---------------------------------------------------------------------------
// Checkpoint compression: a field plane (one y slice) is stored as fp16 or
// bf16 with one fp32 scale per (field, y) slice (max-abs / 2^14 for fp16,
// max-abs for bf16), or copied raw in fp32.
// ---------------------------------------------------------------------------
// Slice maxima, packing and unpacking run on a (chunk, y slice, field) grid:
// nf fields of n values each, slice y of field f at f*n + y*ys.  With VEC the
// slices are read and written four values at a time (ys and n multiples of 4,
// 16-byte aligned fields).
constexpr int kSliceThreads = 256;
constexpr int kSliceVecPerThread = 4;

__device__ __forceinline__ unsigned sliceChunkBegin() { return blockIdx.x * kSliceThreads + threadIdx.x; }

// 16-bit storage types as raw bits, so that four values move as one 8-byte word
__device__ __forceinline__ unsigned halfBits(__half h) { return __half_as_ushort(h); }
__device__ __forceinline__ unsigned halfBits(__nv_bfloat16 h) { return __bfloat16_as_ushort(h); }
template <typename H>
__device__ __forceinline__ float halfValue(unsigned bits);
template <>
__device__ __forceinline__ float halfValue<__half>(unsigned bits) {
  return __half2float(__ushort_as_half((unsigned short)bits));
}
template <>
__device__ __forceinline__ float halfValue<__nv_bfloat16>(unsigned bits) {
  return __bfloat162float(__ushort_as_bfloat16((unsigned short)bits));
}

// out[f*ny + y] = max |a| over slice y of field f; out must be zeroed first.
// NaN values are ignored, as by fmaxf; the block maxima combine through an
// unsigned atomicMax, which orders non-negative floats by their bit patterns.
template <bool VEC>
__global__ void __launch_bounds__(kSliceThreads) kSliceMaxAbs(const float* a, long long n, long long ys, float* out) {
  const long long base = (long long)blockIdx.z * n + (long long)blockIdx.y * ys;
  const unsigned stride = gridDim.x * kSliceThreads;
  float m = 0.0f;
  if (VEC) {
    const float4* v = reinterpret_cast<const float4*>(a + base);
    const unsigned nv = (unsigned)(ys / 4);
    for (unsigned j = sliceChunkBegin(); j < nv; j += stride) {
      const float4 q = __ldg(v + j);
      m = fmaxf(fmaxf(m, fabsf(q.x)), fmaxf(fabsf(q.y), fmaxf(fabsf(q.z), fabsf(q.w))));
    }
  } else {
    for (long long j = sliceChunkBegin(); j < ys; j += stride) m = fmaxf(m, fabsf(__ldg(a + base + j)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ float red[kSliceThreads / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < kSliceThreads / 32 ? red[threadIdx.x] : 0.0f;
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0 && m > 0.0f)
      atomicMax(reinterpret_cast<unsigned*>(out) + (size_t)blockIdx.z * gridDim.y + blockIdx.y, __float_as_uint(m));
  }
}

// Per-slice scaling by a power of two 2^sh chosen so that the slice maximum m
// lands in [2^(topExp-1), 2^topExp): scaling and unscaling are exact, and sh is
// clamped to +-126 so that slices whose maximum is tiny or subnormal (far from
// the wavefront) keep finite scales.  A zero or non-finite maximum stores zeros.
// scales[f*ny + y] receives the unscaling factor.
template <typename H, bool VEC>
__global__ void __launch_bounds__(kSliceThreads) kPackSlices(const float* a, long long n, long long ys,
                                                             const float* smax, int topExp, H* out, float* scales) {
  const size_t slice = (size_t)blockIdx.z * gridDim.y + blockIdx.y;
  const long long base = (long long)blockIdx.z * n + (long long)blockIdx.y * ys;
  const float m = smax[slice];
  float s = 0.0f, inv = 0.0f;
  if (m > 0.0f && isfinite(m)) {
    int e;
    frexpf(m, &e);  // m in [2^(e-1), 2^e)
    const int sh = max(-126, min(126, topExp - e));
    s = ldexpf(1.0f, sh);
    inv = ldexpf(1.0f, -sh);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) scales[slice] = inv;
  const unsigned stride = gridDim.x * kSliceThreads;
  if (VEC) {
    const float4* v = reinterpret_cast<const float4*>(a + base);
    const unsigned nv = (unsigned)(ys / 4);
    for (unsigned j = sliceChunkBegin(); j < nv; j += stride) {
      const float4 q = __ldg(v + j);
      const uint2 w = make_uint2(halfBits(H(q.x * s)) | halfBits(H(q.y * s)) << 16,
                                 halfBits(H(q.z * s)) | halfBits(H(q.w * s)) << 16);
      *reinterpret_cast<uint2*>(out + base + 4 * (long long)j) = w;
    }
  } else {
    for (long long j = sliceChunkBegin(); j < ys; j += stride) out[base + j] = H(__ldg(a + base + j) * s);
  }
}

template <typename H, bool VEC>
__global__ void __launch_bounds__(kSliceThreads) kUnpackSlices(const H* in, long long n, long long ys,
                                                               const float* scales, float* a) {
  const size_t slice = (size_t)blockIdx.z * gridDim.y + blockIdx.y;
  const long long base = (long long)blockIdx.z * n + (long long)blockIdx.y * ys;
  const float sc = scales[slice];
  const unsigned stride = gridDim.x * kSliceThreads;
  if (VEC) {
    float4* v = reinterpret_cast<float4*>(a + base);
    const unsigned nv = (unsigned)(ys / 4);
    for (unsigned j = sliceChunkBegin(); j < nv; j += stride) {
      const uint2 w = __ldg(reinterpret_cast<const uint2*>(in + base + 4 * (long long)j));
      v[j] = make_float4(halfValue<H>(w.x & 0xffffu) * sc, halfValue<H>(w.x >> 16) * sc,
                         halfValue<H>(w.y & 0xffffu) * sc, halfValue<H>(w.y >> 16) * sc);
    }
  } else {
    for (long long j = sliceChunkBegin(); j < ys; j += stride) a[base + j] = float(in[base + j]) * sc;
  }
}

}  // namespace e3d
