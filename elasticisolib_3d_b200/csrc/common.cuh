// Shared definitions of the B200 elastic 3D propagation engine.
//
// Grid layout is the reference's: a field of nz*nx*ny floats, z fastest,
// index = iy*nz*nx + ix*nz + iz (elastic_iso_float/src/kernelsElaGpu_3D.cu:144),
// with a FAT=4 ring that is read as stencil halo but never updated.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace e3d {

constexpr int FAT = 4;
constexpr int NCOMP = 9;   // vx, vy, vz, sxx, syy, szz, sxz, sxy, syz
constexpr int NMED = 8;    // rhoxDtw, rhoyDtw, rhozDtw, lamb2MuDtw, lambDtw, muxzDtw, muxyDtw, muyzDtw
constexpr int NGRID = 7;   // center, x, y, z, xz, xy, yz
constexpr int SUB_MAX = 100;  // varElaDeclare_3D.h:14 (internal sub must be below it)
constexpr int PAD_MAX = 400;  // varElaDeclare_3D.h:13

enum Comp { VX = 0, VY, VZ, SXX, SYY, SZZ, SXZ, SXY, SYZ };
enum Med { RHOX = 0, RHOY, RHOZ, L2M, LAM, MUXZ, MUXY, MUYZ };
enum Grid { GC = 0, GX, GY, GZ, GXZ, GXY, GYZ };

// Stepper modes (kernelsElaGpu_3D.cu:110, :471, :825)
enum StepMode { STEP_FWD = 0, STEP_ADJ_REVERSED = 1, STEP_ADJ_EXACT = 2 };

// Status codes returned through the C ABI (same values as include/elastic3d_b200.h).
#ifndef E3D_OK
#define E3D_OK 0
#define E3D_ERR_ARG 1      /* invalid argument (sizes, null pointers, limits) */
#define E3D_ERR_CUDA 2     /* a CUDA runtime call failed */
#define E3D_ERR_STATE 3    /* call out of order (e.g. propagate before allocate) */
#define E3D_ERR_OOM 4      /* device memory could not be obtained */
#define E3D_ERR_BOUNDS 5   /* acquisition device outside the propagation grid */
#endif

__host__ __device__ inline int gridOfComp(int comp) {
  return comp == VX ? GX : comp == VY ? GY : comp == VZ ? GZ : comp <= SZZ ? GC : comp == SXZ ? GXZ
         : comp == SXY ? GXY : GYZ;
}

// Geometry and constants of one propagation grid; passed by value to kernels.
struct GridConst {
  int nz, nx, ny;
  int minPad;
  long long yStride;  // nz*nx
  long long n;        // nz*nx*ny
  float cz[4], cx[4], cy[4];
  const float* taper;  // device, minPad entries
  int freeSurface;     // 1: free surface at z = FAT, whose face is not tapered (0: the reference's sponge)
  // y-slab of a decomposed grid: local plane y is global plane y + yOff of a grid of nyTaper
  // planes, whose y faces carry the sponge (a whole grid: yOff = 0, nyTaper = ny)
  int yOff, nyTaper;
};

#ifdef __CUDACC__
// Distance to the closest non-FAT edge and the cosine taper there
// (dampCosineEdge_3D, kernelsElaGpu_3D.cu:1182-1226): one minPad for all six
// faces, the top face excluded when the free surface is on.
__device__ __forceinline__ int topDistance(const GridConst& g, int iz) {
  return g.freeSurface ? (1 << 30) : iz - FAT;
}
// Distance of local plane y to the closest tapered y face of the (possibly decomposed) grid.
__device__ __forceinline__ int yDistance(const GridConst& g, int y) {
  const int yg = y + g.yOff;
  return min(yg - FAT, g.nyTaper - yg - 1 - FAT);
}
__device__ __forceinline__ float taperAt(const GridConst& g, int iz, int ix, int iy) {
  int d = min(min(topDistance(g, iz), ix - FAT), min(g.nz - iz - 1 - FAT, g.nx - ix - 1 - FAT));
  d = min(d, yDistance(g, iy));
  return d < g.minPad ? __ldg(g.taper + d) : 1.0f;
}
#endif

}  // namespace e3d

#define E3D_CUDA_TRY(expr)                                   \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) {                                 \
      e3d::setLastError(cudaGetErrorString(_e), __FILE__, __LINE__); \
      return _e == cudaErrorMemoryAllocation ? E3D_ERR_OOM : E3D_ERR_CUDA; \
    }                                                        \
  } while (0)

namespace e3d {
void setLastError(const char* msg, const char* file, int line);
}
