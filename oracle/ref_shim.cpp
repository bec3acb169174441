// Test infrastructure only: extern "C" entry points over the reference's own
// CUDA drivers, which are compiled from the reference sources (not copied)
// into oracle/_ref/ by oracle/Makefile.  The reference drivers have C++
// linkage and process-global state; this shim declares the handful of driver
// functions the fixtures need, with the exact signatures of
//   elastic_iso_float/include/nonlinearPropElasticGpuFunctions_3D.h:9-18
//   elastic_iso_float/include/BornElasticGpuFunctions_3D.h:9-21
// (REF_REAL = float for elastic_iso_float, double for elastic_iso_double),
// and drives one single-GPU propagation per call.
//
// Compiled once per (tree, operator) pair with -DREF_REAL=<type> and
// -DREF_NL or -DREF_BORN, because both trees and both operators define the
// same global symbols.
#include <cstddef>

#ifndef REF_REAL
#error "REF_REAL must be defined"
#endif
typedef REF_REAL R;
typedef long long LL;

#ifdef REF_NL
void initNonlinearElasticGpu_3D(R dz, R dx, R dy, int nz, int nx, int ny, int nts, R dts, int sub, int minPad,
                                int blockSize, R alphaCos, int nGpu, int iGpuId, int iGpuAlloc);
void allocateNonlinearElasticGpu_3D(R* rhoxDtw, R* rhoyDtw, R* rhozDtw, R* lamb2MuDt, R* lambDtw, R* muxzDtw,
                                    R* muxyDtw, R* muyzDtw, int nx, int ny, int nz, int iGpu, int iGpuId);
void deallocateNonlinearElasticGpu_3D(int iGpu, int iGpuId);
void propElasticFwdGpu_3D(R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*,
                          LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL,
                          LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL,
                          int nx, int ny, int nz, int iGpu, int iGpuId);
void propElasticAdjGpu_3D(R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*,
                          LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL,
                          LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL,
                          int nx, int ny, int nz, int iGpu, int iGpuId);
#endif

#ifdef REF_BORN
void initBornElasticGpu_3D(R dz, R dx, R dy, int nz, int nx, int ny, int nts, R dts, int sub, int minPad,
                           int blockSize, R alphaCos, int nGpu, int iGpuId, int iGpuAlloc);
void allocateBornElasticGpu_3D(R* rhoxDtw, R* rhoyDtw, R* rhozDtw, R* lamb2MuDt, R* lambDtw, R* muxzDtw,
                               R* muxyDtw, R* muyzDtw, int nx, int ny, int nz, int iGpu, int iGpuId);
void deallocateBornElasticGpu_3D(int iGpu, int iGpuId);
void allocatePinBornElasticGpu_3D(int nx, int ny, int nz, int nts, int nGpu, int iGpuId, int iGpu, int iGpuAlloc);
void deallocatePinBornElasticGpu_3D(int iGpu, int iGpuId);
void BornElasticFwdGpu_3D(R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*,
                          LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL,
                          LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL,
                          R*, R*, R*, R*, R*, R*, R*, R*, int nx, int ny, int nz, int iGpu, int iGpuId);
void BornElasticAdjGpu_3D(R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*, R*,
                          LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL,
                          LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL, LL*, LL,
                          R*, R*, R*, R*, R*, R*, R*, R*, int nx, int ny, int nz, int iGpu, int iGpuId);
#endif

extern "C" {

// dims: nz, nx, ny, nts, sub (internal), minPad
// reals: dz, dx, dy, dts, alphaCos
// med: 8 medium planes; sig: 9 source (or model) signal arrays; dat: 9 data arrays
// spos/sn, rpos/rn: 7 grids (center, x, y, z, xz, xy, yz)
// pert: 8 perturbation planes (Born only)
#ifdef REF_NL
int ref_nl_run(int adjoint, const int* dims, const double* reals, R** med, R** sig, R** dat, LL** spos,
               const LL* sn, LL** rpos, const LL* rn) {
  const int nz = dims[0], nx = dims[1], ny = dims[2];
  initNonlinearElasticGpu_3D((R)reals[0], (R)reals[1], (R)reals[2], nz, nx, ny, dims[3], (R)reals[3], dims[4],
                             dims[5], 16, (R)reals[4], 1, 0, 0);
  allocateNonlinearElasticGpu_3D(med[0], med[1], med[2], med[3], med[4], med[5], med[6], med[7], nx, ny, nz, 0, 0);
  if (!adjoint) {
    propElasticFwdGpu_3D(sig[0], sig[1], sig[2], sig[3], sig[4], sig[5], sig[6], sig[7], sig[8], dat[0], dat[1],
                         dat[2], dat[3], dat[4], dat[5], dat[6], dat[7], dat[8], spos[0], sn[0], spos[1], sn[1],
                         spos[2], sn[2], spos[3], sn[3], spos[4], sn[4], spos[5], sn[5], spos[6], sn[6], rpos[0],
                         rn[0], rpos[1], rn[1], rpos[2], rn[2], rpos[3], rn[3], rpos[4], rn[4], rpos[5], rn[5],
                         rpos[6], rn[6], nx, ny, nz, 0, 0);
  } else {
    propElasticAdjGpu_3D(sig[0], sig[1], sig[2], sig[3], sig[4], sig[5], sig[6], sig[7], sig[8], dat[0], dat[1],
                         dat[2], dat[3], dat[4], dat[5], dat[6], dat[7], dat[8], spos[0], sn[0], spos[1], sn[1],
                         spos[2], sn[2], spos[3], sn[3], spos[4], sn[4], spos[5], sn[5], spos[6], sn[6], rpos[0],
                         rn[0], rpos[1], rn[1], rpos[2], rn[2], rpos[3], rn[3], rpos[4], rn[4], rpos[5], rn[5],
                         rpos[6], rn[6], nx, ny, nz, 0, 0);
  }
  deallocateNonlinearElasticGpu_3D(0, 0);
  return 0;
}
#endif

#ifdef REF_BORN
int ref_born_run(int adjoint, const int* dims, const double* reals, R** med, R** sig, R** dat, LL** spos,
                 const LL* sn, LL** rpos, const LL* rn, R** pert) {
  const int nz = dims[0], nx = dims[1], ny = dims[2];
  initBornElasticGpu_3D((R)reals[0], (R)reals[1], (R)reals[2], nz, nx, ny, dims[3], (R)reals[3], dims[4], dims[5],
                        16, (R)reals[4], 1, 0, 0);
  allocateBornElasticGpu_3D(med[0], med[1], med[2], med[3], med[4], med[5], med[6], med[7], nx, ny, nz, 0, 0);
  allocatePinBornElasticGpu_3D(nx, ny, nz, dims[3], 1, 0, 0, 0);
  if (!adjoint) {
    BornElasticFwdGpu_3D(sig[0], sig[1], sig[2], sig[3], sig[4], sig[5], sig[6], sig[7], sig[8], dat[0], dat[1],
                         dat[2], dat[3], dat[4], dat[5], dat[6], dat[7], dat[8], spos[0], sn[0], spos[1], sn[1],
                         spos[2], sn[2], spos[3], sn[3], spos[4], sn[4], spos[5], sn[5], spos[6], sn[6], rpos[0],
                         rn[0], rpos[1], rn[1], rpos[2], rn[2], rpos[3], rn[3], rpos[4], rn[4], rpos[5], rn[5],
                         rpos[6], rn[6], pert[0], pert[1], pert[2], pert[3], pert[4], pert[5], pert[6], pert[7], nx,
                         ny, nz, 0, 0);
  } else {
    BornElasticAdjGpu_3D(sig[0], sig[1], sig[2], sig[3], sig[4], sig[5], sig[6], sig[7], sig[8], dat[0], dat[1],
                         dat[2], dat[3], dat[4], dat[5], dat[6], dat[7], dat[8], spos[0], sn[0], spos[1], sn[1],
                         spos[2], sn[2], spos[3], sn[3], spos[4], sn[4], spos[5], sn[5], spos[6], sn[6], rpos[0],
                         rn[0], rpos[1], rn[1], rpos[2], rn[2], rpos[3], rn[3], rpos[4], rn[4], rpos[5], rn[5],
                         rpos[6], rn[6], pert[0], pert[1], pert[2], pert[3], pert[4], pert[5], pert[6], pert[7], nx,
                         ny, nz, 0, 0);
  }
  deallocatePinBornElasticGpu_3D(0, 0);
  deallocateBornElasticGpu_3D(0, 0);
  return 0;
}
#endif

}  // extern "C"
