// Oracle (test infrastructure only): a plain CPU restatement of the elastic
// 3D staggered-grid propagation path of elasticIsoLib_3D.  It exists to check
// the CUDA product and to serve as the timed CPU baseline; nothing in the
// product links or calls it.
//
// Every routine is templated on the arithmetic type so the same source gives
// the FP32 restatement (elastic_iso_float) and the FP64 restatement
// (elastic_iso_double, which is the FP32 tree with double substituted).
//
// Layout: every wavefield / medium array is nz*nx*ny with z fastest,
// index = iy*nz*nx + ix*nz + iz (elastic_iso_float/src/kernelsElaGpu_3D.cu:144).
// Only cells in [FAT, n-FAT) along each axis are ever updated.
//
// Citations are to files inside elastic_iso_lib_3d/elastic_iso_float/.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

constexpr int FAT = 4;

// Component order used everywhere (nonlinearPropElasticShotsGpu_3D.cpp:132-134):
// vx, vy, vz, sxx, syy, szz, sxz, sxy, syz
enum { VX = 0, VY, VZ, SXX, SYY, SZZ, SXZ, SXY, SYZ, NCOMP };
// Medium planes: rhoxDtw, rhoyDtw, rhozDtw, lamb2MuDtw, lambDtw, muxzDtw, muxyDtw, muyzDtw
enum { RHOX = 0, RHOY, RHOZ, L2M, LAM, MUXZ, MUXY, MUYZ, NMED };
// Source / receiver grids: center, x, y, z, xz, xy, yz
enum { GC = 0, GX, GY, GZ, GXZ, GXY, GYZ, NGRID };

template <typename T>
struct Ctx {
  int nz, nx, ny, nts, sub, ntw, minPad, hfilt;
  long long yStride, n;
  T cz[4], cx[4], cy[4];
  std::vector<T> filt;  // 2*(sub+1) time-interpolation weights
  std::vector<T> damp;  // minPad cosine taper
  T dtsInv;             // 1/(2 dts), Born time derivative
  int freeSurface = 0;  // 1: stress-free surface at z = FAT, top face not tapered
};

// Constants of initNonlinearElasticGpu_3D (nonlinearPropElasticGpuFunctions_3D.cu:203-255)
// and initBornElasticGpu_3D (BornElasticGpuFunctions_3D.cu:255-337).  The
// rounding follows the reference: FD coefficients are double quotients stored
// in T; filter weights are built in T; y coefficients use dx (quirk Q1) unless
// fix_q1 is set.
template <typename T>
void makeCtx(Ctx<T>& c, int nz, int nx, int ny, int nts, double dts, int sub, int minPad,
             double dz, double dx, double dy, double alphaCos, int fix_q1) {
  c.nz = nz; c.nx = nx; c.ny = ny; c.nts = nts; c.sub = sub; c.minPad = minPad;
  c.ntw = (nts - 1) * sub + 1;
  c.yStride = (long long)nz * nx;
  c.n = c.yStride * ny;
  const double k[4] = {1.196289062541883, -0.079752604188901, 0.009570312506634, -6.975446437140719e-04};
  const T dzT = (T)dz, dxT = (T)dx, dyT = (T)dy;
  for (int i = 0; i < 4; i++) {
    c.cz[i] = (T)(k[i] / dzT);
    c.cx[i] = (T)(k[i] / dxT);
    c.cy[i] = (T)(k[i] / (fix_q1 ? dyT : dxT));
  }
  c.hfilt = sub + 1;
  c.filt.assign(2 * c.hfilt, T(0));
  // 1/sqrt(ntw/nts) in the arithmetic type of the tree
  const T ratio = (T)c.ntw / (T)nts;
  const double scale = 1.0 / (double)std::sqrt(ratio);
  for (int i = 0; i < c.hfilt; i++) {
    T left = (T)(1.0 - 1.0 * i / sub);
    T right = (T)(1.0 - left);
    c.filt[i] = (T)(left * scale);
    c.filt[i + c.hfilt] = (T)(right * scale);
  }
  c.damp.assign(minPad > 0 ? minPad : 1, T(1));
  const T alpha = (T)alphaCos;
  for (int i = 0; i < minPad; i++) {
    T arg = (T)(M_PI / (1.0 * minPad) * 1.0 * (minPad - i));
    T cs = (T)std::cos(arg);
    c.damp[i] = (T)(alpha + (1.0 - alpha) * cs);
  }
  const T dtsT = (T)dts;
  c.dtsInv = (T)(1.0 / (2.0 * dtsT));
}

// 8th-order staggered first derivatives.  "plus" is the forward-shifted
// operator c0(a[i+1]-a[i]) + ..., "minus" the backward-shifted one
// c0(a[i]-a[i-1]) + ...  (kernelsElaGpu_3D.cu:294-312, 320-348).
template <typename T>
inline T dPlus(const T* a, long long i, long long s, const T* c) {
  return c[0] * (a[i + s] - a[i]) + c[1] * (a[i + 2 * s] - a[i - s]) +
         c[2] * (a[i + 3 * s] - a[i - 2 * s]) + c[3] * (a[i + 4 * s] - a[i - 3 * s]);
}
template <typename T>
inline T dMinus(const T* a, long long i, long long s, const T* c) {
  return c[0] * (a[i] - a[i - s]) + c[1] * (a[i + s] - a[i - 2 * s]) +
         c[2] * (a[i + 2 * s] - a[i - 3 * s]) + c[3] * (a[i + 3 * s] - a[i - 4 * s]);
}

// Modes of the stepper:
//  0: forward leapfrog  p0 = p0 + M D(p1)            (stepFwdGpu_3D, kernelsElaGpu_3D.cu:110-460)
//  1: time-reversed     p0 = p0 - M D(p1)            (stepAdjGpu_3D, kernelsElaGpu_3D.cu:471-822)
//  2: exact transpose   p0 = p0 - D(M p1)            (stepAdjGpuBorn_3D, kernelsElaGpu_3D.cu:825-1177)
template <typename T>
void step(const Ctx<T>& C, T* const* p0, T* const* p1, const T* const* m, int mode) {
  const int nz = C.nz, nx = C.nx, ny = C.ny;
  const long long ys = C.yStride, xs = nz;
  const T* cz = C.cz; const T* cx = C.cx; const T* cy = C.cy;
  // Mode 2 differentiates medium-premultiplied fields; build them once.
  std::vector<T> pre;
  const T* c[NCOMP];
  if (mode == 2) {
    pre.resize((size_t)NCOMP * C.n);
    T* q[NCOMP];
    for (int k = 0; k < NCOMP; k++) q[k] = pre.data() + (size_t)k * C.n;
#pragma omp parallel for
    for (long long i = 0; i < C.n; i++) {
      const T sxx = p1[SXX][i], syy = p1[SYY][i], szz = p1[SZZ][i];
      q[VX][i] = p1[VX][i] * m[RHOX][i];
      q[VY][i] = p1[VY][i] * m[RHOY][i];
      q[VZ][i] = p1[VZ][i] * m[RHOZ][i];
      q[SXX][i] = sxx * m[L2M][i] + (syy + szz) * m[LAM][i];
      q[SYY][i] = syy * m[L2M][i] + (sxx + szz) * m[LAM][i];
      q[SZZ][i] = szz * m[L2M][i] + (sxx + syy) * m[LAM][i];
      q[SXZ][i] = p1[SXZ][i] * m[MUXZ][i];
      q[SXY][i] = p1[SXY][i] * m[MUXY][i];
      q[SYZ][i] = p1[SYZ][i] * m[MUYZ][i];
    }
    for (int k = 0; k < NCOMP; k++) c[k] = q[k];
  } else {
    for (int k = 0; k < NCOMP; k++) c[k] = p1[k];
  }
  const T sgn = (mode == 0) ? T(1) : T(-1);
#pragma omp parallel for collapse(2)
  for (int iy = FAT; iy < ny - FAT; iy++) {
    for (int ix = FAT; ix < nx - FAT; ix++) {
      for (int iz = FAT; iz < nz - FAT; iz++) {
        const long long i = (long long)iy * ys + (long long)ix * xs + iz;
        const T dvx_dx = dPlus(c[VX], i, xs, cx);
        const T dvy_dy = dPlus(c[VY], i, ys, cy);
        const T dvz_dz = dPlus(c[VZ], i, 1, cz);
        const T fvx = dMinus(c[SXX], i, xs, cx) + dPlus(c[SXY], i, ys, cy) + dPlus(c[SXZ], i, 1, cz);
        const T fvy = dPlus(c[SXY], i, xs, cx) + dMinus(c[SYY], i, ys, cy) + dPlus(c[SYZ], i, 1, cz);
        const T fvz = dPlus(c[SXZ], i, xs, cx) + dPlus(c[SYZ], i, ys, cy) + dMinus(c[SZZ], i, 1, cz);
        const T fxy = dMinus(c[VX], i, ys, cy) + dMinus(c[VY], i, xs, cx);
        const T fxz = dMinus(c[VX], i, 1, cz) + dMinus(c[VZ], i, xs, cx);
        const T fyz = dMinus(c[VZ], i, ys, cy) + dMinus(c[VY], i, 1, cz);
        if (mode == 2) {
          p0[VX][i] -= fvx;
          p0[VY][i] -= fvy;
          p0[VZ][i] -= fvz;
          p0[SXX][i] -= dvx_dx;
          p0[SYY][i] -= dvy_dy;
          p0[SZZ][i] -= dvz_dz;
          p0[SXY][i] -= fxy;
          p0[SXZ][i] -= fxz;
          p0[SYZ][i] -= fyz;
        } else {
          p0[VX][i] += sgn * (m[RHOX][i] * fvx);
          p0[VY][i] += sgn * (m[RHOY][i] * fvy);
          p0[VZ][i] += sgn * (m[RHOZ][i] * fvz);
          p0[SXX][i] += sgn * (m[L2M][i] * dvx_dx + m[LAM][i] * (dvy_dy + dvz_dz));
          p0[SYY][i] += sgn * (m[L2M][i] * dvy_dy + m[LAM][i] * (dvx_dx + dvz_dz));
          p0[SZZ][i] += sgn * (m[L2M][i] * dvz_dz + m[LAM][i] * (dvx_dx + dvy_dy));
          p0[SXY][i] += sgn * (m[MUXY][i] * fxy);
          p0[SXZ][i] += sgn * (m[MUXZ][i] * fxz);
          p0[SYZ][i] += sgn * (m[MUYZ][i] * fyz);
        }
      }
    }
  }
}

// Cosine sponge applied to both time levels (dampCosineEdge_3D,
// kernelsElaGpu_3D.cu:1182-1226).  One minPad for every face (quirk Q5).
template <typename T>
void dampBoth(const Ctx<T>& C, T* const* p0, T* const* p1) {
  const int nz = C.nz, nx = C.nx, ny = C.ny;
#pragma omp parallel for collapse(2)
  for (int iy = FAT; iy < ny - FAT; iy++) {
    for (int ix = FAT; ix < nx - FAT; ix++) {
      for (int iz = FAT; iz < nz - FAT; iz++) {
        int d = C.freeSurface ? (1 << 30) : iz - FAT;
        d = std::min(d, ix - FAT);
        d = std::min(d, nz - iz - 1 - FAT);
        d = std::min(d, nx - ix - 1 - FAT);
        d = std::min(d, iy - FAT);
        d = std::min(d, ny - iy - 1 - FAT);
        if (d < C.minPad) {
          const long long i = (long long)iy * C.yStride + (long long)ix * nz + iz;
          const T g = C.damp[d];
          for (int k = 0; k < NCOMP; k++) { p0[k][i] *= g; p1[k][i] *= g; }
        }
      }
    }
  }
}

// Free surface at the first interior row zs = FAT (new physics; the reference
// parses freeSurface but applies it nowhere, fdParamElastic_3D.cpp:19, 44-45).
// Stress imaging: szz = 0 at zs and odd about it; sxz, syz (row r at depth
// r-1/2) odd about zs; vz rows 0..zs held at zero; and sxx, syy at zs with the
// step's lambda*d(vz)/dz replaced through d(vz)/dz = -lambda/(lambda+2mu)
// (d(vx)/dx + d(vy)/dy).  The correction uses the current level as the step
// did, so it is formed before the sponge damps that level, and is applied,
// scaled by the taper, after damping, together with the imaging.
template <typename T>
void freeSurfaceDelta(const Ctx<T>& C, const T* const* p1, const T* const* m, T sgn, std::vector<T>& delta) {
  const long long ys = C.yStride, xs = C.nz;
  delta.assign((size_t)C.nx * C.ny, T(0));
#pragma omp parallel for collapse(2)
  for (int iy = FAT; iy < C.ny - FAT; iy++)
    for (int ix = FAT; ix < C.nx - FAT; ix++) {
      const long long i = (long long)iy * ys + (long long)ix * xs + FAT;
      const T dvx = dPlus(p1[VX], i, xs, C.cx);
      const T dvy = dPlus(p1[VY], i, ys, C.cy);
      const T dvz = dPlus(p1[VZ], i, 1, C.cz);
      const T lam = m[LAM][i], l2m = m[L2M][i];
      delta[(size_t)iy * C.nx + ix] = sgn * (-lam * dvz - (lam * lam / l2m) * (dvx + dvy));
    }
}

template <typename T>
void freeSurfaceApply(const Ctx<T>& C, T* const* p0, const std::vector<T>& delta) {
  const long long ys = C.yStride, xs = C.nz;
#pragma omp parallel for collapse(2)
  for (int iy = FAT; iy < C.ny - FAT; iy++)
    for (int ix = FAT; ix < C.nx - FAT; ix++) {
      const long long col = (long long)iy * ys + (long long)ix * xs;
      const long long i = col + FAT;
      int d = std::min(ix - FAT, C.nx - ix - 1 - FAT);
      d = std::min(d, C.nz - FAT - 1 - FAT);
      d = std::min(d, std::min(iy - FAT, C.ny - iy - 1 - FAT));
      const T g = d < C.minPad ? C.damp[d] : T(1);
      const T corr = g * delta[(size_t)iy * C.nx + ix];
      p0[SXX][i] += corr;
      p0[SYY][i] += corr;
      p0[SZZ][i] = T(0);
      for (int k = 1; k <= FAT; k++) p0[SZZ][i - k] = -p0[SZZ][i + k];
      for (int r = 0; r <= FAT; r++) {
        p0[SXZ][col + r] = -p0[SXZ][col + 2 * FAT + 1 - r];
        p0[SYZ][col + r] = -p0[SYZ][col + 2 * FAT + 1 - r];
        p0[VZ][col + r] = T(0);
      }
    }
}

struct Geom {
  const long long* pos[NGRID];
  long long n[NGRID];
};

// Which grid each component lives on (center grid carries the three normal
// stresses, nonlinearPropElasticGpuFunctions_3D.cu:684-700).
inline int gridOf(int comp) {
  switch (comp) {
    case VX: return GX;
    case VY: return GY;
    case VZ: return GZ;
    case SXX: case SYY: case SZZ: return GC;
    case SXZ: return GXZ;
    case SXY: return GXY;
    default: return GYZ;
  }
}

// Signal injection: slice[pos] += s[its]*f[k] + s[its+1]*f[h+k]
// (ker_inject_source_*Grid_3D, ker_inject_data_*Grid_3D, kernelsElaGpu_3D.cu:11-52).
template <typename T>
void injectSignals(const Ctx<T>& C, T* const* p, const T* const* sig, const Geom& g, int its, int k,
                   const long long* const* posOverride = nullptr) {
  for (int comp = 0; comp < NCOMP; comp++) {
    const int gi = gridOf(comp);
    const long long* pos = posOverride ? posOverride[comp] : g.pos[gi];
    const long long nd = g.n[gi];
    const T* s = sig[comp];
    for (long long d = 0; d < nd; d++) {
      p[comp][pos[d]] += s[C.nts * d + its] * C.filt[k] + s[C.nts * d + its + 1] * C.filt[C.hfilt + k];
    }
  }
}

// Signal recording: out[its] += slice[pos]*f[k], out[its+1] += slice[pos]*f[h+k]
// (ker_record_*, kernelsElaGpu_3D.cu:61-104).
template <typename T>
void recordSignals(const Ctx<T>& C, T* const* p, T* const* out, const Geom& g, int its, int k,
                   const long long* const* posOverride = nullptr) {
  for (int comp = 0; comp < NCOMP; comp++) {
    const int gi = gridOf(comp);
    const long long* pos = posOverride ? posOverride[comp] : g.pos[gi];
    const long long nd = g.n[gi];
    T* o = out[comp];
    for (long long d = 0; d < nd; d++) {
      const T v = p[comp][pos[d]];
      o[C.nts * d + its] += v * C.filt[k];
      o[C.nts * d + its + 1] += v * C.filt[C.hfilt + k];
    }
  }
}

// Receiver position table used for recording/injecting data.  The reference
// copies the XZ receiver positions from the Z-grid list (quirk Q2,
// nonlinearPropElasticGpuFunctions_3D.cu:416); compat mode reproduces that.
inline void receiverTable(const Geom& rec, int q2compat, const long long* out[NCOMP]) {
  for (int comp = 0; comp < NCOMP; comp++) out[comp] = rec.pos[gridOf(comp)];
  if (q2compat) out[SXZ] = rec.pos[GZ];
}

template <typename T>
struct Fields {
  std::vector<T> buf;
  T* p[NCOMP];
  void alloc(long long n) {
    buf.assign((size_t)NCOMP * n, T(0));
    for (int k = 0; k < NCOMP; k++) p[k] = buf.data() + (size_t)k * n;
  }
  void zero() { std::fill(buf.begin(), buf.end(), T(0)); }
};

template <typename T>
void swapFields(Fields<T>& a, Fields<T>& b) {
  for (int k = 0; k < NCOMP; k++) std::swap(a.p[k], b.p[k]);
}

// Nonlinear forward propagation (propElasticFwdGpu_3D,
// nonlinearPropElasticGpuFunctions_3D.cu:876-975): per fine step
// step -> inject source (k=it2-1) -> damp -> record (k=it2) -> swap.
template <typename T>
void nlFwd(const Ctx<T>& C, const T* const* med, const T* const* model, T* const* data,
           const Geom& src, const Geom& rec, int q2compat) {
  Fields<T> p0, p1;
  p0.alloc(C.n); p1.alloc(C.n);
  for (int comp = 0; comp < NCOMP; comp++)
    std::fill(data[comp], data[comp] + (size_t)rec.n[gridOf(comp)] * C.nts, T(0));
  const long long* rpos[NCOMP];
  receiverTable(rec, q2compat, rpos);
  std::vector<T> fs;
  for (int its = 0; its < C.nts - 1; its++) {
    for (int it2 = 1; it2 < C.sub + 1; it2++) {
      step(C, p0.p, p1.p, med, 0);
      injectSignals(C, p0.p, model, src, its, it2 - 1);
      if (C.freeSurface) freeSurfaceDelta(C, p1.p, med, T(1), fs);
      dampBoth(C, p0.p, p1.p);
      if (C.freeSurface) freeSurfaceApply(C, p0.p, fs);
      recordSignals(C, p0.p, data, rec, its, it2, rpos);
      swapFields(p0, p1);
    }
  }
}

// Nonlinear "adjoint" (propElasticAdjGpu_3D, nonlinearPropElasticGpuFunctions_3D.cu:1298-1395):
// time-reversed forward stepper (quirk Q7); per fine step
// step -> inject data (k=it2+1) -> damp -> extract source (k=it2) -> swap.
template <typename T>
void nlAdj(const Ctx<T>& C, const T* const* med, T* const* model, const T* const* data,
           const Geom& src, const Geom& rec, int q2compat) {
  Fields<T> p0, p1;
  p0.alloc(C.n); p1.alloc(C.n);
  for (int comp = 0; comp < NCOMP; comp++)
    std::fill(model[comp], model[comp] + (size_t)src.n[gridOf(comp)] * C.nts, T(0));
  const long long* rpos[NCOMP];
  receiverTable(rec, q2compat, rpos);
  std::vector<T> fs;
  for (int its = C.nts - 2; its > -1; its--) {
    for (int it2 = C.sub - 1; it2 > -1; it2--) {
      step(C, p0.p, p1.p, med, 1);
      injectSignals(C, p0.p, data, rec, its, it2 + 1, rpos);
      if (C.freeSurface) freeSurfaceDelta(C, p1.p, med, T(-1), fs);
      dampBoth(C, p0.p, p1.p);
      if (C.freeSurface) freeSurfaceApply(C, p0.p, fs);
      recordSignals(C, p0.p, model, src, its, it2);
      swapFields(p0, p1);
    }
  }
}

// Source-side velocity wavefield of the Born operator, decimated to the
// coarse grid by the adjoint of linear time interpolation
// (BornElasticGpuFunctions_3D.cu:1268-1316, interpWavefieldVxVyVz_3D
// kernelsElaGpu_3D.cu:1646-1672).  Returns V[t][comp][cell] for t in [0,nts).
template <typename T>
void bornSourceWavefield(const Ctx<T>& C, const T* const* med, const T* const* srcSig,
                         const Geom& src, std::vector<T>& V) {
  Fields<T> p0, p1;
  p0.alloc(C.n); p1.alloc(C.n);
  V.assign((size_t)C.nts * 3 * C.n, T(0));
  for (int its = 0; its < C.nts - 1; its++) {
    T* left = V.data() + (size_t)its * 3 * C.n;
    T* right = V.data() + (size_t)(its + 1) * 3 * C.n;
    for (int it2 = 1; it2 < C.sub + 1; it2++) {
      step(C, p0.p, p1.p, med, 0);
      injectSignals(C, p0.p, srcSig, src, its, it2 - 1);
      dampBoth(C, p0.p, p1.p);
      const T fl = C.filt[it2], fr = C.filt[C.hfilt + it2];
#pragma omp parallel for collapse(2)
      for (int iy = FAT; iy < C.ny - FAT; iy++)
        for (int ix = FAT; ix < C.nx - FAT; ix++)
          for (int iz = FAT; iz < C.nz - FAT; iz++) {
            const long long i = (long long)iy * C.yStride + (long long)ix * C.nz + iz;
            for (int k = 0; k < 3; k++) {
              left[(size_t)k * C.n + i] += p0.p[k][i] * fl;
              right[(size_t)k * C.n + i] += p0.p[k][i] * fr;
            }
          }
      swapFields(p0, p1);
    }
  }
}

// Born scattering / imaging terms at coarse time t (imagingElaFwdGpu_3D
// kernelsElaGpu_3D.cu:1232-1438 and imagingElaAdjGpu_3D :1440-1641).
// The time derivative is (V[t-1]-V[t+1])/(2 dts) with V outside [0,nts) taken
// as zero.  With q3compat the yz shear term uses the xz derivative pair
// (quirk Q3) exactly as the reference does.
template <typename T>
struct ImagingTerms {
  T dvx_dx, dvy_dy, dvz_dz, exz, exy, eyz, tx, ty, tz;
};

template <typename T>
inline ImagingTerms<T> imagingTerms(const Ctx<T>& C, const std::vector<T>& V, int t, long long i,
                                    int q3compat) {
  const long long n = C.n;
  const T* cur = V.data() + (size_t)t * 3 * n;
  const T* vx = cur; const T* vy = cur + n; const T* vz = cur + 2 * n;
  const long long ys = C.yStride, xs = C.nz;
  ImagingTerms<T> r;
  r.dvx_dx = dPlus(vx, i, xs, C.cx);
  r.dvy_dy = dPlus(vy, i, ys, C.cy);
  r.dvz_dz = dPlus(vz, i, 1, C.cz);
  r.exz = dMinus(vx, i, 1, C.cz) + dMinus(vz, i, xs, C.cx);
  r.exy = dMinus(vx, i, ys, C.cy) + dMinus(vy, i, xs, C.cx);
  r.eyz = q3compat ? r.exz : (dMinus(vz, i, ys, C.cy) + dMinus(vy, i, 1, C.cz));
  T d[3];
  for (int k = 0; k < 3; k++) {
    if (t == 0) {
      d[k] = (-V[(size_t)(t + 1) * 3 * n + (size_t)k * n + i]) * C.dtsInv;
    } else if (t == C.nts - 1) {
      d[k] = (V[(size_t)(t - 1) * 3 * n + (size_t)k * n + i]) * C.dtsInv;
    } else {
      d[k] = (V[(size_t)(t - 1) * 3 * n + (size_t)k * n + i] - V[(size_t)(t + 1) * 3 * n + (size_t)k * n + i]) * C.dtsInv;
    }
  }
  r.tx = d[0]; r.ty = d[1]; r.tz = d[2];
  return r;
}

// Born forward (BornElasticFwdGpu_3D, BornElasticGpuFunctions_3D.cu:1226-1461).
// pert holds the 8 staggered, scaled perturbation planes
// drhox, drhoy, drhoz, dlame, dmu, dmuxz, dmuxy, dmuyz.
template <typename T>
void bornFwd(const Ctx<T>& C, const T* const* med, const T* const* srcSig, T* const* data,
             const Geom& src, const Geom& rec, const T* const* pert, int q2compat, int q3compat) {
  std::vector<T> V;
  bornSourceWavefield(C, med, srcSig, src, V);
  const long long n = C.n;
  // Secondary sources S[t][comp][cell]
  std::vector<T> S((size_t)C.nts * NCOMP * n, T(0));
  for (int t = 0; t < C.nts; t++) {
    T* s = S.data() + (size_t)t * NCOMP * n;
#pragma omp parallel for collapse(2)
    for (int iy = FAT; iy < C.ny - FAT; iy++)
      for (int ix = FAT; ix < C.nx - FAT; ix++)
        for (int iz = FAT; iz < C.nz - FAT; iz++) {
          const long long i = (long long)iy * C.yStride + (long long)ix * C.nz + iz;
          const ImagingTerms<T> r = imagingTerms(C, V, t, i, q3compat);
          s[VX * n + i] = pert[0][i] * r.tx;
          s[VY * n + i] = pert[1][i] * r.ty;
          s[VZ * n + i] = pert[2][i] * r.tz;
          const T div = r.dvx_dx + r.dvy_dy + r.dvz_dz;
          s[SXX * n + i] = (T)(pert[3][i] * div + 2.0 * pert[4][i] * r.dvx_dx);
          s[SYY * n + i] = (T)(pert[3][i] * div + 2.0 * pert[4][i] * r.dvy_dy);
          s[SZZ * n + i] = (T)(pert[3][i] * div + 2.0 * pert[4][i] * r.dvz_dz);
          s[SXZ * n + i] = pert[5][i] * r.exz;
          s[SXY * n + i] = pert[6][i] * r.exy;
          s[SYZ * n + i] = pert[7][i] * r.eyz;
        }
  }
  Fields<T> p0, p1;
  p0.alloc(n); p1.alloc(n);
  for (int comp = 0; comp < NCOMP; comp++)
    std::fill(data[comp], data[comp] + (size_t)rec.n[gridOf(comp)] * C.nts, T(0));
  const long long* rpos[NCOMP];
  receiverTable(rec, q2compat, rpos);
  for (int its = 0; its < C.nts - 1; its++) {
    const T* sl = S.data() + (size_t)its * NCOMP * n;
    const T* sr = S.data() + (size_t)(its + 1) * NCOMP * n;
    for (int it2 = 1; it2 < C.sub + 1; it2++) {
      step(C, p0.p, p1.p, med, 0);
      const T fl = C.filt[it2 - 1], fr = C.filt[C.hfilt + it2 - 1];
#pragma omp parallel for collapse(2)
      for (int iy = FAT; iy < C.ny - FAT; iy++)
        for (int ix = FAT; ix < C.nx - FAT; ix++)
          for (int iz = FAT; iz < C.nz - FAT; iz++) {
            const long long i = (long long)iy * C.yStride + (long long)ix * C.nz + iz;
            for (int k = 0; k < NCOMP; k++) p0.p[k][i] += sl[(size_t)k * n + i] * fl + sr[(size_t)k * n + i] * fr;
          }
      dampBoth(C, p0.p, p1.p);
      recordSignals(C, p0.p, data, rec, its, it2, rpos);
      swapFields(p0, p1);
    }
  }
}

// Born adjoint (BornElasticAdjGpu_3D, BornElasticGpuFunctions_3D.cu:2103-2336).
// The 8 perturbation planes are accumulated into (the reference copies the
// caller's planes to the device first and adds the image to them).
template <typename T>
void bornAdj(const Ctx<T>& C, const T* const* med, const T* const* srcSig, const T* const* data,
             const Geom& src, const Geom& rec, T* const* pert, int q2compat, int q3compat) {
  std::vector<T> V;
  bornSourceWavefield(C, med, srcSig, src, V);
  const long long n = C.n;
  // Adjoint wavefield decimated to coarse samples: A[t][comp][cell]
  std::vector<T> A((size_t)C.nts * NCOMP * n, T(0));
  Fields<T> p0, p1;
  p0.alloc(n); p1.alloc(n);
  const long long* rpos[NCOMP];
  receiverTable(rec, q2compat, rpos);
  auto image = [&](int t) {
    const T* a = A.data() + (size_t)t * NCOMP * n;
#pragma omp parallel for collapse(2)
    for (int iy = FAT; iy < C.ny - FAT; iy++)
      for (int ix = FAT; ix < C.nx - FAT; ix++)
        for (int iz = FAT; iz < C.nz - FAT; iz++) {
          const long long i = (long long)iy * C.yStride + (long long)ix * C.nz + iz;
          const ImagingTerms<T> r = imagingTerms(C, V, t, i, q3compat);
          pert[0][i] += a[VX * n + i] * r.tx;
          pert[1][i] += a[VY * n + i] * r.ty;
          pert[2][i] += a[VZ * n + i] * r.tz;
          pert[3][i] += (a[SXX * n + i] + a[SYY * n + i] + a[SZZ * n + i]) * (r.dvx_dx + r.dvy_dy + r.dvz_dz);
          pert[4][i] = (T)(pert[4][i] + 2.0 * (r.dvx_dx * a[SXX * n + i] + r.dvy_dy * a[SYY * n + i] + r.dvz_dz * a[SZZ * n + i]));
          pert[5][i] += a[SXZ * n + i] * r.exz;
          pert[6][i] += a[SXY * n + i] * r.exy;
          pert[7][i] += a[SYZ * n + i] * r.eyz;
        }
  };
  for (int its = C.nts - 2; its > -1; its--) {
    T* al = A.data() + (size_t)its * NCOMP * n;
    T* ar = A.data() + (size_t)(its + 1) * NCOMP * n;
    for (int it2 = C.sub - 1; it2 > -1; it2--) {
      step(C, p0.p, p1.p, med, 2);
      injectSignals(C, p0.p, data, rec, its, it2 + 1, rpos);
      dampBoth(C, p0.p, p1.p);
      const T fl = C.filt[it2], fr = C.filt[C.hfilt + it2];
#pragma omp parallel for collapse(2)
      for (int iy = FAT; iy < C.ny - FAT; iy++)
        for (int ix = FAT; ix < C.nx - FAT; ix++)
          for (int iz = FAT; iz < C.nz - FAT; iz++) {
            const long long i = (long long)iy * C.yStride + (long long)ix * C.nz + iz;
            for (int k = 0; k < NCOMP; k++) {
              al[(size_t)k * n + i] += p0.p[k][i] * fl;
              ar[(size_t)k * n + i] += p0.p[k][i] * fr;
            }
          }
      swapFields(p0, p1);
    }
    image(its + 1);
  }
  image(0);
}

template <typename T>
Geom makeGeom(const long long* const* pos, const long long* n) {
  Geom g;
  for (int k = 0; k < NGRID; k++) { g.pos[k] = pos[k]; g.n[k] = n[k]; }
  return g;
}

}  // namespace

extern "C" {

// Parameters shared by every oracle entry point (internal sub, i.e. twice
// the parfile value, as passed to initNonlinearElasticGpu_3D).
struct oracle_params {
  int nz, nx, ny, nts, sub, minPad;
  double dz, dx, dy, dts, alphaCos;
  int q2compat, q3compat, fix_q1;
  int free_surface;  // nonlinear propagation only; the Born entry points reject it
};

int oracle_num_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}

#define ORACLE_ENTRY(T, SUF)                                                                             \
  int oracle_nl_fwd_##SUF(const oracle_params* P, const T* const* med, const T* const* model,           \
                          T* const* data, const long long* const* spos, const long long* sn,            \
                          const long long* const* rpos, const long long* rn) {                          \
    Ctx<T> C;                                                                                            \
    makeCtx(C, P->nz, P->nx, P->ny, P->nts, P->dts, P->sub, P->minPad, P->dz, P->dx, P->dy,             \
            P->alphaCos, P->fix_q1);                                                                     \
    C.freeSurface = P->free_surface;                                                                     \
    nlFwd(C, med, model, data, makeGeom<T>(spos, sn), makeGeom<T>(rpos, rn), P->q2compat);             \
    return 0;                                                                                            \
  }                                                                                                      \
  int oracle_nl_adj_##SUF(const oracle_params* P, const T* const* med, T* const* model,                 \
                          const T* const* data, const long long* const* spos, const long long* sn,      \
                          const long long* const* rpos, const long long* rn) {                          \
    Ctx<T> C;                                                                                            \
    makeCtx(C, P->nz, P->nx, P->ny, P->nts, P->dts, P->sub, P->minPad, P->dz, P->dx, P->dy,             \
            P->alphaCos, P->fix_q1);                                                                     \
    C.freeSurface = P->free_surface;                                                                     \
    nlAdj(C, med, model, data, makeGeom<T>(spos, sn), makeGeom<T>(rpos, rn), P->q2compat);             \
    return 0;                                                                                            \
  }                                                                                                      \
  int oracle_born_fwd_##SUF(const oracle_params* P, const T* const* med, const T* const* src,           \
                            T* const* data, const long long* const* spos, const long long* sn,          \
                            const long long* const* rpos, const long long* rn, const T* const* pert) {  \
    Ctx<T> C;                                                                                            \
    makeCtx(C, P->nz, P->nx, P->ny, P->nts, P->dts, P->sub, P->minPad, P->dz, P->dx, P->dy,             \
            P->alphaCos, P->fix_q1);                                                                     \
    if (P->free_surface) return 1;                                                                       \
    bornFwd(C, med, src, data, makeGeom<T>(spos, sn), makeGeom<T>(rpos, rn), pert, P->q2compat,        \
            P->q3compat);                                                                                \
    return 0;                                                                                            \
  }                                                                                                      \
  int oracle_born_adj_##SUF(const oracle_params* P, const T* const* med, const T* const* src,           \
                            const T* const* data, const long long* const* spos, const long long* sn,    \
                            const long long* const* rpos, const long long* rn, T* const* pert) {        \
    Ctx<T> C;                                                                                            \
    makeCtx(C, P->nz, P->nx, P->ny, P->nts, P->dts, P->sub, P->minPad, P->dz, P->dx, P->dy,             \
            P->alphaCos, P->fix_q1);                                                                     \
    if (P->free_surface) return 1;                                                                       \
    bornAdj(C, med, src, data, makeGeom<T>(spos, sn), makeGeom<T>(rpos, rn), pert, P->q2compat,        \
            P->q3compat);                                                                                \
    return 0;                                                                                            \
  }                                                                                                      \
  /* One stepper application on caller arrays (unit tests and the CPU baseline). */                     \
  int oracle_step_##SUF(const oracle_params* P, T* const* p0, T* const* p1, const T* const* med,        \
                        int mode, int damp) {                                                            \
    Ctx<T> C;                                                                                            \
    makeCtx(C, P->nz, P->nx, P->ny, P->nts, P->dts, P->sub, P->minPad, P->dz, P->dx, P->dy,             \
            P->alphaCos, P->fix_q1);                                                                     \
    step(C, p0, p1, med, mode);                                                                          \
    if (damp) dampBoth(C, p0, p1);                                                                       \
    return 0;                                                                                            \
  }                                                                                                      \
  /* Constant tables (FD coefficients z,x,y; time filter; taper) for inspection. */                     \
  int oracle_constants_##SUF(const oracle_params* P, T* coef12, T* filt, T* taper, T* dtsInv) {         \
    Ctx<T> C;                                                                                            \
    makeCtx(C, P->nz, P->nx, P->ny, P->nts, P->dts, P->sub, P->minPad, P->dz, P->dx, P->dy,             \
            P->alphaCos, P->fix_q1);                                                                     \
    for (int i = 0; i < 4; i++) { coef12[i] = C.cz[i]; coef12[4 + i] = C.cx[i]; coef12[8 + i] = C.cy[i]; } \
    for (int i = 0; i < 2 * C.hfilt; i++) filt[i] = C.filt[i];                                           \
    for (int i = 0; i < P->minPad; i++) taper[i] = C.damp[i];                                            \
    *dtsInv = C.dtsInv;                                                                                  \
    return 0;                                                                                            \
  }

ORACLE_ENTRY(float, f32)
ORACLE_ENTRY(double, f64)

}  // extern "C"
