// Native host preparation: medium staggering/scaling, staggering operators
// and trilinear acquisition mapping.  Arithmetic follows the reference's
// mixed float/double expressions so that indices (bit-exact contract),
// weights and medium planes match it exactly.
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "../../include/elastic3d_b200.h"
#include "common.cuh"

using e3d::setLastError;

namespace {

inline long long idx(int nz, int nx, int iz, int ix, int iy) {
  return (long long)iy * nz * nx + (long long)ix * nz + iz;
}

// staggerZ/X/Y adjoint: m[i] += 0.5(d[i]+d[i-1]) (1<=i<n-1), m[0] += 0.5 d[0],
// m[n-1] += d[n-1] + 0.5 d[n-2]          (stagger_3D.cpp:47-70)
// forward: d[i] += 0.5(m[i]+m[i+1]) (i<n-1), d[n-1] += m[n-1]   (stagger_3D.cpp:23-45)
void stagger(int nz, int nx, int ny, int axis, bool adjoint, bool add, const float* in, float* out) {
  const long long n = (long long)nz * nx * ny;
  if (!add) std::memset(out, 0, n * sizeof(float));
  const int len = axis == 0 ? nz : axis == 1 ? nx : ny;
  const long long stride = axis == 0 ? 1 : axis == 1 ? nz : (long long)nz * nx;
  // iterate over all lines along `axis`
  const int n1 = axis == 0 ? nx : nz;  // the two other axes
  const int n2 = axis == 2 ? nx : ny;
#pragma omp parallel for collapse(2)
  for (int b = 0; b < n2; b++) {
    for (int a = 0; a < n1; a++) {
      long long base;
      if (axis == 0) base = idx(nz, nx, 0, a, b);
      else if (axis == 1) base = idx(nz, nx, a, 0, b);
      else base = idx(nz, nx, a, b, 0);
      const float* d = in + base;
      float* m = out + base;
      if (adjoint) {
        for (int i = 1; i < len - 1; i++) m[i * stride] += 0.5 * (d[i * stride] + d[(i - 1) * stride]);
        m[0] += 0.5 * d[0];
        m[(len - 1) * stride] += d[(len - 1) * stride] + 0.5 * d[(len - 2) * stride];
      } else {
        for (int i = 0; i < len - 1; i++) m[i * stride] += 0.5 * (d[i * stride] + d[(i + 1) * stride]);
        m[(len - 1) * stride] += d[(len - 1) * stride];
      }
    }
  }
}

struct Pads {
  int fat, zPadMinus, zPadPlus, xPadMinus, xPadPlus, yPad;
};
struct Grid {
  int nz, nx, ny;
  float oz, ox, oy, dz, dx, dy;
};

// spaceInterpGpu_3D::checkOutOfBounds (spaceInterpGpu_3D.cpp:178-213): every
// device inside the model interior (float arithmetic, with a tolerance)
bool devicesInside(const Grid& g, const Pads& p, const float* z, const float* x, const float* y, long long nDev,
                   float tol) {
  const int nzS = g.nz - 2 * p.fat - p.zPadMinus - p.zPadPlus;
  const int nxS = g.nx - 2 * p.fat - p.xPadMinus - p.xPadPlus;
  const int nyS = g.ny - 2 * p.fat - 2 * p.yPad;
  const float zMin = g.oz + (p.fat + p.zPadMinus) * g.dz;
  const float xMin = g.ox + (p.fat + p.xPadMinus) * g.dx;
  const float yMin = g.oy + (p.fat + p.yPad) * g.dy;
  const float zMax = zMin + (nzS - 1) * g.dz;
  const float xMax = xMin + (nxS - 1) * g.dx;
  const float yMax = yMin + (nyS - 1) * g.dy;
  for (long long i = 0; i < nDev; i++)
    if (z[i] - zMax > tol || z[i] - zMin < -tol || x[i] - xMax > tol || x[i] - xMin < -tol || y[i] - yMax > tol ||
        y[i] - yMin < -tol)
      return false;
  return true;
}

// Trilinear pole (spaceInterpGpu_3D.cpp:216-270): the 8 corners of the cell
// holding the point, z fastest, with the reference's float/double mix
// (w = 1 - frac rounded to float; each weight is the reference's own product
// expression, some evaluated in float and some in double, and the second pole
// of a dipole carries a (-1.0) factor in front).  dyPole is the y sampling the
// offset is divided by.  False when a corner leaves the model interior.
bool linearPole(const Grid& g, const Pads& p, float zd, float xd, float yd, float dyPole, bool second,
                long long* index, float* weight) {
  float wz = (zd - g.oz) / g.dz;
  float wx = (xd - g.ox) / g.dx;
  float wy = (yd - g.oy) / dyPole;
  const long long zr = (long long)wz, xr = (long long)wx, yr = (long long)wy;
  wz = wz - zr; wz = 1.0 - wz;
  wx = wx - xr; wx = 1.0 - wx;
  wy = wy - yr; wy = 1.0 - wy;
  if (yr < p.fat + p.yPad || yr + 1 >= g.ny - p.fat - p.yPad || xr < p.fat + p.xPadMinus ||
      xr + 1 >= g.nx - p.fat - p.xPadPlus || zr < p.fat + p.zPadMinus || zr + 1 >= g.nz - p.fat - p.zPadPlus)
    return false;
  const long long nz = g.nz, nzx = (long long)g.nz * g.nx;
  const long long b = yr * nzx + xr * nz + zr;
  const long long off[8] = {0, 1, nz, nz + 1, nzx, nzx + 1, nzx + nz, nzx + nz + 1};
  for (int k = 0; k < 8; k++) index[k] = b + off[k];
  if (!second) {
    weight[0] = wz * wx * wy;
    weight[1] = (1.0 - wz) * wx * wy;
    weight[2] = wz * (1.0 - wx) * wy;
    weight[3] = (1.0 - wz) * (1.0 - wx) * wy;
    weight[4] = wz * wx * (1.0 - wy);
    weight[5] = (1.0 - wz) * wx * (1.0 - wy);
    weight[6] = wz * (1.0 - wx) * (1.0 - wy);
    weight[7] = (1.0 - wz) * (1.0 - wx) * (1.0 - wy);
  } else {
    weight[0] = (-1.0) * wz * wx * wy;
    weight[1] = (-1.0) * (1.0 - wz) * wx * wy;
    weight[2] = (-1.0) * wz * (1.0 - wx) * wy;
    weight[3] = (-1.0) * (1.0 - wz) * (1.0 - wx) * wy;
    weight[4] = (-1.0) * wz * wx * (1.0 - wy);
    weight[5] = (-1.0) * (1.0 - wz) * wx * (1.0 - wy);
    weight[6] = (-1.0) * wz * (1.0 - wx) * (1.0 - wy);
    weight[7] = (-1.0) * (1.0 - wz) * (1.0 - wx) * (1.0 - wy);
  }
  return true;
}

// sin(a)/a in double with its limit 1 at a = 0: below |a| = 1.2e-4 the Taylor
// series 1 - a^2/6 + a^4/120 (its next term is below 1e-20 there).
double sincOfArg(double a) {
  if (std::fabs(a) < 1.2e-4) {
    const double a2 = a * a;
    return 1.0 - a2 / 6.0 + a2 * a2 / 120.0;
  }
  return std::sin(a) / a;
}

// Windowless sinc pole (spaceInterpGpu_3D.cpp:351-413): the 2h points per
// axis r-h+1 .. r+h around the cell corner r below the point, y then x then z
// (z fastest); weight sinc(pi wz) sinc(pi wx) sinc(pi wy) in double, stored
// as float, with w = (device - point) / d in float.  The reference's bounds
// test is inverted and rejects every in-bounds stencil; here the stencil must
// lie inside the array (false otherwise).
bool sincPole(const Grid& g, int h, float zd, float xd, float yd, long long* index, float* weight) {
  const float zReg = (zd - g.oz) / g.dz;
  const float xReg = (xd - g.ox) / g.dx;
  const float yReg = (yd - g.oy) / g.dy;
  const long long zr = (long long)zReg, xr = (long long)xReg, yr = (long long)yReg;
  if (yr - h + 1 < 0 || yr + h >= g.ny || xr - h + 1 < 0 || xr + h >= g.nx || zr - h + 1 < 0 || zr + h >= g.nz)
    return false;
  const int nf1 = 2 * h;
  for (int iy = 0; iy < nf1; iy++)
    for (int ix = 0; ix < nf1; ix++)
      for (int iz = 0; iz < nf1; iz++) {
        const long long py = yr + iy - h + 1, px = xr + ix - h + 1, pz = zr + iz - h + 1;
        const float yCur = py * g.dy + g.oy;
        const float xCur = px * g.dx + g.ox;
        const float zCur = pz * g.dz + g.oz;
        const float wy = (yd - yCur) / g.dy;
        const float wx = (xd - xCur) / g.dx;
        const float wz = (zd - zCur) / g.dz;
        const long long k = ((long long)iy * nf1 + ix) * nf1 + iz;
        index[k] = (long long)g.nz * g.nx * py + (long long)g.nz * px + pz;
        weight[k] = (float)(sincOfArg(M_PI * wz) * sincOfArg(M_PI * wx) * sincOfArg(M_PI * wy));
      }
  return true;
}

// spaceInterpGpu_3D::convertIrregToReg (spaceInterpGpu_3D.cpp:113-138): unique
// grid points in first-seen order, keyed, as the reference's std::map<int,int>
// is, by the index converted to int; slot[i] = position of index[i] among them.
void uniquePoints(const long long* index, long long n, long long* unique, long long* slot, long long* nUnique) {
  std::unordered_map<long long, long long> seen;
  seen.reserve((size_t)(n * 2 + 16));
  long long nu = 0;
  for (long long i = 0; i < n; i++) {
    const long long key = (long long)(int)index[i];
    auto it = seen.find(key);
    if (it == seen.end()) {
      seen.emplace(key, nu);
      unique[nu] = index[i];
      slot[i] = nu++;
    } else {
      slot[i] = it->second;
    }
  }
  *nUnique = nu;
}

}  // namespace

extern "C" {

int e3d_stagger(int nz, int nx, int ny, int axis, int adjoint, int add, const float* in, float* out) {
  if (nz < 2 || nx < 2 || ny < 2 || axis < 0 || axis > 2 || !in || !out) {
    setLastError("bad stagger arguments", __FILE__, __LINE__);
    return E3D_ERR_ARG;
  }
  stagger(nz, nx, ny, axis, adjoint != 0, add != 0, in, out);
  return E3D_OK;
}

// fdParamElastic_3D::fdParamElastic_3D medium preparation (fdParamElastic_3D.cpp:130-193)
int e3d_medium_planes(int nz, int nx, int ny, float dtw, const float* elastic, float* const* out8) {
  if (nz < 2 || nx < 2 || ny < 2 || !elastic || !out8 || !(dtw > 0)) {
    setLastError("bad medium arguments", __FILE__, __LINE__);
    return E3D_ERR_ARG;
  }
  for (int k = 0; k < 8; k++)
    if (!out8[k]) {
      setLastError("null output plane", __FILE__, __LINE__);
      return E3D_ERR_ARG;
    }
  const long long n = (long long)nz * nx * ny;
  const float* rho = elastic;
  const float* lam = elastic + n;
  const float* mu = elastic + 2 * n;
  std::vector<float> t1(n), t2(n);
  stagger(nz, nx, ny, 1, true, false, rho, out8[0]);  // rho_x
  stagger(nz, nx, ny, 2, true, false, rho, out8[1]);  // rho_y
  stagger(nz, nx, ny, 0, true, false, rho, out8[2]);  // rho_z
  stagger(nz, nx, ny, 1, true, false, mu, t1.data());
  stagger(nz, nx, ny, 0, true, false, t1.data(), out8[5]);  // mu_xz
  stagger(nz, nx, ny, 2, true, false, t1.data(), out8[6]);  // mu_xy
  stagger(nz, nx, ny, 2, true, false, mu, t2.data());
  stagger(nz, nx, ny, 0, true, false, t2.data(), out8[7]);  // mu_yz
  const double twoDtw = 2.0 * (double)dtw;
#pragma omp parallel for
  for (long long i = 0; i < n; i++) {
    out8[0][i] = (float)(twoDtw / out8[0][i]);
    out8[1][i] = (float)(twoDtw / out8[1][i]);
    out8[2][i] = (float)(twoDtw / out8[2][i]);
    out8[4][i] = (float)(twoDtw * lam[i]);
    out8[3][i] = (float)(twoDtw * ((double)lam[i] + 2.0 * mu[i]));
    out8[5][i] = (float)(twoDtw * out8[5][i]);
    out8[6][i] = (float)(twoDtw * out8[6][i]);
    out8[7][i] = (float)(twoDtw * out8[7][i]);
  }
  return E3D_OK;
}

// spaceInterpGpu_3D: checkOutOfBounds + calcLinearWeights / calcSincWeights +
// convertIrregToReg (spaceInterpGpu_3D.cpp:113-138, 178-480).
int e3d_space_interp(int method, int hFilter, const float* z, const float* x, const float* y, long long nDev, int nz,
                     int nx, int ny, float oz, float ox, float oy, float dz, float dx, float dy, const int* pads,
                     float tol, int dipole, float zshift, float xshift, float yshift, int compat, long long* index,
                     float* weight, long long* unique, long long* slot, long long* nUnique) {
  if (nDev < 0 || !pads || !index || !weight || !unique || !slot || !nUnique || (nDev > 0 && (!z || !x || !y))) {
    setLastError("bad spaceInterp arguments", __FILE__, __LINE__);
    return E3D_ERR_ARG;
  }
  if (method == E3D_INTERP_LINEAR && hFilter != 1) {
    setLastError("linear interpolation requires a half filter length of 1", __FILE__, __LINE__);
    return E3D_ERR_ARG;
  }
  if ((method != E3D_INTERP_LINEAR && method != E3D_INTERP_SINC) || hFilter < 1 || hFilter > 16) {
    setLastError("unsupported interpolation method or half filter length", __FILE__, __LINE__);
    return E3D_ERR_ARG;
  }
  const Pads pd{pads[0], pads[1], pads[2], pads[3], pads[4], pads[5]};
  const Grid g{nz, nx, ny, oz, ox, oy, dz, dx, dy};
  if (!devicesInside(g, pd, z, x, y, nDev, tol)) {
    setLastError("acquisition device outside the model interior", __FILE__, __LINE__);
    return E3D_ERR_BOUNDS;
  }
  const int nf1 = 2 * hFilter;
  const long long nPole = (long long)nf1 * nf1 * nf1;
  const long long nf = dipole ? 2 * nPole : nPole;
  // the reference keeps the dipole shifts in int members (spaceInterpGpu_3D.h:25)
  const float zs = compat ? (float)(int)zshift : zshift;
  const float xs = compat ? (float)(int)xshift : xshift;
  const float ys = compat ? (float)(int)yshift : yshift;
  for (long long d = 0; d < nDev; d++) {
    for (int part = 0; part < (dipole ? 2 : 1); part++) {
      long long* ix = index + d * nf + part * nPole;
      float* w = weight + d * nf + part * nPole;
      const float zd = part ? z[d] + zs : z[d];
      const float xd = part ? x[d] + xs : x[d];
      const float yd = part ? y[d] + ys : y[d];
      bool ok;
      if (method == E3D_INTERP_LINEAR) {
        // the reference divides the second pole's y offset by dz; the second
        // pole enters with negative weights
        ok = linearPole(g, pd, zd, xd, yd, part && compat ? dz : dy, part == 1, ix, w);
      } else {
        ok = sincPole(g, hFilter, zd, xd, yd, ix, w);
        // the reference's sinc dipole keeps positive weights; the corrected form
        // subtracts the second pole as the linear dipole does
        if (part && !compat)
          for (long long k = 0; k < nPole; k++) w[k] = -w[k];
      }
      if (!ok) {
        setLastError("interpolation stencil outside the grid", __FILE__, __LINE__);
        return E3D_ERR_BOUNDS;
      }
    }
  }
  uniquePoints(index, nDev * nf, unique, slot, nUnique);
  return E3D_OK;
}

int e3d_space_interp_linear(const float* z, const float* x, const float* y, long long nDev, int nz, int nx, int ny,
                            float oz, float ox, float oy, float dz, float dx, float dy, const int* pads,
                            float tol, int dipole, float zshift, float xshift, float yshift, long long* index,
                            float* weight, long long* unique, long long* slot, long long* nUnique) {
  return e3d_space_interp(E3D_INTERP_LINEAR, 1, z, x, y, nDev, nz, nx, ny, oz, ox, oy, dz, dx, dy, pads, tol, dipole,
                          zshift, xshift, yshift, 1, index, weight, unique, slot, nUnique);
}

}  // extern "C"
