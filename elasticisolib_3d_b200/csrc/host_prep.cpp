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

// spaceInterpGpu_3D::checkOutOfBounds + calcLinearWeights + convertIrregToReg
// (spaceInterpGpu_3D.cpp:113-138, 178-348)
int e3d_space_interp_linear(const float* z, const float* x, const float* y, long long nDev, int nz, int nx, int ny,
                            float oz, float ox, float oy, float dz, float dx, float dy, const int* pads,
                            float tol, int dipole, float zshift, float xshift, float yshift, long long* index,
                            float* weight, long long* unique, long long* slot, long long* nUnique) {
  if (nDev < 0 || !pads || !index || !weight || !unique || !slot || !nUnique || (nDev > 0 && (!z || !x || !y))) {
    setLastError("bad spaceInterp arguments", __FILE__, __LINE__);
    return E3D_ERR_ARG;
  }
  const int fat = pads[0], zPadMinus = pads[1], zPadPlus = pads[2], xPadMinus = pads[3], xPadPlus = pads[4],
            yPad = pads[5];
  // bounds of the model interior (float arithmetic)
  const int nzS = nz - 2 * fat - zPadMinus - zPadPlus;
  const int nxS = nx - 2 * fat - xPadMinus - xPadPlus;
  const int nyS = ny - 2 * fat - 2 * yPad;
  const float zMin = oz + (fat + zPadMinus) * dz;
  const float xMin = ox + (fat + xPadMinus) * dx;
  const float yMin = oy + (fat + yPad) * dy;
  const float zMax = zMin + (nzS - 1) * dz;
  const float xMax = xMin + (nxS - 1) * dx;
  const float yMax = yMin + (nyS - 1) * dy;
  for (long long i = 0; i < nDev; i++) {
    if (z[i] - zMax > tol || z[i] - zMin < -tol || x[i] - xMax > tol || x[i] - xMin < -tol || y[i] - yMax > tol ||
        y[i] - yMin < -tol) {
      setLastError("acquisition device outside the model interior", __FILE__, __LINE__);
      return E3D_ERR_BOUNDS;
    }
  }
  const int nf = dipole ? 16 : 8;
  // the reference stores the dipole shifts in int members (spaceInterpGpu_3D.h:25)
  const int zs = (int)zshift, xs = (int)xshift, ys = (int)yshift;
  for (long long d = 0; d < nDev; d++) {
    for (int part = 0; part < (dipole ? 2 : 1); part++) {
      float wz, wx, wy;
      if (part == 0) {
        wz = (z[d] - oz) / dz;
        wx = (x[d] - ox) / dx;
        wy = (y[d] - oy) / dy;
      } else {  // dipole point; the reference divides the y offset by dz
        wz = (z[d] + zs - oz) / dz;
        wx = (x[d] + xs - ox) / dx;
        wy = (y[d] + ys - oy) / dz;
      }
      const long long zr = (long long)wz, xr = (long long)wx, yr = (long long)wy;
      wz = wz - zr; wz = 1.0 - wz;
      wx = wx - xr; wx = 1.0 - wx;
      wy = wy - yr; wy = 1.0 - wy;
      if (yr < fat + yPad || yr + 1 >= ny - fat - yPad || xr < fat + xPadMinus || xr + 1 >= nx - fat - xPadPlus ||
          zr < fat + zPadMinus || zr + 1 >= nz - fat - zPadPlus) {
        setLastError("interpolation stencil outside the model interior", __FILE__, __LINE__);
        return E3D_ERR_BOUNDS;
      }
      const long long i1 = d * nf + part * 8;
      const long long b = yr * nz * nx + xr * nz + zr;
      const long long off[8] = {0, 1, nz, nz + 1, (long long)nz * nx, (long long)nz * nx + 1,
                                (long long)nz * nx + nz, (long long)nz * nx + nz + 1};
      for (int k = 0; k < 8; k++) index[i1 + k] = b + off[k];
      if (part == 0) {
        weight[i1 + 0] = wz * wx * wy;
        weight[i1 + 1] = (1.0 - wz) * wx * wy;
        weight[i1 + 2] = wz * (1.0 - wx) * wy;
        weight[i1 + 3] = (1.0 - wz) * (1.0 - wx) * wy;
        weight[i1 + 4] = wz * wx * (1.0 - wy);
        weight[i1 + 5] = (1.0 - wz) * wx * (1.0 - wy);
        weight[i1 + 6] = wz * (1.0 - wx) * (1.0 - wy);
        weight[i1 + 7] = (1.0 - wz) * (1.0 - wx) * (1.0 - wy);
      } else {
        weight[i1 + 0] = (-1.0) * wz * wx * wy;
        weight[i1 + 1] = (-1.0) * (1.0 - wz) * wx * wy;
        weight[i1 + 2] = (-1.0) * wz * (1.0 - wx) * wy;
        weight[i1 + 3] = (-1.0) * (1.0 - wz) * (1.0 - wx) * wy;
        weight[i1 + 4] = (-1.0) * wz * wx * (1.0 - wy);
        weight[i1 + 5] = (-1.0) * (1.0 - wz) * wx * (1.0 - wy);
        weight[i1 + 6] = (-1.0) * wz * (1.0 - wx) * (1.0 - wy);
        weight[i1 + 7] = (-1.0) * (1.0 - wz) * (1.0 - wx) * (1.0 - wy);
      }
    }
  }
  // unique grid points in first-seen order; the reference keys an
  // std::map<int,int> by the index converted to int
  std::unordered_map<long long, long long> seen;
  seen.reserve((size_t)(nDev * nf * 2 + 16));
  long long nu = 0;
  for (long long i = 0; i < nDev * nf; i++) {
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
  return E3D_OK;
}

}  // extern "C"
