// Host C++ operator classes with the reference's names and call shapes, over
// the C ABI of include/elastic3d_b200.h, bound to Python as
// pyElastic_iso_float_3D (the reference binds its C++ classes the same way,
// python_float/pyElastic_iso_float_nl_3D.cpp, pyElastic_iso_float_born_3D.cpp).
//
//   paramObj                        parameter set (getInt / getFloat / getString with defaults)
//   hypercube, float4DReg           minimal stand-ins for the SEP types the reference's classes take
//   spaceInterpGpu_3D               spaceInterpGpu_3D.cpp:13-175 (linear interpolation only)
//   fdParamElastic_3D               fdParamElastic_3D.cpp:13-313 (time axes, QC, medium planes)
//   nonlinearPropElasticShotsGpu_3D nonlinearPropElasticShotsGpu_3D.cpp:122-420 with the per-shot
//                                   work of nonlinearPropElasticGpu_3D.cpp:66-615
//   BornElasticShotsGpu_3D          BornElasticShotsGpu_3D.cpp:143-605, BornElasticGpu_3D.cpp:70-330
//
// Arrays use the numpy view of the reference's hypercubes (slowest axis first):
// elastic / Born model (3, ny, nx, nz); nonlinear model (1 or nExp, 9, nSim, nts);
// data (nExp, 9, nRec, nts); Born source signals (9, nSim, nts) per shot or one for all.
// Shots are dealt to the GPUs of `nGpu` / `iGpu` by one host thread per GPU.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <atomic>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "elastic3d_b200.h"

namespace py = pybind11;

namespace e3dops {

static void check(int st) {
  if (st != E3D_OK) throw std::runtime_error(e3d_last_error());
}

// ---------------------------------------------------------------------------
class paramObj {
 public:
  paramObj() = default;
  explicit paramObj(const std::map<std::string, std::string>& kv) : kv_(kv) {}
  int getInt(const std::string& k, py::object def = py::none()) const { return std::stoi(get(k, def)); }
  float getFloat(const std::string& k, py::object def = py::none()) const { return std::stof(get(k, def)); }
  std::string getString(const std::string& k, py::object def = py::none()) const { return get(k, def); }
  bool has(const std::string& k) const { return kv_.count(k) > 0; }

 private:
  std::string get(const std::string& k, const py::object& def) const {
    auto it = kv_.find(k);
    if (it != kv_.end()) return it->second;
    if (def.is_none()) throw std::runtime_error("missing parameter " + k);
    return py::str(def);
  }
  std::map<std::string, std::string> kv_;
};

struct axis {
  int n = 1;
  float o = 0.f, d = 1.f;
};

class hypercube {
 public:
  explicit hypercube(const std::vector<axis>& axes) : axes_(axes) {}
  // 1-based like SEP
  axis getAxis(int i) const { return axes_.at(i - 1); }
  int getNdim() const { return (int)axes_.size(); }
  const std::vector<axis>& axes() const { return axes_; }

 private:
  std::vector<axis> axes_;
};

// A float array in the numpy view of a hypercube (the hypercube's axis 1 is the last numpy axis).
class float4DReg {
 public:
  float4DReg(std::shared_ptr<hypercube> h, py::array_t<float, py::array::c_style> a) : hyper_(std::move(h)), a_(a) {
    if (!a_.writeable()) throw std::runtime_error("float4DReg needs a writeable float32 array");
  }
  std::shared_ptr<hypercube> getHyper() const { return hyper_; }
  py::array_t<float, py::array::c_style> getNdArray() const { return a_; }
  float* vals() { return a_.mutable_data(); }
  const float* vals() const { return a_.data(); }
  size_t size() const { return (size_t)a_.size(); }
  std::vector<ssize_t> shape() const { return std::vector<ssize_t>(a_.shape(), a_.shape() + a_.ndim()); }

 private:
  std::shared_ptr<hypercube> hyper_;
  py::array_t<float, py::array::c_style> a_;
};

// ---------------------------------------------------------------------------
class spaceInterpGpu_3D {
 public:
  spaceInterpGpu_3D(py::array_t<float, py::array::c_style | py::array::forcecast> z,
                    py::array_t<float, py::array::c_style | py::array::forcecast> x,
                    py::array_t<float, py::array::c_style | py::array::forcecast> y, std::shared_ptr<hypercube> grid,
                    int nt, std::shared_ptr<paramObj> par, int dipole = 0, float zShift = 0.f, float xShift = 0.f,
                    float yShift = 0.f, std::string method = "linear", int hFilter1d = 1, int compat = 1)
      : nt_(nt) {
    if (method != "linear" && method != "sinc") throw std::runtime_error("unsupported spatial interpolation method");
    if (method == "linear" && hFilter1d != 1) throw std::runtime_error("linear interpolation requires hFilter1d = 1");
    if (hFilter1d < 1 || hFilter1d > 16) throw std::runtime_error("hFilter1d must be 1 .. 16");
    const long long n = (long long)z.size();
    if ((long long)x.size() != n || (long long)y.size() != n) throw std::runtime_error("coordinate sizes differ");
    const axis az = grid->getAxis(1), ax = grid->getAxis(2), ay = grid->getAxis(3);
    nf_ = 8 * hFilter1d * hFilter1d * hFilter1d * (dipole ? 2 : 1);
    nIrreg_ = n;
    index_.resize((size_t)n * nf_);
    weight_.resize((size_t)n * nf_);
    slot_.resize((size_t)n * nf_);
    std::vector<long long> uniq(std::max<long long>(n * nf_, 1));
    const int pads[6] = {par->getInt("fat", py::int_(4)), par->getInt("zPadMinus"), par->getInt("zPadPlus"),
                         par->getInt("xPadMinus"), par->getInt("xPadPlus"), par->getInt("yPad")};
    long long nu = 0;
    check(e3d_space_interp(method == "sinc" ? E3D_INTERP_SINC : E3D_INTERP_LINEAR, hFilter1d, z.data(), x.data(),
                           y.data(), n, az.n, ax.n, ay.n, az.o, ax.o, ay.o, az.d, ax.d, ay.d, pads,
                           par->getFloat("errorTolerance", py::float_(1e-6)), dipole, zShift, xShift, yShift, compat,
                           index_.data(), weight_.data(), uniq.data(), slot_.data(), &nu));
    unique_.assign(uniq.begin(), uniq.begin() + nu);
  }
  const std::vector<long long>& getRegPosUnique() const { return unique_; }
  long long getNDeviceReg() const { return (long long)unique_.size(); }
  long long getNDeviceIrreg() const { return nIrreg_; }
  int getNt() const { return nt_; }
  // regular (nReg, nts) -> irregular (nIrreg, nts), device then filter order
  void forward(bool add, const float* reg, float* irr, int nts) const {
    if (!add) std::fill(irr, irr + (size_t)nIrreg_ * nts, 0.f);
    for (long long i = 0; i < nIrreg_; i++)
      for (int f = 0; f < nf_; f++) {
        const size_t e = (size_t)i * nf_ + f;
        const float w = weight_[e];
        const float* m = reg + (size_t)slot_[e] * nts;
        float* d = irr + (size_t)i * nts;
        for (int t = 0; t < nts; t++) d[t] += w * m[t];
      }
  }
  // irregular -> regular, accumulated in device then filter order
  void adjoint(bool add, float* reg, const float* irr, int nts) const {
    if (!add) std::fill(reg, reg + unique_.size() * nts, 0.f);
    for (long long i = 0; i < nIrreg_; i++)
      for (int f = 0; f < nf_; f++) {
        const size_t e = (size_t)i * nf_ + f;
        const float w = weight_[e];
        float* m = reg + (size_t)slot_[e] * nts;
        const float* d = irr + (size_t)i * nts;
        for (int t = 0; t < nts; t++) m[t] += w * d[t];
      }
  }

 private:
  int nt_ = 0, nf_ = 8;
  long long nIrreg_ = 0;
  std::vector<long long> index_, slot_, unique_;
  std::vector<float> weight_;
};
using Interp = std::shared_ptr<spaceInterpGpu_3D>;

// Grid of each wavefield component: vx -> x, vy -> y, vz -> z, normal stresses -> center, sxz, sxy, syz.
static const int kCompGrid[9] = {1, 2, 3, 0, 0, 0, 4, 5, 6};

// ---------------------------------------------------------------------------
class fdParamElastic_3D {
 public:
  fdParamElastic_3D(const float4DReg& elastic, std::shared_ptr<paramObj> par) {
    nts = par->getInt("nts");
    dts = par->getFloat("dts", py::float_(0.0));
    sub = 2 * par->getInt("sub");
    if (sub > 100) throw std::runtime_error("2*sub exceeds SUB_MAX");
    dtw = dts / (float)sub;
    nz = par->getInt("nz");
    nx = par->getInt("nx");
    ny = par->getInt("ny");
    freeSurface = par->getInt("freeSurface", py::int_(0));
    const int zpm = par->getInt("zPadMinus"), zpp = par->getInt("zPadPlus");
    const int xpm = par->getInt("xPadMinus"), xpp = par->getInt("xPadPlus");
    const int zPad = freeSurface ? zpp : std::min(zpm, zpp);
    minPad = std::min(zPad, std::min(xpm, xpp));
    const int modPar = par->getInt("mod_par", py::int_(2));
    dz = par->getFloat("dz", py::float_(-1.0));
    dx = par->getFloat("dx", py::float_(-1.0));
    dy = par->getFloat("dy", py::float_(-1.0));
    if (modPar == 2) {  // km -> m (fdParamElastic_3D.cpp:71-79)
      dz *= 1000.f;
      dx *= 1000.f;
      dy *= 1000.f;
    }
    alphaCos = par->getFloat("alphaCos", py::float_(0.99));
    const float fMax = par->getFloat("fMax", py::float_(1000.0));
    const int blockSize = par->getInt("blockSize", py::int_(16)), fat = par->getInt("fat", py::int_(4));
    auto sh = elastic.shape();
    if (sh.size() != 4 || sh[0] != 3 || sh[1] != ny || sh[2] != nx || sh[3] != nz)
      throw std::runtime_error("elastic parameter cube not consistent with nz/nx/ny");
    // velocity bounds over the window the reference scans (fdParamElastic_3D.cpp:96-114)
    const float* ep = elastic.vals();
    const size_t n = (size_t)nz * nx * ny;
    double vmin = 10000.0, vmax = -1.0;
    for (int iy = fat; iy < ny - 2 * fat; iy++)
      for (int ix = fat; ix < nx - 2 * fat; ix++)
        for (int iz = fat; iz < nz - 2 * fat; iz++) {
          const size_t i = ((size_t)iy * nx + ix) * nz + iz;
          const float rho = ep[i], lam = ep[n + i], mu = ep[2 * n + i];
          const float vp = std::sqrt((lam + 2 * mu) / rho), vs = std::sqrt(mu / rho);
          vmin = std::min<double>(vmin, vp);
          if (vs != 0) vmin = std::min<double>(vmin, vs);
          vmax = std::max<double>(vmax, std::max(vp, vs));
        }
    const double courant = vmax * (double)dtw * 2.0 / std::min(dz, std::min(dx, dy));
    if (courant > 0.45) throw std::runtime_error("Courant is too big");
    if (vmin / (fMax * std::max(dz, std::max(dx, dy))) < 3.0) throw std::runtime_error("Dispersion is too small");
    if ((nz - 2 * fat) % blockSize || (nx - 2 * fat) % blockSize)
      throw std::runtime_error("nz-2*FAT and nx-2*FAT must be multiples of blockSize");
    planes.assign(8 * n, 0.f);
    std::vector<float*> out(8);
    for (int k = 0; k < 8; k++) out[k] = planes.data() + k * n;
    check(e3d_medium_planes(nz, nx, ny, dtw, ep, out.data()));
  }
  const float* plane(int k) const { return planes.data() + (size_t)k * nz * nx * ny; }
  int nz, nx, ny, nts, sub, minPad, freeSurface;
  float dz, dx, dy, dts, dtw, alphaCos;
  std::vector<float> planes;  // rhox, rhoy, rhoz, lambda+2mu, lambda, muxz, muxy, muyz (2dtw-scaled)
};

// ---------------------------------------------------------------------------
// Medium scaling of regular-grid signals in place (nonlinearPropElasticGpu_3D.cpp:200-277, :481-558)
static void scaleSignals(std::vector<std::vector<float>>& reg, const std::vector<Interp>& dev7,
                         const fdParamElastic_3D& fd, int nts) {
  const int simple[6][2] = {{0, 0}, {1, 1}, {2, 2}, {6, 5}, {7, 6}, {8, 7}};
  for (auto& km : simple) {
    const auto& pos = dev7[kCompGrid[km[0]]]->getRegPosUnique();
    const float* m = fd.plane(km[1]);
    for (size_t r = 0; r < pos.size(); r++)
      for (int t = 0; t < nts; t++) reg[km[0]][r * nts + t] *= m[pos[r]];
  }
  const auto& pos = dev7[0]->getRegPosUnique();
  const float* l2m = fd.plane(3);
  const float* lam = fd.plane(4);
  for (size_t r = 0; r < pos.size(); r++)
    for (int t = 0; t < nts; t++) {
      const size_t i = r * nts + t;
      const float sxx = reg[3][i], syy = reg[4][i], szz = reg[5][i];
      const float a = l2m[pos[r]], b = lam[pos[r]];
      reg[3][i] = sxx * a + (syy + szz) * b;
      reg[4][i] = syy * a + (sxx + szz) * b;
      reg[5][i] = szz * a + (sxx + syy) * b;
    }
  const float area = (float)(1.0 / (double)((fd.dx * fd.dy) * fd.dz));
  for (auto& v : reg)
    for (auto& x : v) x *= area;
}

// ---------------------------------------------------------------------------
class ShotOperatorBase {
 public:
  ShotOperatorBase(const float4DReg& elastic, std::shared_ptr<paramObj> par, const std::vector<std::vector<Interp>>& dev14)
      : par_(std::move(par)), fd_(std::make_shared<fdParamElastic_3D>(elastic, par_)) {
    if (dev14.size() != 14) throw std::runtime_error("expected 7 source and 7 receiver acquisition lists");
    for (int g = 0; g < 7; g++) src_.push_back(dev14[g]);
    for (int g = 0; g < 7; g++) rec_.push_back(dev14[7 + g]);
    nExp_ = (int)src_[0].size();
    constRec_ = rec_[0].size() == 1;
    std::vector<int> gpus;
    std::stringstream ss(par_->getString("iGpu", py::str("-1")));
    for (std::string tok; std::getline(ss, tok, ',');)
      if (!tok.empty()) gpus.push_back(std::stoi(tok));
    if (gpus.empty() || gpus[0] < 0) {
      gpus.clear();
      for (int i = 0; i < par_->getInt("nGpu", py::int_(1)); i++) gpus.push_back(i);
    }
    if ((int)gpus.size() > nExp_) throw std::runtime_error("more GPUs than shots to model");
    for (int dev : gpus) {
      e3d_desc d{};
      d.device = dev;
      d.nz = fd_->nz; d.nx = fd_->nx; d.ny = fd_->ny; d.nts = fd_->nts; d.sub = fd_->sub; d.minPad = fd_->minPad;
      d.dz = fd_->dz; d.dx = fd_->dx; d.dy = fd_->dy; d.dts = fd_->dts; d.alphaCos = fd_->alphaCos;
      d.fix_q1 = 0; d.q2compat = 1; d.q3compat = 1; d.free_surface = fd_->freeSurface;
      e3d_context* c = nullptr;
      check(e3d_context_create(&d, &c));
      ctx_.push_back(c);
    }
    setMedium();
  }
  virtual ~ShotOperatorBase() {
    for (auto* c : ctx_) e3d_context_destroy(c);
  }
  void setBackground(const float4DReg& elastic) {
    fd_ = std::make_shared<fdParamElastic_3D>(elastic, par_);
    setMedium();
  }

 protected:
  void setMedium() {
    const size_t n = (size_t)fd_->nz * fd_->nx * fd_->ny;
    std::vector<const float*> p(8);
    for (int k = 0; k < 8; k++) p[k] = fd_->planes.data() + k * n;
    for (auto* c : ctx_) check(e3d_set_medium(c, p.data(), 0));
  }
  std::vector<Interp> srcs(int i) const {
    std::vector<Interp> v;
    for (int g = 0; g < 7; g++) v.push_back(src_[g][i]);
    return v;
  }
  std::vector<Interp> recs(int i) const {
    std::vector<Interp> v;
    for (int g = 0; g < 7; g++) v.push_back(rec_[g][constRec_ ? 0 : i]);
    return v;
  }
  // shots dealt dynamically to one host thread per GPU (nonlinearPropElasticShotsGpu_3D.cpp:178-204)
  template <typename F>
  void runShots(F&& fn) {
    std::atomic<int> next{0};
    std::vector<std::string> errors;
    std::mutex mu;
    auto worker = [&](e3d_context* c) {
      for (int i = next++; i < nExp_; i = next++) {
        try {
          fn(c, i);
        } catch (const std::exception& e) {
          std::lock_guard<std::mutex> lk(mu);
          errors.push_back(e.what());
          return;
        }
      }
    };
    {
      py::gil_scoped_release release;
      std::vector<std::thread> th;
      for (auto* c : ctx_) th.emplace_back(worker, c);
      for (auto& t : th) t.join();
    }
    if (!errors.empty()) throw std::runtime_error(errors[0]);
  }
  static void posTables(const std::vector<Interp>& d7, std::vector<const long long*>& pos, std::vector<long long>& n) {
    pos.resize(7);
    n.resize(7);
    for (int g = 0; g < 7; g++) {
      pos[g] = d7[g]->getRegPosUnique().data();
      n[g] = d7[g]->getNDeviceReg();
    }
  }
  std::vector<std::vector<float>> scaledSources(const std::vector<Interp>& s7, const float* model9, int nSim) const {
    const int nts = fd_->nts;
    std::vector<std::vector<float>> reg(9);
    for (int k = 0; k < 9; k++) {
      reg[k].assign((size_t)s7[kCompGrid[k]]->getNDeviceReg() * nts, 0.f);
      s7[kCompGrid[k]]->adjoint(false, reg[k].data(), model9 + (size_t)k * nSim * nts, nts);
    }
    scaleSignals(reg, s7, *fd_, nts);
    return reg;
  }

  std::shared_ptr<paramObj> par_;
  std::shared_ptr<fdParamElastic_3D> fd_;
  std::vector<std::vector<Interp>> src_, rec_;
  std::vector<e3d_context*> ctx_;
  int nExp_ = 0;
  bool constRec_ = true;
  std::mutex outMu_;
};

// ---------------------------------------------------------------------------
class nonlinearPropElasticShotsGpu_3D : public ShotOperatorBase {
 public:
  nonlinearPropElasticShotsGpu_3D(const float4DReg& elastic, std::shared_ptr<paramObj> par,
                                  std::vector<std::vector<Interp>> dev14)
      : ShotOperatorBase(elastic, std::move(par), dev14) {}

  // model (1 or nExp, 9, nSim, nts) -> data (nExp, 9, nRec, nts)
  void forward(bool add, const float4DReg& model, float4DReg& data) {
    const auto ms = model.shape(), ds = data.shape();
    if (ms.size() != 4 || ms[1] != 9) throw std::runtime_error("model must be (1|nExp, 9, nSim, nts)");
    const int nts = fd_->nts, nSim = (int)ms[2], nRec = (int)ds[2];
    const bool constant = ms[0] == 1;
    if (!add) std::fill(data.vals(), data.vals() + data.size(), 0.f);
    const float* m = model.vals();
    float* out = data.vals();
    runShots([&](e3d_context* c, int i) {
      auto s7 = srcs(i), r7 = recs(i);
      auto reg = scaledSources(s7, m + (size_t)(constant ? 0 : i) * 9 * nSim * nts, nSim);
      std::vector<std::vector<float>> dreg(9);
      std::vector<const float*> in(9);
      std::vector<float*> dout(9);
      for (int k = 0; k < 9; k++) {
        in[k] = reg[k].data();
        dreg[k].assign((size_t)r7[kCompGrid[k]]->getNDeviceReg() * nts, 0.f);
        dout[k] = dreg[k].data();
      }
      std::vector<const long long*> sp, rp;
      std::vector<long long> sn, rn;
      posTables(s7, sp, sn);
      posTables(r7, rp, rn);
      check(e3d_nl_forward(c, in.data(), dout.data(), sp.data(), sn.data(), rp.data(), rn.data()));
      std::vector<float> irr((size_t)9 * nRec * nts, 0.f);
      for (int k = 0; k < 9; k++)
        r7[kCompGrid[k]]->forward(false, dreg[k].data(), irr.data() + (size_t)k * nRec * nts, nts);
      std::lock_guard<std::mutex> lk(outMu_);
      float* o = out + (size_t)i * 9 * nRec * nts;
      for (size_t j = 0; j < irr.size(); j++) o[j] += irr[j];
    });
  }

  // data -> model, the reference's time-reversed stepper (quirk Q7)
  void adjoint(bool add, float4DReg& model, const float4DReg& data) {
    const auto ms = model.shape(), ds = data.shape();
    const int nts = fd_->nts, nSim = (int)ms[2], nRec = (int)ds[2];
    const bool constant = ms[0] == 1;
    if (!add) std::fill(model.vals(), model.vals() + model.size(), 0.f);
    const float* d = data.vals();
    float* out = model.vals();
    runShots([&](e3d_context* c, int i) {
      auto s7 = srcs(i), r7 = recs(i);
      std::vector<std::vector<float>> reg(9), sreg(9);
      std::vector<float*> in(9), sout(9);
      for (int k = 0; k < 9; k++) {
        reg[k].assign((size_t)r7[kCompGrid[k]]->getNDeviceReg() * nts, 0.f);
        r7[kCompGrid[k]]->adjoint(false, reg[k].data(), d + ((size_t)i * 9 + k) * nRec * nts, nts);
      }
      scaleSignals(reg, r7, *fd_, nts);
      for (int k = 0; k < 9; k++) {
        in[k] = reg[k].data();
        sreg[k].assign((size_t)s7[kCompGrid[k]]->getNDeviceReg() * nts, 0.f);
        sout[k] = sreg[k].data();
      }
      std::vector<const long long*> sp, rp;
      std::vector<long long> sn, rn;
      posTables(s7, sp, sn);
      posTables(r7, rp, rn);
      check(e3d_nl_adjoint(c, sout.data(), (const float* const*)in.data(), sp.data(), sn.data(), rp.data(),
                           rn.data()));
      std::vector<float> irr((size_t)9 * nSim * nts, 0.f);
      for (int k = 0; k < 9; k++)
        s7[kCompGrid[k]]->forward(false, sreg[k].data(), irr.data() + (size_t)k * nSim * nts, nts);
      std::lock_guard<std::mutex> lk(outMu_);
      float* o = out + (size_t)(constant ? 0 : i) * 9 * nSim * nts;
      for (size_t j = 0; j < irr.size(); j++) o[j] += irr[j];
    });
  }
};

// ---------------------------------------------------------------------------
// Born model preparation and its adjoint (BornElasticShotsGpu_3D.cpp:167-235, :528-605)
static std::vector<float> stagger(const fdParamElastic_3D& fd, const float* in, int axis, int adjoint) {
  std::vector<float> out((size_t)fd.nz * fd.nx * fd.ny, 0.f);
  check(e3d_stagger(fd.nz, fd.nx, fd.ny, axis, adjoint, 0, in, out.data()));
  return out;
}

class BornElasticShotsGpu_3D : public ShotOperatorBase {
 public:
  BornElasticShotsGpu_3D(const float4DReg& elastic, std::shared_ptr<paramObj> par, std::vector<float4DReg> sources,
                         std::vector<std::vector<Interp>> dev14)
      : ShotOperatorBase(elastic, std::move(par), dev14) {
    for (auto& s : sources) {
      const float* v = s.vals();
      sources_.emplace_back(v, v + s.size());
      nSim_.push_back((int)s.shape()[1]);
    }
    if (sources_.size() != 1 && (int)sources_.size() != nExp_)
      throw std::runtime_error("source signals: one for all shots or one per shot");
  }

  // (drho, dlambda, dmu) (3, ny, nx, nz) -> data (nExp, 9, nRec, nts)
  void forward(bool add, const float4DReg& model, float4DReg& data) {
    const int nts = fd_->nts, nRec = (int)data.shape()[2];
    const size_t n = (size_t)fd_->nz * fd_->nx * fd_->ny;
    const float* m = model.vals();
    // 0 = z, 1 = x, 2 = y
    std::vector<std::vector<float>> pert(8);
    pert[0] = stagger(*fd_, m, 1, 1);
    pert[1] = stagger(*fd_, m, 2, 1);
    pert[2] = stagger(*fd_, m, 0, 1);
    pert[3].assign(m + n, m + 2 * n);
    pert[4].assign(m + 2 * n, m + 3 * n);
    pert[5] = stagger(*fd_, stagger(*fd_, m + 2 * n, 1, 1).data(), 0, 1);
    pert[6] = stagger(*fd_, stagger(*fd_, m + 2 * n, 1, 1).data(), 2, 1);
    pert[7] = stagger(*fd_, stagger(*fd_, m + 2 * n, 2, 1).data(), 0, 1);
    const double two = 2.0 * (double)fd_->dtw;
    for (int k = 0; k < 3; k++)
      for (size_t i = 0; i < n; i++) pert[k][i] *= fd_->plane(k)[i];
    for (int k = 3; k < 8; k++)
      for (size_t i = 0; i < n; i++) pert[k][i] = (float)((double)pert[k][i] * two);
    if (!add) std::fill(data.vals(), data.vals() + data.size(), 0.f);
    float* out = data.vals();
    runShots([&](e3d_context* c, int i) {
      auto s7 = srcs(i), r7 = recs(i);
      const int si = sources_.size() == 1 ? 0 : i;
      auto reg = scaledSources(s7, sources_[si].data(), nSim_[si]);
      std::vector<const float*> in(9), pp(8);
      std::vector<std::vector<float>> dreg(9);
      std::vector<float*> dout(9);
      for (int k = 0; k < 9; k++) {
        in[k] = reg[k].data();
        dreg[k].assign((size_t)r7[kCompGrid[k]]->getNDeviceReg() * nts, 0.f);
        dout[k] = dreg[k].data();
      }
      for (int k = 0; k < 8; k++) pp[k] = pert[k].data();
      std::vector<const long long*> sp, rp;
      std::vector<long long> sn, rn;
      posTables(s7, sp, sn);
      posTables(r7, rp, rn);
      check(e3d_born_forward(c, in.data(), dout.data(), sp.data(), sn.data(), rp.data(), rn.data(), pp.data()));
      std::vector<float> irr((size_t)9 * nRec * nts, 0.f);
      for (int k = 0; k < 9; k++)
        r7[kCompGrid[k]]->forward(false, dreg[k].data(), irr.data() + (size_t)k * nRec * nts, nts);
      std::lock_guard<std::mutex> lk(outMu_);
      float* o = out + (size_t)i * 9 * nRec * nts;
      for (size_t j = 0; j < irr.size(); j++) o[j] += irr[j];
    });
  }

  // data -> (drho, dlambda, dmu)
  void adjoint(bool add, float4DReg& model, const float4DReg& data) {
    const int nts = fd_->nts, nRec = (int)data.shape()[2];
    const size_t n = (size_t)fd_->nz * fd_->nx * fd_->ny;
    std::vector<float> acc(8 * n, 0.f);
    const float* d = data.vals();
    runShots([&](e3d_context* c, int i) {
      auto s7 = srcs(i), r7 = recs(i);
      const int si = sources_.size() == 1 ? 0 : i;
      auto reg = scaledSources(s7, sources_[si].data(), nSim_[si]);
      std::vector<std::vector<float>> dreg(9);
      std::vector<const float*> in(9), dd(9);
      for (int k = 0; k < 9; k++) {
        in[k] = reg[k].data();
        dreg[k].assign((size_t)r7[kCompGrid[k]]->getNDeviceReg() * nts, 0.f);
        r7[kCompGrid[k]]->adjoint(false, dreg[k].data(), d + ((size_t)i * 9 + k) * nRec * nts, nts);
        dd[k] = dreg[k].data();
      }
      std::vector<float> pert(8 * n, 0.f);
      std::vector<float*> pp(8);
      for (int k = 0; k < 8; k++) pp[k] = pert.data() + k * n;
      std::vector<const long long*> sp, rp;
      std::vector<long long> sn, rn;
      posTables(s7, sp, sn);
      posTables(r7, rp, rn);
      check(e3d_born_adjoint(c, in.data(), dd.data(), sp.data(), sn.data(), rp.data(), rn.data(), pp.data()));
      std::lock_guard<std::mutex> lk(outMu_);
      for (size_t j = 0; j < acc.size(); j++) acc[j] += pert[j];
    });
    // gradient post-processing: scale, unstagger (BornElasticShotsGpu_3D.cpp:528-605)
    const double two = 2.0 * (double)fd_->dtw;
    std::vector<std::vector<float>> g(8);
    for (int k = 0; k < 8; k++) {
      g[k].assign(acc.begin() + k * n, acc.begin() + (k + 1) * n);
      for (size_t i = 0; i < n; i++)
        g[k][i] = k < 3 ? g[k][i] * fd_->plane(k)[i] : (float)((double)g[k][i] * two);
    }
    auto sx = stagger(*fd_, g[0].data(), 1, 0), sy = stagger(*fd_, g[1].data(), 2, 0), sz = stagger(*fd_, g[2].data(), 0, 0);
    auto t1 = stagger(*fd_, stagger(*fd_, g[5].data(), 0, 0).data(), 1, 0);
    auto t2 = stagger(*fd_, stagger(*fd_, g[6].data(), 2, 0).data(), 1, 0);
    auto t3 = stagger(*fd_, stagger(*fd_, g[7].data(), 0, 0).data(), 2, 0);
    float* m = model.vals();
    for (size_t i = 0; i < n; i++) {
      float drho = sx[i];
      drho += sy[i];
      drho += sz[i];
      float tt = t1[i];
      tt += t2[i];
      tt += t3[i];
      const float dlam = g[3][i], dmu = g[4][i] + tt;
      if (add) {
        m[i] += drho;
        m[n + i] += dlam;
        m[2 * n + i] += dmu;
      } else {
        m[i] = drho;
        m[n + i] = dlam;
        m[2 * n + i] = dmu;
      }
    }
  }

 private:
  std::vector<std::vector<float>> sources_;
  std::vector<int> nSim_;
};

// Dot-product test of forward/adjoint without and with add (operator.h:50-92).
template <typename Op>
bool dotTest(Op& op, const std::vector<ssize_t>& dshape, const std::vector<ssize_t>& rshape, bool verbose,
             float maxError, std::shared_ptr<hypercube> h) {
  std::mt19937 rng(1234);
  std::uniform_real_distribution<float> u(-1.f, 1.f);
  auto mk = [&](const std::vector<ssize_t>& s, bool rnd) {
    py::array_t<float, py::array::c_style> a(s);
    float* p = a.mutable_data();
    for (ssize_t i = 0; i < a.size(); i++) p[i] = rnd ? u(rng) : 0.f;
    return float4DReg(h, a);
  };
  auto m1 = mk(dshape, true), d1 = mk(rshape, true), m2 = mk(dshape, false), d2 = mk(rshape, false);
  auto dot = [](const float4DReg& a, const float4DReg& b) {
    double s = 0;
    for (size_t i = 0; i < a.size(); i++) s += (double)a.vals()[i] * b.vals()[i];
    return s;
  };
  op.adjoint(false, m2, d1);
  op.forward(false, m1, d2);
  const double e1 = std::fabs((dot(d1, d2) - dot(m1, m2)) / dot(m1, m2));
  op.forward(true, m1, d2);
  op.adjoint(true, m2, d1);
  const double e2 = std::fabs((dot(d1, d2) - dot(m1, m2)) / dot(m1, m2));
  if (verbose) py::print("dot test error without add:", e1, "with add:", e2);
  return e1 <= maxError && e2 <= maxError;
}

}  // namespace e3dops

// ---------------------------------------------------------------------------
PYBIND11_MODULE(pyElastic_iso_float_3D, m) {
  using namespace e3dops;
  m.doc() = "Elastic 3D shot operators (reference class names) over the B200 C ABI";
  py::class_<axis>(m, "axis")
      .def(py::init([](int n, float o, float d) { return axis{n, o, d}; }), py::arg("n") = 1, py::arg("o") = 0.f,
           py::arg("d") = 1.f)
      .def_readwrite("n", &axis::n)
      .def_readwrite("o", &axis::o)
      .def_readwrite("d", &axis::d);
  py::class_<hypercube, std::shared_ptr<hypercube>>(m, "hypercube")
      .def(py::init<const std::vector<axis>&>(), py::arg("axes"))
      .def("getAxis", &hypercube::getAxis)
      .def("getNdim", &hypercube::getNdim);
  py::class_<paramObj, std::shared_ptr<paramObj>>(m, "paramObj")
      .def(py::init([](const py::dict& d) {
        std::map<std::string, std::string> kv;
        for (auto item : d) kv[py::str(item.first)] = py::str(item.second);
        return std::make_shared<paramObj>(kv);
      }))
      .def("getInt", &paramObj::getInt, py::arg("key"), py::arg("default") = py::none())
      .def("getFloat", &paramObj::getFloat, py::arg("key"), py::arg("default") = py::none())
      .def("getString", &paramObj::getString, py::arg("key"), py::arg("default") = py::none());
  py::class_<float4DReg>(m, "float4DReg")
      .def(py::init<std::shared_ptr<hypercube>, py::array_t<float, py::array::c_style>>())
      .def("getHyper", &float4DReg::getHyper)
      .def("getNdArray", &float4DReg::getNdArray);
  py::class_<fdParamElastic_3D, std::shared_ptr<fdParamElastic_3D>>(m, "fdParamElastic_3D")
      .def(py::init<const float4DReg&, std::shared_ptr<paramObj>>(), py::arg("elasticParam"), py::arg("par"))
      .def_readonly("nz", &fdParamElastic_3D::nz)
      .def_readonly("nx", &fdParamElastic_3D::nx)
      .def_readonly("ny", &fdParamElastic_3D::ny)
      .def_readonly("nts", &fdParamElastic_3D::nts)
      .def_readonly("sub", &fdParamElastic_3D::sub)
      .def_readonly("minPad", &fdParamElastic_3D::minPad)
      .def_readonly("freeSurface", &fdParamElastic_3D::freeSurface)
      .def_readonly("dz", &fdParamElastic_3D::dz)
      .def_readonly("dx", &fdParamElastic_3D::dx)
      .def_readonly("dy", &fdParamElastic_3D::dy)
      .def_readonly("dts", &fdParamElastic_3D::dts)
      .def_readonly("dtw", &fdParamElastic_3D::dtw)
      .def_readonly("alphaCos", &fdParamElastic_3D::alphaCos)
      // the eight 2dtw-scaled medium planes, (8, ny, nx, nz), copied out
      .def("getPlanes", [](const fdParamElastic_3D& f) {
        py::array_t<float> out({(ssize_t)8, (ssize_t)f.ny, (ssize_t)f.nx, (ssize_t)f.nz});
        std::copy(f.planes.begin(), f.planes.end(), out.mutable_data());
        return out;
      });
  py::class_<spaceInterpGpu_3D, std::shared_ptr<spaceInterpGpu_3D>>(m, "spaceInterpGpu_3D")
      .def(py::init<py::array_t<float, py::array::c_style | py::array::forcecast>,
                    py::array_t<float, py::array::c_style | py::array::forcecast>,
                    py::array_t<float, py::array::c_style | py::array::forcecast>, std::shared_ptr<hypercube>, int,
                    std::shared_ptr<paramObj>, int, float, float, float, std::string, int, int>(),
           py::arg("zCoord"), py::arg("xCoord"), py::arg("yCoord"), py::arg("grid"), py::arg("nt"), py::arg("par"),
           py::arg("dipole") = 0, py::arg("zShift") = 0.f, py::arg("xShift") = 0.f, py::arg("yShift") = 0.f,
           py::arg("method") = "linear", py::arg("hFilter1d") = 1, py::arg("compat") = 1)
      .def("getRegPosUnique", &spaceInterpGpu_3D::getRegPosUnique)
      .def("getNDeviceReg", &spaceInterpGpu_3D::getNDeviceReg)
      .def("getNDeviceIrreg", &spaceInterpGpu_3D::getNDeviceIrreg);
  py::class_<nonlinearPropElasticShotsGpu_3D, std::shared_ptr<nonlinearPropElasticShotsGpu_3D>>(
      m, "nonlinearPropElasticShotsGpu_3D")
      .def(py::init([](const float4DReg& ep, std::shared_ptr<paramObj> par, std::vector<Interp> s0,
                       std::vector<Interp> s1, std::vector<Interp> s2, std::vector<Interp> s3, std::vector<Interp> s4,
                       std::vector<Interp> s5, std::vector<Interp> s6, std::vector<Interp> r0, std::vector<Interp> r1,
                       std::vector<Interp> r2, std::vector<Interp> r3, std::vector<Interp> r4, std::vector<Interp> r5,
                       std::vector<Interp> r6) {
        return std::make_shared<nonlinearPropElasticShotsGpu_3D>(
            ep, par, std::vector<std::vector<Interp>>{s0, s1, s2, s3, s4, s5, s6, r0, r1, r2, r3, r4, r5, r6});
      }))
      .def("forward", &nonlinearPropElasticShotsGpu_3D::forward)
      .def("adjoint", &nonlinearPropElasticShotsGpu_3D::adjoint)
      .def("setBackground", &nonlinearPropElasticShotsGpu_3D::setBackground)
      .def("dotTest", [](nonlinearPropElasticShotsGpu_3D& op, const float4DReg& model, const float4DReg& data,
                         bool verbose, float maxError) {
        return dotTest(op, model.shape(), data.shape(), verbose, maxError, model.getHyper());
      });
  py::class_<BornElasticShotsGpu_3D, std::shared_ptr<BornElasticShotsGpu_3D>>(m, "BornElasticShotsGpu_3D")
      .def(py::init([](const float4DReg& ep, std::shared_ptr<paramObj> par, std::vector<float4DReg> sources,
                       std::vector<Interp> s0, std::vector<Interp> s1, std::vector<Interp> s2, std::vector<Interp> s3,
                       std::vector<Interp> s4, std::vector<Interp> s5, std::vector<Interp> s6, std::vector<Interp> r0,
                       std::vector<Interp> r1, std::vector<Interp> r2, std::vector<Interp> r3, std::vector<Interp> r4,
                       std::vector<Interp> r5, std::vector<Interp> r6) {
        return std::make_shared<BornElasticShotsGpu_3D>(
            ep, par, sources, std::vector<std::vector<Interp>>{s0, s1, s2, s3, s4, s5, s6, r0, r1, r2, r3, r4, r5, r6});
      }))
      .def("forward", &BornElasticShotsGpu_3D::forward)
      .def("adjoint", &BornElasticShotsGpu_3D::adjoint)
      .def("setBackground", &BornElasticShotsGpu_3D::setBackground)
      .def("dotTest", [](BornElasticShotsGpu_3D& op, const float4DReg& model, const float4DReg& data, bool verbose,
                         float maxError) {
        return dotTest(op, model.shape(), data.shape(), verbose, maxError, model.getHyper());
      });
}
