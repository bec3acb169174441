// Engine: device memory, time loops and checkpointing of the elastic 3D
// propagation path.  Per-shot loops restate the reference drivers
//   propElasticFwdGpu_3D / propElasticAdjGpu_3D (nonlinearPropElasticGpuFunctions_3D.cu:876-975, :1298-1395)
//   BornElasticFwdGpu_3D / BornElasticAdjGpu_3D (BornElasticGpuFunctions_3D.cu:1226-1461, :2103-2336)
// with three B200 changes: the sponge is fused into the stepper, all signals
// live on the device time-major for coalesced injection/recording, and the
// Born source-side velocity is never sent to host memory (the forward Born
// runs the source propagation two coarse blocks ahead of the scattered one;
// the adjoint Born recomputes it per segment from on-device checkpoints).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>
#include <atomic>
#include <mutex>
#include <unordered_map>

#include "engine.h"
#include "kernels.cuh"
#include "schedule.h"

namespace e3d {

static thread_local std::string g_err;
void setLastError(const char* msg, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s (%s:%d)", msg, file, line);
  g_err = buf;
}
const char* lastError() { return g_err.c_str(); }

#define E3D_ARG(cond, msg)                        \
  do {                                            \
    if (!(cond)) {                                \
      setLastError(msg, __FILE__, __LINE__);      \
      return E3D_ERR_ARG;                         \
    }                                             \
  } while (0)

#define E3D_RET(expr)               \
  do {                              \
    int _s = (expr);                \
    if (_s != E3D_OK) return _s;    \
  } while (0)

#define E3D_LAUNCH_CHECK() E3D_CUDA_TRY(cudaGetLastError())

// ---------------------------------------------------------------------------
struct Fields9 {
  float* p[NCOMP] = {};
};

struct Context {
  ContextDesc d;
  cudaStream_t st = nullptr;     // stream all work is queued on
  cudaStream_t own = nullptr;    // the context's own stream
  GridConst g{};
  float* taper = nullptr;
  int hfilt = 0;
  std::vector<float> filt;  // 2*(sub+1)
  float dtsInv = 0.f;
  float* med[NMED] = {};
  bool haveMedium = false;
  int tx = 8;
  int stages = 3;            // shared-memory pipeline depth of the stepper
  // 0: plain loads, 1: cp.async, 2: TMA bulk tensor copies, 3-5: TMA forms with a rotating
  // y-window, 6: split velocity/stress roles for every mode, 7: split roles for the forward and
  // time-reversed steps, loader 2's two-stage stepper for the exact adjoint, 8 (default): 7 with
  // two z cells per thread (measured on B200 in the 288^3 gradient: steppers 3.5-4 % faster)
  int loader = 8;
  int yChunks = 0;           // y chunks per (z, x) tile column of the stepper grid (0: automatic)
  int numSMs = 148;          // multiprocessors of the device
  int graphLoop = 1;         // 1: replay coarse blocks of the nonlinear loop as a CUDA graph
  bool inCapture = false;    // a coarse block is being captured (no timing samples)
  int* blockIndex = nullptr; // device coarse-time index of replayed blocks
  unsigned* posFlag = nullptr;  // device word of the position-table check
  Fields9 bw0, bw1;          // batched nonlinear forward: the shots' levels, stacked per field
  int batchShots = 0;
  std::unordered_map<unsigned long long, CUtensorMap> tmaps;  // (pointer, box) -> tensor map
  std::vector<void*> owned;  // every device allocation of this context
  // working wavefields (primary propagation)
  Fields9 w0, w1;
  // Born / FWI buffers, allocated on first use
  Fields9 s0, s1;            // source-side state
  std::vector<float*> vSlots;  // decimated source velocity slots, FP32 (3 fields each)
  std::vector<void*> vStore;   // FP16 velocity slots with per-(field, y-slice) scales
  int vType = -1;              // velocity slot storage requested: -1 auto, 0 FP32, 1 FP16
  int vUsed = 0;               // storage of the current plan
  float* traceRing = nullptr;  // two regular-grid receiver slices (irregular trace mode)
  size_t traceRingFloats = 0;
  Fields9 ss[2];             // secondary sources (forward) / decimated adjoint field (adjoint)
  Fields9 q0, q1;            // premultiplied adjoint levels (dual-state exact adjoint)
  // Rings of fine time levels for the gradient's passes (empty: decimation
  // accumulators fused into the stepper instead).  Level m lives in
  // lev[m mod size]; the first two entries are the s0/s1 (source) and w0/w1
  // (adjoint) buffers, so those always point into the ring.
  std::vector<Fields9> srcRing, adjRing;
  int ringMode = 1;          // 1: decimate from rings when sub allows it
  int imgChunks = 0;         // y chunks of the y-marching imaging launch (0: automatic)
  int imgVariant = 0;        // block imaging kernel: 0 automatic, 1 kImagingBlock, 2 kImagingTma, 3/4 kImagingLev 8/4 wide
  // exact adjoint state of the ring passes: 1 premultiplied-only where the medium's premultiplication
  // is well conditioned (premCond <= kPremCondMax), 0 always the dual raw + premultiplied state
  int premMode = 1;
  double premCond = -1.0;    // condition number of the current medium's premultiplication (-1: unknown)
  float* pertDev[NMED] = {};
  // checkpoints
  int ckptType = CKPT_AUTO;
  int ckptUsed = CKPT_F32;     // storage type of the current checkpoints
  int vAllocType = -1;         // velocity slot storage currently allocated
  int segment = 0;           // coarse blocks per segment (0 = automatic)
  double budget = 0;         // bytes available for checkpoints + velocity slots (0 = automatic)
  std::vector<void*> ckpt;   // one per segment (index = segment id), packed 18-field states
  std::vector<float*> ckptScale;
  int ckptSegLen = 0;
  int ckptAllocType = -1;
  bool ckptValid = false;
  bool tailValid = false;    // the last segment's velocity slots were filled by the forward pass
  // scratch for transposes / signal staging
  void* scratch = nullptr;
  size_t scratchBytes = 0;
  // launch accounting and sampled stepper timing
  long long launches = 0;
  int timingEvery = 0;       // 0: off; n: time every n-th stepper launch
  long long kindCounter[8] = {};
  std::vector<cudaEvent_t> evPool;
  struct Timed { int mode; cudaEvent_t a, b; };
  std::vector<Timed> timed;
};

static int devAlloc(Context* c, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMallocAsync(p, bytes, c->st);
  if (e != cudaSuccess) {
    setLastError(cudaGetErrorString(e), __FILE__, __LINE__);
    return e == cudaErrorMemoryAllocation ? E3D_ERR_OOM : E3D_ERR_CUDA;
  }
  c->owned.push_back(*p);
  return E3D_OK;
}

static void devFree(Context* c, void* p) {
  if (!p) return;
  auto it = std::find(c->owned.begin(), c->owned.end(), p);
  if (it != c->owned.end()) c->owned.erase(it);
  cudaFreeAsync(p, c->st);
}

static int allocFields(Context* c, Fields9& f, bool zero) {
  const size_t bytes = (size_t)c->g.n * sizeof(float);
  for (int k = 0; k < NCOMP; k++) {
    if (!f.p[k]) E3D_RET(devAlloc(c, (void**)&f.p[k], bytes));
    if (zero) E3D_CUDA_TRY(cudaMemsetAsync(f.p[k], 0, bytes, c->st));
  }
  return E3D_OK;
}

static int zeroFields(Context* c, Fields9& f, int ncomp = NCOMP) {
  for (int k = 0; k < ncomp; k++) E3D_CUDA_TRY(cudaMemsetAsync(f.p[k], 0, (size_t)c->g.n * sizeof(float), c->st));
  return E3D_OK;
}

static int scratchAtLeast(Context* c, size_t bytes) {
  if (c->scratchBytes >= bytes) return E3D_OK;
  devFree(c, c->scratch);
  c->scratch = nullptr;
  c->scratchBytes = 0;
  E3D_RET(devAlloc(c, &c->scratch, bytes));
  c->scratchBytes = bytes;
  return E3D_OK;
}

// ---------------------------------------------------------------------------
int createContext(const ContextDesc& d, Context** out) {
  E3D_ARG(out != nullptr, "null output handle");
  E3D_ARG(d.nz > 2 * FAT && d.nx > 2 * FAT && d.ny > 2 * FAT, "grid must exceed 2*FAT on every axis");
  E3D_ARG(d.nts >= 3, "nts must be at least 3");
  E3D_ARG(d.sub >= 1 && d.sub < SUB_MAX, "sub must be in [1, SUB_MAX)");
  E3D_ARG(d.minPad >= 0 && d.minPad < PAD_MAX, "minPad must be in [0, PAD_MAX)");
  E3D_ARG(d.dz > 0 && d.dx > 0 && d.dy > 0 && d.dts > 0, "sampling must be positive");
  E3D_ARG((long long)d.nz * d.nx * d.ny < (1LL << 40), "grid too large");
  E3D_ARG(!d.freeSurface || d.nz >= 3 * FAT + 2, "the free surface needs nz >= 3*FAT+2");
  Context* c = new Context();
  c->d = d;
  cudaError_t e = cudaSetDevice(d.device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
  c->st = c->own;
  if (e != cudaSuccess) {
    setLastError(cudaGetErrorString(e), __FILE__, __LINE__);
    delete c;
    return E3D_ERR_CUDA;
  }
  {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d.device) == cudaSuccess && sms > 0)
      c->numSMs = sms;
  }
  GridConst& g = c->g;
  g.nz = d.nz; g.nx = d.nx; g.ny = d.ny; g.minPad = d.minPad;
  g.yOff = 0; g.nyTaper = d.ny;
  g.freeSurface = d.freeSurface ? 1 : 0;
  g.yStride = (long long)d.nz * d.nx;
  g.n = g.yStride * d.ny;
  // FD coefficients (nonlinearPropElasticGpuFunctions_3D.cu:207-220): double
  // quotients stored as float; y uses dx unless fixQ1 (quirk Q1).
  const double k[4] = {1.196289062541883, -0.079752604188901, 0.009570312506634, -6.975446437140719e-04};
  for (int i = 0; i < 4; i++) {
    g.cz[i] = (float)(k[i] / d.dz);
    g.cx[i] = (float)(k[i] / d.dx);
    g.cy[i] = (float)(k[i] / (d.fixQ1 ? d.dy : d.dx));
  }
  // time-interpolation filter (nonlinearPropElasticGpuFunctions_3D.cu:223-241)
  const int ntw = (d.nts - 1) * d.sub + 1;
  c->hfilt = d.sub + 1;
  c->filt.assign(2 * c->hfilt, 0.f);
  const double scale = 1.0 / std::sqrt((float)ntw / (float)d.nts);
  for (int i = 0; i < c->hfilt; i++) {
    float left = (float)(1.0 - 1.0 * i / d.sub);
    float right = (float)(1.0 - left);
    c->filt[i] = (float)(left * scale);
    c->filt[i + c->hfilt] = (float)(right * scale);
  }
  // cosine taper (nonlinearPropElasticGpuFunctions_3D.cu:243-255)
  std::vector<float> taper(std::max(d.minPad, 1), 1.f);
  for (int i = 0; i < d.minPad; i++) {
    float arg = (float)(M_PI / (1.0 * d.minPad) * 1.0 * (d.minPad - i));
    taper[i] = (float)(d.alphaCos + (1.0 - d.alphaCos) * std::cos(arg));
  }
  c->dtsInv = (float)(1.0 / (2.0 * d.dts));
  int s = devAlloc(c, (void**)&c->taper, taper.size() * sizeof(float));
  if (s == E3D_OK) {
    e = cudaMemcpyAsync(c->taper, taper.data(), taper.size() * sizeof(float), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) {
      setLastError(cudaGetErrorString(e), __FILE__, __LINE__);
      s = E3D_ERR_CUDA;
    }
  }
  if (s != E3D_OK) {
    destroyContext(c);
    return s;
  }
  g.taper = c->taper;
  *out = c;
  return E3D_OK;
}

void destroyContext(Context* c) {
  if (!c) return;
  cudaSetDevice(c->d.device);
  for (auto& t : c->timed) {
    c->evPool.push_back(t.a);
    c->evPool.push_back(t.b);
  }
  for (cudaEvent_t e : c->evPool) cudaEventDestroy(e);
  for (void* p : c->owned) cudaFreeAsync(p, c->st);
  c->owned.clear();
  if (c->st) cudaStreamSynchronize(c->st);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
}

cudaStream_t stream(Context* c) { return c->st; }
int setStream(Context* c, cudaStream_t s, bool useOwn) {
  E3D_ARG(c != nullptr, "null context");
  if (c->st == (useOwn ? c->own : s)) return E3D_OK;
  E3D_CUDA_TRY(cudaStreamSynchronize(c->st));
  c->st = useOwn ? c->own : s;
  return E3D_OK;
}
long long cellsPerStep(const Context* c) {
  return (long long)(c->d.nz - 2 * FAT) * (c->d.nx - 2 * FAT) * (c->d.ny - 2 * FAT);
}
double deviceBytesInUse(const Context* c) {
  size_t free = 0, total = 0;
  cudaMemGetInfo(&free, &total);
  return (double)(total - free);
}

int setMedium(Context* c, const float* const* planes, bool onDevice) {
  E3D_ARG(c && planes, "null argument");
  E3D_CUDA_TRY(cudaSetDevice(c->d.device));
  const size_t bytes = (size_t)c->g.n * sizeof(float);
  for (int k = 0; k < NMED; k++) {
    E3D_ARG(planes[k] != nullptr, "null medium plane");
    if (!c->med[k]) E3D_RET(devAlloc(c, (void**)&c->med[k], bytes));
    E3D_CUDA_TRY(cudaMemcpyAsync(c->med[k], planes[k], bytes, onDevice ? cudaMemcpyDeviceToDevice
                                                                        : cudaMemcpyHostToDevice, c->st));
  }
  E3D_CUDA_TRY(cudaStreamSynchronize(c->st));
  c->haveMedium = true;
  c->ckptValid = false;
  c->tailValid = false;
  c->premCond = -1.0;
  return E3D_OK;
}

int setStepperVariant(Context* c, int tx, int stages, int loader) {
  E3D_ARG(c && (tx == 8 || tx == 16), "tile width must be 8 or 16");
  E3D_ARG(loader >= 0 && loader <= 8, "loader must be 0 (plain), 1 (cp.async), 2-5 (TMA forms), 6-8 (split TMA)");
  E3D_ARG(stages == 2 || stages == 3 || (loader >= 6 && stages == 4),
          "pipeline depth must be 2 or 3 (4 with the split stepper)");
  E3D_ARG(!(tx == 16 && stages == 3), "16-wide tiles fit two stages at most");
  E3D_ARG(loader < 6 || tx == 8, "the split stepper uses 8-wide tiles");
  c->tx = tx;
  c->stages = stages;
  c->loader = loader;
  return E3D_OK;
}

int setImagingChunks(Context* c, int chunks) {
  E3D_ARG(c && chunks >= 0, "bad chunk count");
  c->imgChunks = chunks;
  return E3D_OK;
}

int setImagingVariant(Context* c, int variant) {
  E3D_ARG(c != nullptr, "null context");
  E3D_ARG(variant >= 0 && variant <= 4, "imaging variant must be 0 (automatic), 1, 2, 3 or 4");
  c->imgVariant = variant;
  return E3D_OK;
}

int setStepperChunks(Context* c, int chunks) {
  E3D_ARG(c && chunks >= 0, "chunk count must be >= 0");
  c->yChunks = chunks;
  return E3D_OK;
}

int checkPipeError(Context* c) {
  unsigned flag = 0;
  E3D_CUDA_TRY(cudaMemcpyFromSymbolAsync(&flag, g_e3dPipeError, sizeof(flag), 0, cudaMemcpyDeviceToHost, c->st));
  E3D_CUDA_TRY(cudaStreamSynchronize(c->st));
  if (flag) {
    const unsigned zero = 0;
    cudaMemcpyToSymbolAsync(g_e3dPipeError, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, c->st);
    cudaStreamSynchronize(c->st);
    setLastError("stepper pipeline wait expired (bulk copies did not complete)", __FILE__, __LINE__);
    return E3D_ERR_CUDA;
  }
  return E3D_OK;
}

int setCheckpointPolicy(Context* c, int type, int segment, double budget) {
  E3D_ARG(c && type >= CKPT_AUTO && type <= CKPT_BF16, "bad checkpoint type");
  E3D_ARG(segment >= 0, "segment length must be >= 0");
  c->ckptType = type;
  c->segment = segment;
  c->budget = budget;
  c->ckptValid = false;
  c->tailValid = false;
  return E3D_OK;
}

// ---------------------------------------------------------------------------
// Launch helpers
// ---------------------------------------------------------------------------
static StepPtrs makeStep(Context* c, Fields9& o, const Fields9& cur) {
  StepPtrs p{};
  for (int k = 0; k < NCOMP; k++) {
    p.o[k] = o.p[k];
    p.c[k] = cur.p[k];
  }
  for (int k = 0; k < NMED; k++) p.m[k] = c->med[k];
  return p;
}

// A step that writes its new level into `nw` (a ring slot) instead of over the old level.
static StepPtrs makeRingStep(Context* c, Fields9& o, const Fields9& cur, Fields9& nw) {
  StepPtrs p = makeStep(c, o, cur);
  for (int k = 0; k < NCOMP; k++) p.nw[k] = nw.p[k];
  return p;
}

// The pointers the post-step kernels (injection, recording, refresh, source
// extraction) act on: the new level as their "o".
static StepPtrs afterStep(const StepPtrs& p) {
  StepPtrs q = p;
  if (p.nw[0])
    for (int k = 0; k < NCOMP; k++) {
      q.o[k] = p.nw[k];
      q.nw[k] = nullptr;
    }
  return q;
}

// Opt a kernel into its dynamic shared memory once per device (function
// attributes are per device; several GPUs may be driven from one process).
static int ensureSmemAttr(const void* fn, size_t smem, std::atomic<unsigned long long>& doneMask) {
  int dev = 0;
  E3D_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long bit = 1ULL << (dev & 63);
  if (doneMask.load() & bit) return E3D_OK;
  E3D_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  doneMask.fetch_or(bit);
  return E3D_OK;
}

template <int MODE, int TX, int STAGES>
static int launchPipe(Context* c, const StepPtrs& p, dim3 grid, int yChunk) {
  constexpr size_t smem = (size_t)STAGES * PipeLayout<TX>::STAGE_F * sizeof(float);
  static std::atomic<unsigned long long> configured{0};
  E3D_RET(ensureSmemAttr((const void*)kStepPipe<MODE, TX, STAGES>, smem, configured));
  kStepPipe<MODE, TX, STAGES><<<grid, dim3(TZ, TX), smem, c->st>>>(p, c->g, yChunk);
  return E3D_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link dependency)
static PFN_cuTensorMapEncodeTiled_v12000 tmaEncoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)f;
  }
  return fn;
}

// 3D map over a (nz, nx, ny) float field with a boxZ x boxX x 1 box, zero fill outside; with
// shots > 0 a 4D (nz, nx, ny, shots) map over that many fields stacked at stride n.
static int tensorMap(Context* c, const float* ptr, int boxZ, int boxX, const CUtensorMap** out, int shots = 0) {
  const unsigned long long key = (reinterpret_cast<unsigned long long>(ptr) << 8) ^
                                 (unsigned long long)(boxZ * 64 + boxX) ^ ((unsigned long long)shots << 52);
  auto it = c->tmaps.find(key);
  if (it != c->tmaps.end()) {
    *out = &it->second;
    return E3D_OK;
  }
  auto enc = tmaEncoder();
  E3D_ARG(enc != nullptr, "cuTensorMapEncodeTiled unavailable");
  E3D_ARG((reinterpret_cast<unsigned long long>(ptr) & 15) == 0, "field not 16-byte aligned");
  CUtensorMap m;
  cuuint64_t dims[4] = {(cuuint64_t)c->d.nz, (cuuint64_t)c->d.nx, (cuuint64_t)c->d.ny, (cuuint64_t)std::max(shots, 1)};
  cuuint64_t strides[3] = {(cuuint64_t)c->d.nz * 4, (cuuint64_t)c->g.yStride * 4, (cuuint64_t)c->g.n * 4};
  cuuint32_t box[4] = {(cuuint32_t)boxZ, (cuuint32_t)boxX, 1, 1};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, shots > 0 ? 4 : 3, const_cast<float*>(ptr), dims, strides,
                   box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    setLastError("cuTensorMapEncodeTiled failed", __FILE__, __LINE__);
    return E3D_ERR_CUDA;
  }
  auto ins = c->tmaps.emplace(key, m);
  *out = &ins.first->second;
  return E3D_OK;
}

template <int TX>
static int buildMaps(Context* c, const StepPtrs& p, TmaMaps& mp) {
  const CUtensorMap* m = nullptr;
  const float* tileSrc[NTILE] = {p.c[VX], p.c[VY], p.c[VZ], p.c[SXX], p.c[SZZ], p.c[SXY], p.c[SXZ], p.c[SYZ]};
  const float* leadSrc[NQUEUE] = {p.c[VX], p.c[VY], p.c[VZ], p.c[SYY], p.c[SXY], p.c[SYZ]};
  for (int t = 0; t < NTILE; t++) {
    E3D_RET(tensorMap(c, tileSrc[t], SZ, TX + 2 * HALO, &m));
    mp.halo[t] = *m;
  }
  for (int q = 0; q < NQUEUE; q++) {
    E3D_RET(tensorMap(c, leadSrc[q], TZ, TX, &m));
    mp.lead[q] = *m;
  }
  for (int k = 0; k < NCOMP; k++) {
    E3D_RET(tensorMap(c, p.o[k], TZ, TX, &m));
    mp.old[k] = *m;
  }
  for (int k = 0; k < NMED; k++) {
    E3D_RET(tensorMap(c, p.m[k], TZ, TX, &m));
    mp.med[k] = *m;
  }
  return E3D_OK;
}

template <int MODE, int TX, int STAGES>
static int launchTma(Context* c, const StepPtrs& p, dim3 grid, int yChunk) {
  constexpr size_t smem = (size_t)STAGES * PipeLayout<TX>::STAGE_F * sizeof(float);
  static std::atomic<unsigned long long> configured{0};
  E3D_RET(ensureSmemAttr((const void*)kStepTma<MODE, TX, STAGES>, smem, configured));
  TmaMaps mp;
  E3D_RET(buildMaps<TX>(c, p, mp));
  kStepTma<MODE, TX, STAGES><<<grid, dim3(TZ, TX), smem, c->st>>>(mp, p, c->g, yChunk);
  return E3D_OK;
}

static int chooseChunks(const Context* c, long long tiles, int nyi, int perSM = 2);

// Split stepper: role V maps (stress halos and leads, old velocities, rho planes) and role S maps
// (velocity halos and leads, old stresses, lambda/mu planes).  shots > 0: the field maps cover
// that many shots stacked per field (4D); the medium maps stay 3D.
static int buildSplitMaps(Context* c, const StepPtrs& p, SplitMaps& mp, int shots = 0) {
  const CUtensorMap* m = nullptr;
  const int vHalo[5] = {SXX, SXY, SXZ, SYZ, SZZ}, vLead[3] = {SXY, SYY, SYZ};
  int i = 0;
  for (int f : vHalo) { E3D_RET(tensorMap(c, p.c[f], SZ, 8 + 2 * HALO, &m, shots)); mp.v[i++] = *m; }
  for (int f : vLead) { E3D_RET(tensorMap(c, p.c[f], TZ, 8, &m, shots)); mp.v[i++] = *m; }
  for (int k = VX; k <= VZ; k++) { E3D_RET(tensorMap(c, p.o[k], TZ, 8, &m, shots)); mp.v[i++] = *m; }
  for (int k = RHOX; k <= RHOZ; k++) { E3D_RET(tensorMap(c, p.m[k], TZ, 8, &m)); mp.v[i++] = *m; }
  i = 0;
  for (int f = VX; f <= VZ; f++) { E3D_RET(tensorMap(c, p.c[f], SZ, 8 + 2 * HALO, &m, shots)); mp.s[i++] = *m; }
  for (int f = VX; f <= VZ; f++) { E3D_RET(tensorMap(c, p.c[f], TZ, 8, &m, shots)); mp.s[i++] = *m; }
  for (int k = SXX; k <= SYZ; k++) { E3D_RET(tensorMap(c, p.o[k], TZ, 8, &m, shots)); mp.s[i++] = *m; }
  for (int k = L2M; k <= MUYZ; k++) { E3D_RET(tensorMap(c, p.m[k], TZ, 8, &m)); mp.s[i++] = *m; }
  return E3D_OK;
}

template <int MODE, int STAGES, int MINB>
static int launchSplit(Context* c, const StepPtrs& p, int tiz, int tix, int nyi) {
  constexpr size_t smem = (size_t)STAGES * SPL_STAGE_F * sizeof(float);
  static std::atomic<unsigned long long> configured{0};
  E3D_RET(ensureSmemAttr((const void*)kStepSplit<MODE, STAGES, MINB>, smem, configured));
  SplitMaps mp;
  E3D_RET(buildSplitMaps(c, p, mp));
  // y runs measured best on B200 (392^3 and 288^3 grids, 3 stages): about 32 planes for the
  // forward and time-reversed steps (0.84-0.85 of the copy bandwidth), about 10 for the
  // dual-state exact adjoint (0.78-0.79; 0.59-0.64 with one long run)
  int chunks = c->yChunks > 0 ? std::min(c->yChunks, nyi) : (nyi + (MODE == STEP_ADJ_EXACT ? 9 : 31)) /
                                                                (MODE == STEP_ADJ_EXACT ? 10 : 32);
  chunks = std::max(chunks, 1);
  const int yChunk = (nyi + chunks - 1) / chunks;
  chunks = (nyi + yChunk - 1) / yChunk;
  kStepSplit<MODE, STAGES, MINB><<<dim3(tiz, tix, 2 * chunks), dim3(TZ, 8), smem, c->st>>>(mp, p, c->g, yChunk,
                                                                                              chunks, 1, 0);
  return E3D_OK;
}

// One step of `shots` shots stacked per field (fields of n*shots floats), 3-stage split stepper.
template <int MODE>
static int launchSplitBatch(Context* c, const StepPtrs& p, int shots) {
  constexpr size_t smem = (size_t)3 * SPL_STAGE_F * sizeof(float);
  static std::atomic<unsigned long long> configured{0};
  E3D_RET(ensureSmemAttr((const void*)kStepSplit<MODE, 3, 3, true>, smem, configured));
  SplitMaps mp;
  E3D_RET(buildSplitMaps(c, p, mp, shots));
  const GridConst& g = c->g;
  const int tiz = (g.nz - 2 * FAT + TZ - 1) / TZ;
  const int tix = (g.nx - 2 * FAT + 7) / 8;
  const int nyi = g.ny - 2 * FAT;
  int chunks = c->yChunks > 0 ? std::min(c->yChunks, nyi) : (nyi + 31) / 32;
  chunks = std::max(chunks, 1);
  const int yChunk = (nyi + chunks - 1) / chunks;
  chunks = (nyi + yChunk - 1) / yChunk;
  kStepSplit<MODE, 3, 3, true><<<dim3(tiz * shots, tix, 2 * chunks), dim3(TZ, 8), smem, c->st>>>(
      mp, p, c->g, yChunk, chunks, shots, g.n);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

// Paired split stepper (two z cells per thread, blockDim TZ/2 x 8): the y runs of launchSplit.
template <int MODE, int STAGES, int MINB>
static int launchSplitPair(Context* c, const StepPtrs& p, int tiz, int tix, int nyi) {
  constexpr size_t smem = (size_t)STAGES * SPL_STAGE_F * sizeof(float);
  static std::atomic<unsigned long long> configured{0};
  E3D_RET(ensureSmemAttr((const void*)kStepSplitPair<MODE, STAGES, MINB>, smem, configured));
  SplitMaps mp;
  E3D_RET(buildSplitMaps(c, p, mp));
  int chunks = c->yChunks > 0 ? std::min(c->yChunks, nyi) : (nyi + 31) / 32;
  chunks = std::max(chunks, 1);
  const int yChunk = (nyi + chunks - 1) / chunks;
  chunks = (nyi + yChunk - 1) / yChunk;
  kStepSplitPair<MODE, STAGES, MINB><<<dim3(tiz, tix, 2 * chunks), dim3(TZ / 2, 8), smem, c->st>>>(mp, p, c->g,
                                                                                                   yChunk, chunks);
  return E3D_OK;
}

template <int MODE>
static int launchSplitPairVariant(Context* c, const StepPtrs& p, int tiz, int tix, int nyi) {
  if (c->stages == 4) return launchSplitPair<MODE, 4, 2>(c, p, tiz, tix, nyi);
  if (c->stages == 2) return launchSplitPair<MODE, 2, 4>(c, p, tiz, tix, nyi);
  return launchSplitPair<MODE, 3, 3>(c, p, tiz, tix, nyi);
}

template <int MODE>
static int launchSplitVariant(Context* c, const StepPtrs& p, int tiz, int tix, int nyi) {
  if (c->stages == 4) return launchSplit<MODE, 4, 2>(c, p, tiz, tix, nyi);
  if (c->stages == 2) return launchSplit<MODE, 2, 3>(c, p, tiz, tix, nyi);
  return launchSplit<MODE, 3, 3>(c, p, tiz, tix, nyi);
}

template <int MODE, int TX, int STAGES, bool OM_SMEM, int MINB>
static int launchTma2(Context* c, const StepPtrs& p, dim3 grid, int yChunk) {
  constexpr size_t smem = (size_t)STAGES * Tma2Layout<TX, OM_SMEM>::STAGE_F * sizeof(float);
  static std::atomic<unsigned long long> configured{0};
  E3D_RET(ensureSmemAttr((const void*)kStepTma2<MODE, TX, STAGES, OM_SMEM, MINB>, smem, configured));
  TmaMaps mp;
  E3D_RET(buildMaps<TX>(c, p, mp));
  kStepTma2<MODE, TX, STAGES, OM_SMEM, MINB><<<grid, dim3(TZ, TX), smem, c->st>>>(mp, p, c->g, yChunk);
  return E3D_OK;
}

template <int MODE>
static int launchVariant(Context* c, const StepPtrs& p, dim3 grid, int yChunk) {
  const int key = c->tx * 10 + c->stages;
  if (c->loader == 3) {  // rotating window, old level and medium in shared memory
    switch (key) {
      case 82: return launchTma2<MODE, 8, 2, true, 2>(c, p, grid, yChunk);
      case 83: return launchTma2<MODE, 8, 3, true, 1>(c, p, grid, yChunk);
      default: return launchTma2<MODE, 16, 2, true, 1>(c, p, grid, yChunk);
    }
  }
  if (c->loader == 4) {  // rotating window, old level and medium by plain loads, 3 CTAs/SM
    switch (key) {
      case 82: return launchTma2<MODE, 8, 2, false, 3>(c, p, grid, yChunk);
      case 83: return launchTma2<MODE, 8, 3, false, 3>(c, p, grid, yChunk);
      default: return launchTma2<MODE, 16, 2, false, 1>(c, p, grid, yChunk);
    }
  }
  if (c->loader == 5) {  // as 4 with the register budget of 2 CTAs/SM
    switch (key) {
      case 82: return launchTma2<MODE, 8, 2, false, 2>(c, p, grid, yChunk);
      default: return launchTma2<MODE, 8, 3, false, 2>(c, p, grid, yChunk);
    }
  }
  if (c->loader >= 6) return launchTma<MODE, 8, 2>(c, p, grid, yChunk);  // split loaders: fused steps
  if (c->loader == 2) {
    switch (key) {
      case 82: return launchTma<MODE, 8, 2>(c, p, grid, yChunk);
      case 83: return launchTma<MODE, 8, 3>(c, p, grid, yChunk);
      default: return launchTma<MODE, 16, 2>(c, p, grid, yChunk);
    }
  }
  switch (key) {
    case 82: return launchPipe<MODE, 8, 2>(c, p, grid, yChunk);
    case 83: return launchPipe<MODE, 8, 3>(c, p, grid, yChunk);
    default: return launchPipe<MODE, 16, 2>(c, p, grid, yChunk);
  }
}

static int launchStepRaw(Context* c, int mode, const StepPtrs& p);

static cudaEvent_t takeEvent(Context* c) {
  if (c->evPool.empty()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
  }
  cudaEvent_t e = c->evPool.back();
  c->evPool.pop_back();
  return e;
}

// Sampled launch timing: with sampling on, every n-th launch of each timed
// kind is bracketed with CUDA events on the launching stream.  Kinds: stepper
// modes 0..2, the same with a fused decimation or secondary source 3..5, the
// block imaging of the decimation ring 6, its velocity decimation 7.
struct TimedLaunch {
  Context* c;
  int kind;
  cudaEvent_t a = nullptr, b = nullptr;
  TimedLaunch(Context* cc, int k) : c(cc), kind(k) {
    if (c->inCapture || c->timingEvery <= 0) return;
    if ((c->kindCounter[kind]++ % c->timingEvery) != 0) return;
    a = takeEvent(c);
    b = takeEvent(c);
    if (a && b) cudaEventRecord(a, c->st);
  }
  ~TimedLaunch() {
    if (!(a && b)) {
      if (a) c->evPool.push_back(a);
      if (b) c->evPool.push_back(b);
      return;
    }
    cudaEventRecord(b, c->st);
    c->timed.push_back({kind, a, b});
  }
};

// Every stepper launch goes through here: counts it and samples its time.
static int launchStep(Context* c, int mode, const StepPtrs& p) {
  c->launches++;
  // launches that also fuse a decimation or a secondary source are kept apart (mode + 3)
  const bool fused = p.accL[0] != nullptr || p.ssL[0] != nullptr;
  TimedLaunch t(c, mode + (fused ? 3 : 0));
  return launchStepRaw(c, mode, p);
}

int setKernelTiming(Context* c, int every) {
  E3D_ARG(c && every >= 0, "bad timing interval");
  c->timingEvery = every;
  for (auto& k : c->kindCounter) k = 0;
  return E3D_OK;
}

int readKernelTiming(Context* c, int mode, double* avgMs, long long* count) {
  E3D_ARG(c && avgMs && count, "null argument");
  E3D_ARG(mode >= 0 && mode < 8, "bad timed kind");
  double sum = 0;
  long long n = 0;
  std::vector<Context::Timed> keep;
  for (auto& t : c->timed) {
    if (t.mode != mode) {
      keep.push_back(t);
      continue;
    }
    float ms = 0;
    E3D_CUDA_TRY(cudaEventSynchronize(t.b));
    E3D_CUDA_TRY(cudaEventElapsedTime(&ms, t.a, t.b));
    sum += ms;
    n++;
    c->evPool.push_back(t.a);
    c->evPool.push_back(t.b);
  }
  c->timed.swap(keep);
  *avgMs = n ? sum / n : 0.0;
  *count = n;
  return E3D_OK;
}

long long launchCount(const Context* c) { return c->launches; }

// y chunks of a y-marching launch over `tiles` (z, x) tile columns: the CTAs
// run in waves of perSM per SM, and each CTA pays about two planes of pipeline
// start-up, so pick the chunk count (y runs of at least 24 planes) that
// minimises waves * (planes per CTA + 2).
static int chooseChunks(const Context* c, long long tiles, int nyi, int perSM) {
  int chunks = 1;
  const long long slots = (long long)perSM * c->numSMs;
  long long bestCost = -1;
  for (int ch = 1; ch <= std::max(1, nyi / 24); ch++) {
    const long long waves = (tiles * ch + slots - 1) / slots;
    const long long cost = waves * ((nyi + ch - 1) / ch + 2);
    if (bestCost < 0 || cost < bestCost) {
      bestCost = cost;
      chunks = ch;
    }
  }
  return chunks;
}

static int launchStepRaw(Context* c, int mode, const StepPtrs& p) {
  const GridConst& g = c->g;
  const int tiz = (g.nz - 2 * FAT + TZ - 1) / TZ;
  const int tix = (g.nx - 2 * FAT + c->tx - 1) / c->tx;
  const int nyi = g.ny - 2 * FAT;
  // enough CTAs for several waves over 148 SMs, chunks of at least 32 planes
  const long long tiles = (long long)tiz * tix;
  // y chunks (chooseChunks).  Measured on B200: at 288^3 this takes the forward
  // from 0.54 to 0.67 of the copy bandwidth (10 chunks instead of 2); at 392^3
  // it keeps the long runs.
  int chunks = chooseChunks(c, tiles, nyi);
  const bool dual = mode == STEP_ADJ_EXACT && p.oP[0] != nullptr;
  // the split stepper (loader 6; loader 7: all but the exact adjoint, which keeps kStepTma; loader
  // 8: loader 7 with two z cells per thread) takes every step without a fused decimation or
  // secondary source
  if (c->loader == 8 && mode != STEP_ADJ_EXACT && g.nz % 4 == 0 && p.accL[0] == nullptr && p.ssL[0] == nullptr) {
    const int tixS = (g.nx - 2 * FAT + 7) / 8;
    if (mode == STEP_FWD) E3D_RET(launchSplitPairVariant<STEP_FWD>(c, p, tiz, tixS, nyi));
    else E3D_RET(launchSplitPairVariant<STEP_ADJ_REVERSED>(c, p, tiz, tixS, nyi));
    E3D_LAUNCH_CHECK();
    return E3D_OK;
  }
  if ((c->loader == 6 || (c->loader == 7 && mode != STEP_ADJ_EXACT)) && g.nz % 4 == 0 && p.accL[0] == nullptr &&
      p.ssL[0] == nullptr) {
    const int tixS = (g.nx - 2 * FAT + 7) / 8;
    if (mode == STEP_FWD) E3D_RET(launchSplitVariant<STEP_FWD>(c, p, tiz, tixS, nyi));
    else if (mode == STEP_ADJ_REVERSED) E3D_RET(launchSplitVariant<STEP_ADJ_REVERSED>(c, p, tiz, tixS, nyi));
    else E3D_RET(launchSplitVariant<STEP_ADJ_EXACT>(c, p, tiz, tixS, nyi));
    E3D_LAUNCH_CHECK();
    return E3D_OK;
  }
  // The dual-state adjoint runs faster on short y runs: measured on B200 at
  // 392x392x388, about 16 planes per CTA with the 9-field decimation fused
  // (0.64 -> 0.75 of the copy bandwidth) and about 32 without it; the other
  // steps prefer the long runs above.
  if (dual) chunks = std::max(chunks, (nyi + (p.accL[0] ? 15 : 31)) / (p.accL[0] ? 16 : 32));
  if (c->yChunks > 0) chunks = std::min(c->yChunks, nyi);
  chunks = std::max(chunks, 1);
  const int yChunk = (nyi + chunks - 1) / chunks;
  chunks = (nyi + yChunk - 1) / yChunk;
  dim3 grid(tiz, tix, chunks);
  const bool pipe = (g.nz % 4 == 0) && mode != STEP_ADJ_EXACT && c->loader > 0;
  if (dual) {
    E3D_ARG(g.nz % 4 == 0, "dual-state adjoint needs nz % 4 == 0");
    if (c->tx == 16) E3D_RET((launchTma<STEP_ADJ_EXACT, 16, 2>(c, p, grid, yChunk)));
    else if (c->stages == 3 && c->loader < 6) E3D_RET((launchTma<STEP_ADJ_EXACT, 8, 3>(c, p, grid, yChunk)));
    else E3D_RET((launchTma<STEP_ADJ_EXACT, 8, 2>(c, p, grid, yChunk)));
  } else if (pipe) {
    if (mode == STEP_FWD) E3D_RET(launchVariant<STEP_FWD>(c, p, grid, yChunk));
    else E3D_RET(launchVariant<STEP_ADJ_REVERSED>(c, p, grid, yChunk));
  } else if (c->tx == 16) {
    dim3 block(TZ, 16);
    if (mode == STEP_FWD) kStep<STEP_FWD, 16><<<grid, block, 0, c->st>>>(p, g, yChunk);
    else if (mode == STEP_ADJ_REVERSED) kStep<STEP_ADJ_REVERSED, 16><<<grid, block, 0, c->st>>>(p, g, yChunk);
    else kStep<STEP_ADJ_EXACT, 16><<<grid, block, 0, c->st>>>(p, g, yChunk);
  } else {
    dim3 block(TZ, 8);
    if (mode == STEP_FWD) kStep<STEP_FWD, 8><<<grid, block, 0, c->st>>>(p, g, yChunk);
    else if (mode == STEP_ADJ_REVERSED) kStep<STEP_ADJ_REVERSED, 8><<<grid, block, 0, c->st>>>(p, g, yChunk);
    else kStep<STEP_ADJ_EXACT, 8><<<grid, block, 0, c->st>>>(p, g, yChunk);
  }
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

// Injection of time slices sigL (its) and sigR (its+1), filter weights k.
static int launchInjectSlices(Context* c, const StepPtrs& p, const DevSignals& s, const float* sigL,
                              const float* sigR, int k) {
  SparseSet ss;
  ss.pos = s.pos;
  for (int i = 0; i <= NCOMP; i++) ss.off[i] = s.off[i];
  const int n = s.off[NCOMP];
  if (n == 0) return E3D_OK;
  c->launches++;
  kInject<<<(n + 127) / 128, 128, 0, c->st>>>(p, c->g, ss, sigL, sigR, c->filt[k], c->filt[c->hfilt + k]);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

// Injection from a time-major [nts][ntot] signal array at coarse time its.
static int launchInject(Context* c, const StepPtrs& p, const DevSignals& s, const float* sig, int its, int k) {
  const size_t ntot = (size_t)s.off[NCOMP];
  return launchInjectSlices(c, p, s, sig + (size_t)its * ntot, sig + (size_t)(its + 1) * ntot, k);
}

static int launchRecordSlices(Context* c, const StepPtrs& p, const DevSignals& s, float* outL, float* outR, int k) {
  SparseSet ss;
  ss.pos = s.pos;
  for (int i = 0; i <= NCOMP; i++) ss.off[i] = s.off[i];
  const int n = s.off[NCOMP];
  if (n == 0) return E3D_OK;
  c->launches++;
  kRecord<<<(n + 127) / 128, 128, 0, c->st>>>(p, ss, outL, outR, c->filt[k], c->filt[c->hfilt + k]);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

static int launchRecord(Context* c, const StepPtrs& p, const DevSignals& s, float* out, int its, int k) {
  const size_t ntot = (size_t)s.off[NCOMP];
  return launchRecordSlices(c, p, s, out + (size_t)its * ntot, out + (size_t)(its + 1) * ntot, k);
}

static int launchExtractSource(Context* c, const StepPtrs& p, const DevSignals& s, float* out, int its, int k) {
  SparseSet ss;
  ss.pos = s.pos;
  for (int i = 0; i <= NCOMP; i++) ss.off[i] = s.off[i];
  const int n = s.off[NCOMP];
  if (n == 0) return E3D_OK;
  const size_t ntot = (size_t)n;
  c->launches++;
  kExtractSource<<<(n + 127) / 128, 128, 0, c->st>>>(p, c->g, ss, out + (size_t)its * ntot,
                                                     out + (size_t)(its + 1) * ntot, c->filt[k],
                                                     c->filt[c->hfilt + k]);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

static int launchRefresh(Context* c, const StepPtrs& p, const DevSignals& s);

// Receiver injection into the premultiplied-only state (slices its, its+1, filter weights k);
// the three normal-stress tables must have equal counts (the caller checks).
static int launchInjectPremultiplied(Context* c, const StepPtrs& p, const DevSignals& s, const float* sigL,
                                     const float* sigR, int k) {
  SparseSet ss;
  ss.pos = s.pos;
  for (int i = 0; i <= NCOMP; i++) ss.off[i] = s.off[i];
  const int n = s.off[NCOMP];
  if (n == 0) return E3D_OK;
  c->launches++;
  kInjectPremultiplied<<<(n + 127) / 128, 128, 0, c->st>>>(p, c->g, ss, sigL, sigR, c->filt[k],
                                                          c->filt[c->hfilt + k]);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

// Receiver injection (slices its, its+1, filter weights k) and premultiplied refresh of the dual
// adjoint in one launch when the three normal-stress tables have equal counts (they share the
// center grid); otherwise the two launches.
static int launchInjectRefresh(Context* c, const StepPtrs& p, const DevSignals& s, const float* sigL,
                               const float* sigR, int k) {
  const int nc = s.off[SXX + 1] - s.off[SXX];
  if (p.accL[0] != nullptr || s.off[SYY + 1] - s.off[SYY] != nc || s.off[SZZ + 1] - s.off[SZZ] != nc) {
    E3D_RET(launchInjectSlices(c, p, s, sigL, sigR, k));
    return launchRefresh(c, p, s);
  }
  SparseSet ss;
  ss.pos = s.pos;
  for (int i = 0; i <= NCOMP; i++) ss.off[i] = s.off[i];
  const int n = s.off[NCOMP];
  if (n == 0) return E3D_OK;
  c->launches++;
  kInjectRefresh<<<(n + 127) / 128, 128, 0, c->st>>>(p, c->g, ss, sigL, sigR, c->filt[k], c->filt[c->hfilt + k]);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

static int launchRefresh(Context* c, const StepPtrs& p, const DevSignals& s) {
  SparseSet ss;
  ss.pos = s.pos;
  for (int i = 0; i <= NCOMP; i++) ss.off[i] = s.off[i];
  const int n = s.off[NCOMP];
  if (n == 0) return E3D_OK;
  c->launches++;
  kRefreshPremultiplied<<<(n + 127) / 128, 128, 0, c->st>>>(p, ss);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

// Free-surface conditions on the new level after a step and its injection
// (nonlinear propagation only; sgn +1 forward, -1 time-reversed).
static int launchFreeSurface(Context* c, const StepPtrs& p, float sgn) {
  if (!c->g.freeSurface) return E3D_OK;
  const int nxi = c->d.nx - 2 * FAT, nyi = c->d.ny - 2 * FAT;
  c->launches++;
  kFreeSurface<<<dim3((nxi + 127) / 128, nyi), 128, 0, c->st>>>(p, c->g, sgn);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

static int rejectFreeSurface(const Context* c) {
  if (c->g.freeSurface) {
    setLastError("the free surface is implemented for nonlinear propagation only (no exact adjoint of it yet)",
                 __FILE__, __LINE__);
    return E3D_ERR_ARG;
  }
  return E3D_OK;
}

static void swapF(Fields9& a, Fields9& b) {
  for (int k = 0; k < NCOMP; k++) std::swap(a.p[k], b.p[k]);
}

// transpose a (rows x cols) row-major matrix; one 32x32 tile per CTA over a 1D grid
__global__ void kTranspose(const float* in, float* out, long long rows, long long cols) {
  __shared__ float t[32][33];
  const long long tilesC = (cols + 31) / 32;
  const long long r0 = (long long)(blockIdx.x / tilesC) * 32, c0 = (long long)(blockIdx.x % tilesC) * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const long long r = r0 + j, cc = c0 + threadIdx.x;
    if (r < rows && cc < cols) t[j][threadIdx.x] = in[r * cols + cc];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const long long cc = c0 + j, r = r0 + threadIdx.x;
    if (r < rows && cc < cols) out[cc * rows + r] = t[threadIdx.x][j];
  }
}

static int transpose(Context* c, const float* in, float* out, long long rows, long long cols) {
  if (rows == 0 || cols == 0) return E3D_OK;
  const long long tiles = ((rows + 31) / 32) * ((cols + 31) / 32);
  E3D_ARG(tiles < (1LL << 31), "transpose too large");
  c->launches++;
  kTranspose<<<(unsigned)tiles, dim3(32, 8), 0, c->st>>>(in, out, rows, cols);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

// ---------------------------------------------------------------------------
// Host (reference-layout) <-> device (time-major) signal staging
// ---------------------------------------------------------------------------
struct Staged {
  DevSignals set{};
  long long* pos = nullptr;
  float* sig = nullptr;  // time-major [nts][ntot]
  int ntot = 0;
};

// Component k uses the positions of grid gridOf(k); with q2 the sxz receiver
// table is the z-grid table (nonlinearPropElasticGpuFunctions_3D.cu:416).
static int stageGeom(Context* c, const HostGeom& g, bool receivers, Staged& s) {
  long long tot = 0;
  for (int k = 0; k < NCOMP; k++) {
    const int gi = gridOfComp(k);
    E3D_ARG(g.n[gi] >= 0 && g.n[gi] < (1LL << 30), "bad device count");
    s.set.off[k] = (int)tot;
    tot += g.n[gi];
  }
  E3D_ARG(tot < (1LL << 31), "too many acquisition points");
  s.set.off[NCOMP] = (int)tot;
  s.ntot = (int)tot;
  std::vector<long long> h(std::max<long long>(tot, 1));
  for (int k = 0; k < NCOMP; k++) {
    int gi = gridOfComp(k);
    const long long* src = g.pos[gi];
    if (receivers && k == SXZ && c->d.q2compat) {
      // reference copies nReceiversRegXZGrid entries of the z-grid table
      E3D_ARG(g.n[GXZ] <= g.n[GZ], "sxz receivers read past the z-grid table (reference quirk Q2)");
      src = g.pos[GZ];
    }
    const long long n = g.n[gi];
    E3D_ARG(n == 0 || src != nullptr, "null position table");
    for (long long i = 0; i < n; i++) {
      const long long p = src[i];
      E3D_ARG(p >= 0 && p < c->g.n, "acquisition point outside the grid");
      const long long iz = p % c->d.nz, ix = (p / c->d.nz) % c->d.nx, iy = p / c->g.yStride;
      if (iz < FAT || iz >= c->d.nz - FAT || ix < FAT || ix >= c->d.nx - FAT || iy < FAT || iy >= c->d.ny - FAT) {
        setLastError("acquisition point inside the FAT ring", __FILE__, __LINE__);
        return E3D_ERR_BOUNDS;
      }
      h[s.set.off[k] + i] = p;
    }
  }
  E3D_RET(devAlloc(c, (void**)&s.pos, h.size() * sizeof(long long)));
  E3D_CUDA_TRY(cudaMemcpyAsync(s.pos, h.data(), h.size() * sizeof(long long), cudaMemcpyHostToDevice, c->st));
  s.set.pos = s.pos;
  return E3D_OK;
}

// Copy 9 reference-layout host blocks ([n_k][nts]) to a time-major device array.
static int stageSignalsIn(Context* c, Staged& s, const float* const* host) {
  const int nts = c->d.nts;
  const size_t bytes = (size_t)std::max(s.ntot, 1) * nts * sizeof(float);
  E3D_RET(devAlloc(c, (void**)&s.sig, bytes));
  E3D_RET(scratchAtLeast(c, bytes));
  float* tmp = (float*)c->scratch;
  for (int k = 0; k < NCOMP; k++) {
    const long long n = s.set.off[k + 1] - s.set.off[k];
    if (n == 0) continue;
    E3D_ARG(host[k] != nullptr, "null signal block");
    E3D_CUDA_TRY(cudaMemcpyAsync(tmp + (size_t)s.set.off[k] * nts, host[k], (size_t)n * nts * sizeof(float),
                                 cudaMemcpyHostToDevice, c->st));
  }
  return transpose(c, tmp, s.sig, s.ntot, nts);
}

static int stageSignalsZero(Context* c, Staged& s) {
  const size_t bytes = (size_t)std::max(s.ntot, 1) * c->d.nts * sizeof(float);
  E3D_RET(devAlloc(c, (void**)&s.sig, bytes));
  E3D_CUDA_TRY(cudaMemsetAsync(s.sig, 0, bytes, c->st));
  return E3D_OK;
}

static int stageSignalsOut(Context* c, Staged& s, float* const* host) {
  const int nts = c->d.nts;
  const size_t bytes = (size_t)std::max(s.ntot, 1) * nts * sizeof(float);
  E3D_RET(scratchAtLeast(c, bytes));
  float* tmp = (float*)c->scratch;
  E3D_RET(transpose(c, s.sig, tmp, nts, s.ntot));
  for (int k = 0; k < NCOMP; k++) {
    const long long n = s.set.off[k + 1] - s.set.off[k];
    if (n == 0) continue;
    E3D_ARG(host[k] != nullptr, "null output block");
    E3D_CUDA_TRY(cudaMemcpyAsync(host[k], tmp + (size_t)s.set.off[k] * nts, (size_t)n * nts * sizeof(float),
                                 cudaMemcpyDeviceToHost, c->st));
  }
  return E3D_OK;
}

static void releaseStaged(Context* c, Staged& s) {
  devFree(c, s.pos);
  devFree(c, s.sig);
  s.pos = nullptr;
  s.sig = nullptr;
}

// ---------------------------------------------------------------------------
// Nonlinear propagation
// ---------------------------------------------------------------------------
// Forward (propElasticFwdGpu_3D): per fine step  step -> inject (k=it2-1) ->
// [damp fused] -> record (k=it2) -> swap.
// Adjoint (propElasticAdjGpu_3D, time-reversed stepper, quirk Q7): per fine
// step step -> inject data (k=it2+1) -> record source (k=it2) -> swap.
__global__ void kSetIndex(int* its, int v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *its = v;
}

static int launchInjectIdx(Context* c, const StepPtrs& p, const DevSignals& s, const float* sig, const int* idx,
                           int k) {
  SparseSet ss;
  ss.pos = s.pos;
  for (int i = 0; i <= NCOMP; i++) ss.off[i] = s.off[i];
  const int n = s.off[NCOMP];
  if (n == 0) return E3D_OK;
  c->launches++;
  kInjectIdx<<<(n + 127) / 128, 128, 0, c->st>>>(p, c->g, ss, sig, idx, c->filt[k], c->filt[c->hfilt + k]);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

static int launchRecordIdx(Context* c, const StepPtrs& p, const DevSignals& s, float* out, const int* idx, int k) {
  SparseSet ss;
  ss.pos = s.pos;
  for (int i = 0; i <= NCOMP; i++) ss.off[i] = s.off[i];
  const int n = s.off[NCOMP];
  if (n == 0) return E3D_OK;
  c->launches++;
  kRecordIdx<<<(n + 127) / 128, 128, 0, c->st>>>(p, ss, out, idx, c->filt[k], c->filt[c->hfilt + k]);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

// One coarse block of the nonlinear loops.  Forward (propElasticFwdGpu_3D):
// per fine step it2 = 1..sub  step -> inject (k=it2-1) -> [free surface] ->
// record (k=it2) -> swap.  Time-reversed (propElasticAdjGpu_3D, quirk Q7):
// it2 = sub-1..0  step -> inject data (k=it2+1) -> [free surface] -> record
// source (k=it2) -> swap.  With idx the coarse index is read on the device.
// Fine step s of coarse block its (the reference's loop order): step, inject, free surface,
// record; the new level ends in c->w1.
static int nlSubStep(Context* c, bool adjoint, const DevSignals& srcSet, const DevSignals& recSet, float* srcSig,
                     float* recSig, int its, int s, const int* idx) {
  const int sub = c->d.sub;
  const DevSignals& inSet = adjoint ? recSet : srcSet;
  const DevSignals& outSet = adjoint ? srcSet : recSet;
  float* inSig = adjoint ? recSig : srcSig;
  float* outSig = adjoint ? srcSig : recSig;
  const int it2 = adjoint ? sub - 1 - s : s + 1;
  const int kIn = adjoint ? it2 + 1 : it2 - 1;
  StepPtrs p = makeStep(c, c->w0, c->w1);
  E3D_RET(launchStep(c, adjoint ? STEP_ADJ_REVERSED : STEP_FWD, p));
  if (idx) E3D_RET(launchInjectIdx(c, p, inSet, inSig, idx, kIn));
  else E3D_RET(launchInject(c, p, inSet, inSig, its, kIn));
  E3D_RET(launchFreeSurface(c, p, adjoint ? -1.f : 1.f));
  if (idx) E3D_RET(launchRecordIdx(c, p, outSet, outSig, idx, it2));
  else E3D_RET(launchRecord(c, p, outSet, outSig, its, it2));
  swapF(c->w0, c->w1);
  return E3D_OK;
}

static int nlBlock(Context* c, bool adjoint, const DevSignals& srcSet, const DevSignals& recSet, float* srcSig,
                   float* recSig, int its, const int* idx) {
  for (int s = 0; s < c->d.sub; s++) E3D_RET(nlSubStep(c, adjoint, srcSet, recSet, srcSig, recSig, its, s, idx));
  return E3D_OK;
}

// Capture one coarse block (block(idx) with the device-resident coarse index,
// then the index advanced by `delta`) into an executable graph.  Counted launches
// of the capture are returned in *perBlock and taken back out of the context's count.
template <class Block>
static int captureBlockWith(Context* c, Block block, int delta, cudaGraphExec_t* exec, long long* perBlock) {
  const long long before = c->launches;
  cudaGraph_t graph = nullptr;
  E3D_CUDA_TRY(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
  c->inCapture = true;
  int st = block(c->blockIndex);
  if (st == E3D_OK) {
    kAdvanceIndex<<<1, 32, 0, c->st>>>(c->blockIndex, delta);
    c->launches++;
    if (cudaGetLastError() != cudaSuccess) {
      setLastError("index advance launch failed", __FILE__, __LINE__);
      st = E3D_ERR_CUDA;
    }
  }
  c->inCapture = false;
  const cudaError_t e = cudaStreamEndCapture(c->st, &graph);
  *perBlock = c->launches - before;
  c->launches = before;
  if (st == E3D_OK && e != cudaSuccess) {
    setLastError(cudaGetErrorString(e), __FILE__, __LINE__);
    st = E3D_ERR_CUDA;
  }
  if (st == E3D_OK) {
    const cudaError_t ei = cudaGraphInstantiate(exec, graph, 0);
    if (ei != cudaSuccess) {
      setLastError(cudaGetErrorString(ei), __FILE__, __LINE__);
      st = E3D_ERR_CUDA;
    }
  }
  if (graph) cudaGraphDestroy(graph);
  return st;
}

// Replay of coarse blocks 1..blocks-1 after block 0 ran eagerly: one captured block (two when
// sub is odd, for the two pointer parities of the leapfrog levels lv0/lv1), the coarse index on
// the device starting at `next` and moving by `delta`.
template <class Block>
static int replayBlocks(Context* c, Block block, int blocks, int next, int delta, Fields9& lv0, Fields9& lv1) {
  if (!c->blockIndex) E3D_RET(devAlloc(c, (void**)&c->blockIndex, sizeof(int)));
  kSetIndex<<<1, 32, 0, c->st>>>(c->blockIndex, next);
  c->launches++;
  E3D_LAUNCH_CHECK();
  const int sub = c->d.sub;
  const int ng = (sub % 2) ? 2 : 1;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  long long perBlock[2] = {0, 0};
  int st = E3D_OK;
  for (int i = 0; i < ng && st == E3D_OK; i++) st = captureBlockWith(c, block, delta, &exec[i], &perBlock[i]);
  for (int b = 1; b < blocks && st == E3D_OK; b++) {
    const int i = (b - 1) % ng;
    const cudaError_t e = cudaGraphLaunch(exec[i], c->st);
    if (e != cudaSuccess) {
      setLastError(cudaGetErrorString(e), __FILE__, __LINE__);
      st = E3D_ERR_CUDA;
    }
    c->launches += perBlock[i];
  }
  // the host-side level pointers follow the replayed blocks: each capture swapped them sub
  // times, and capture ng - 1 more blocks' worth than ran
  if (st == E3D_OK) {
    const long long swapsCaptured = (long long)ng * sub, swapsRun = (long long)(blocks - 1) * sub;
    if ((swapsCaptured + swapsRun) % 2) swapF(lv0, lv1);
  }
  for (int i = 0; i < ng; i++)
    if (exec[i]) cudaGraphExecDestroy(exec[i]);
  return st;
}

int setGraphLoop(Context* c, int on) {
  E3D_ARG(c, "null context");
  c->graphLoop = on ? 1 : 0;
  return E3D_OK;
}

// Nonlinear propagation (propElasticFwdGpu_3D / propElasticAdjGpu_3D).  The
// first coarse block runs eagerly; with the graph loop on (and a stream other
// than the legacy default stream) the remaining blocks replay one captured
// block (two when sub is odd, for the two pointer parities), the coarse index
// living on the device.
// Device position tables checked before any injection or recording (the host
// path checks host tables the same way): every entry an updated cell.  flagDev
// is a device word the check may overwrite; the result is read back on `st`.
static int checkDevicePositions(const DevSignals* const* sets, int nsets, int nz, int nx, int ny, unsigned* flagDev,
                                cudaStream_t st, int shots = 1) {
  bool any = false;
  for (int i = 0; i < nsets; i++) any = any || sets[i]->off[NCOMP] > 0;
  if (!any) return E3D_OK;
  E3D_CUDA_TRY(cudaMemsetAsync(flagDev, 0, sizeof(unsigned), st));
  for (int i = 0; i < nsets; i++) {
    const int n = sets[i]->off[NCOMP];
    if (n == 0) continue;
    E3D_ARG(sets[i]->pos != nullptr, "null position table");
    kCheckPositions<<<(n + 255) / 256, 256, 0, st>>>(sets[i]->pos, n, nz, nx, ny, shots, flagDev);
    E3D_LAUNCH_CHECK();
  }
  unsigned bad = 0;
  E3D_CUDA_TRY(cudaMemcpyAsync(&bad, flagDev, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  E3D_CUDA_TRY(cudaStreamSynchronize(st));
  if (bad) {
    setLastError("device position table holds a point inside the FAT ring or outside the grid", __FILE__, __LINE__);
    return E3D_ERR_BOUNDS;
  }
  return E3D_OK;
}

int validateDeviceSets(Context* c, const DevSignals& a, const DevSignals& b, int shots) {
  E3D_ARG(c != nullptr, "null context");
  E3D_CUDA_TRY(cudaSetDevice(c->d.device));
  if (!c->posFlag) E3D_RET(devAlloc(c, (void**)&c->posFlag, sizeof(unsigned)));
  const DevSignals* sets[2] = {&a, &b};
  c->launches += (a.off[NCOMP] > 0) + (b.off[NCOMP] > 0);
  return checkDevicePositions(sets, 2, c->d.nz, c->d.nx, c->d.ny, c->posFlag, c->st, shots);
}

// ---------------------------------------------------------------------------
// Batched nonlinear forward: `shots` shots of one medium advanced together.
// Each field holds the shots stacked (shot s at offset s*n), every fine step is
// one split-stepper launch for all shots (CTAs of one tile for consecutive
// shots adjacent, so the medium tile comes from L2 after the first shot), one
// injection and one recording launch over the combined tables, whose
// positions carry the shot offset.  Loop order of propElasticFwdGpu_3D.
// ---------------------------------------------------------------------------
int nlForwardBatchDevice(Context* c, int shots, const DevSignals& srcSet, const DevSignals& recSet,
                         const float* srcSig, float* recSig) {
  E3D_ARG(c && c->haveMedium, "medium not set");
  E3D_ARG(shots >= 1 && shots <= 1024, "shots must be in [1, 1024]");
  E3D_ARG(c->d.nz % 4 == 0, "batched propagation needs nz % 4 == 0");
  E3D_ARG(!c->d.freeSurface, "batched propagation has no free surface");
  E3D_CUDA_TRY(cudaSetDevice(c->d.device));
  const size_t bytes = (size_t)shots * c->g.n * sizeof(float);
  if (c->batchShots != shots) {
    for (int k = 0; k < NCOMP; k++) {
      devFree(c, c->bw0.p[k]);
      devFree(c, c->bw1.p[k]);
      c->bw0.p[k] = c->bw1.p[k] = nullptr;
    }
    c->batchShots = 0;
    for (int k = 0; k < NCOMP; k++) {
      E3D_RET(devAlloc(c, (void**)&c->bw0.p[k], bytes));
      E3D_RET(devAlloc(c, (void**)&c->bw1.p[k], bytes));
    }
    c->batchShots = shots;
  }
  for (int k = 0; k < NCOMP; k++) {
    E3D_CUDA_TRY(cudaMemsetAsync(c->bw0.p[k], 0, bytes, c->st));
    E3D_CUDA_TRY(cudaMemsetAsync(c->bw1.p[k], 0, bytes, c->st));
  }
  const int nts = c->d.nts, sub = c->d.sub;
  E3D_CUDA_TRY(cudaMemsetAsync(recSig, 0, (size_t)std::max(recSet.off[NCOMP], 1) * nts * sizeof(float), c->st));
  // one coarse block (its, or the device index idx) of all shots
  auto block = [&](int its, const int* idx) -> int {
    for (int it2 = 1; it2 <= sub; it2++) {
      StepPtrs p = makeStep(c, c->bw0, c->bw1);
      {
        c->launches++;
        TimedLaunch t(c, STEP_FWD);
        E3D_RET(launchSplitBatch<STEP_FWD>(c, p, shots));
      }
      if (idx) E3D_RET(launchInjectIdx(c, p, srcSet, srcSig, idx, it2 - 1));
      else E3D_RET(launchInject(c, p, srcSet, srcSig, its, it2 - 1));
      if (idx) E3D_RET(launchRecordIdx(c, p, recSet, recSig, idx, it2));
      else E3D_RET(launchRecord(c, p, recSet, recSig, its, it2));
      swapF(c->bw0, c->bw1);
    }
    return E3D_OK;
  };
  const int blocks = nts - 1;
  const bool graph = c->graphLoop && c->st != nullptr && c->timingEvery == 0 && blocks >= 4;
  if (!graph) {
    for (int its = 0; its < blocks; its++) E3D_RET(block(its, nullptr));
    return E3D_OK;
  }
  // the time loop as replays of one captured coarse block, as nlPropagateDevice
  E3D_RET(block(0, nullptr));
  return replayBlocks(c, [&](const int* idx) { return block(0, idx); }, blocks, 1, 1, c->bw0, c->bw1);
}

int nlPropagateDevice(Context* c, bool adjoint, const DevSignals& srcSet, const DevSignals& recSet, float* srcSig,
                      float* recSig) {
  E3D_ARG(c && c->haveMedium, "medium not set");
  E3D_CUDA_TRY(cudaSetDevice(c->d.device));
  E3D_RET(allocFields(c, c->w0, true));
  E3D_RET(allocFields(c, c->w1, true));
  const int nts = c->d.nts, sub = c->d.sub;
  const int blocks = nts - 1;
  float* outSig = adjoint ? srcSig : recSig;
  const DevSignals& outSet = adjoint ? srcSet : recSet;
  E3D_CUDA_TRY(cudaMemsetAsync(outSig, 0, (size_t)std::max(outSet.off[NCOMP], 1) * nts * sizeof(float), c->st));
  const int first = adjoint ? nts - 2 : 0;
  const int dir = adjoint ? -1 : 1;
  const bool graph = c->graphLoop && c->st != nullptr && c->timingEvery == 0 && blocks >= 4;
  if (!graph) {
    for (int b = 0; b < blocks; b++) E3D_RET(nlBlock(c, adjoint, srcSet, recSet, srcSig, recSig, first + dir * b, nullptr));
    return E3D_OK;
  }
  E3D_RET(nlBlock(c, adjoint, srcSet, recSet, srcSig, recSig, first, nullptr));
  return replayBlocks(
      c, [&](const int* idx) { return nlBlock(c, adjoint, srcSet, recSet, srcSig, recSig, 0, idx); }, blocks,
      first + dir, dir, c->w0, c->w1);
}

int nlPropagateHost(Context* c, bool adjoint, float* const* model, float* const* data, const HostGeom& src,
                    const HostGeom& rec) {
  E3D_ARG(c && model && data, "null argument");
  E3D_CUDA_TRY(cudaSetDevice(c->d.device));
  Staged S, R;
  int st = stageGeom(c, src, false, S);
  if (st == E3D_OK) st = stageGeom(c, rec, true, R);
  if (st == E3D_OK) st = adjoint ? stageSignalsZero(c, S) : stageSignalsIn(c, S, model);
  if (st == E3D_OK) st = adjoint ? stageSignalsIn(c, R, data) : stageSignalsZero(c, R);
  if (st == E3D_OK) st = nlPropagateDevice(c, adjoint, S.set, R.set, S.sig, R.sig);
  if (st == E3D_OK) st = adjoint ? stageSignalsOut(c, S, model) : stageSignalsOut(c, R, data);
  if (st == E3D_OK) st = checkPipeError(c);
  if (st == E3D_OK) {
    cudaError_t e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) {
      setLastError(cudaGetErrorString(e), __FILE__, __LINE__);
      st = E3D_ERR_CUDA;
    }
  }
  releaseStaged(c, S);
  releaseStaged(c, R);
  return st;
}

// ---------------------------------------------------------------------------
// y-slab domain decomposition of the nonlinear propagation
// (propElasticFwdGpudomDec_3D / propElasticAdjGpudomDec_3D,
// nonlinearPropElasticGpuFunctions_3D.cu:976-1297, 1396-1719; slab sizes as
// nonlinearPropElasticShotsGpu_3D.cpp:48-76).  Slab s is a context over the
// global planes [Y_s, Y_s + ny_s), Y_0 = 0 and Y_{s+1} = Y_s + ny_s - 2 FAT, so
// neighbours overlap by 2 FAT planes: each updates its own planes
// [FAT, ny_s - FAT) and keeps its neighbours' boundary planes in its FAT
// planes.  After every fine step and its injection the new level's boundary
// planes (FAT planes of the nine fields) are copied into the neighbours' ghost
// planes; events order the copies between the slabs' streams, so no kernel waits
// on another.  Every acquisition point goes to the slab that updates it, and
// every cell is updated with the arithmetic of the undivided grid (the taper
// reads global y), so the result is the undivided propagation's.
// ---------------------------------------------------------------------------
namespace {
struct SlabRun {
  Context* c = nullptr;
  long long y0 = 0;  // global plane of local plane 0
  Staged S, R;
  std::vector<long long> pos[2][NCOMP], rows[2][NCOMP];  // [0] sources, [1] receivers
  std::vector<float> sig[2][NCOMP];
  cudaEvent_t stepped = nullptr, copied = nullptr;
};

// Component tables of one side (sources or receivers) in component order, with the sxz receiver
// rule (quirk Q2) applied, as stageGeom builds them.
int componentTable(const Context* c, const HostGeom& g, bool receivers, int k, const long long** tab, long long* n) {
  const int gi = gridOfComp(k);
  E3D_ARG(g.n[gi] >= 0 && g.n[gi] < (1LL << 30), "bad device count");
  const long long* src = g.pos[gi];
  if (receivers && k == SXZ && c->d.q2compat) {
    E3D_ARG(g.n[GXZ] <= g.n[GZ], "sxz receivers read past the z-grid table (reference quirk Q2)");
    src = g.pos[GZ];
  }
  E3D_ARG(g.n[gi] == 0 || src != nullptr, "null position table");
  *tab = src;
  *n = g.n[gi];
  return E3D_OK;
}

int stageSlabTables(Context* c, const std::vector<long long>* pos, Staged& s) {
  long long tot = 0;
  for (int k = 0; k < NCOMP; k++) {
    s.set.off[k] = (int)tot;
    tot += (long long)pos[k].size();
  }
  s.set.off[NCOMP] = (int)tot;
  s.ntot = (int)tot;
  std::vector<long long> h(std::max<long long>(tot, 1));
  for (int k = 0; k < NCOMP; k++) std::copy(pos[k].begin(), pos[k].end(), h.begin() + s.set.off[k]);
  E3D_RET(devAlloc(c, (void**)&s.pos, h.size() * sizeof(long long)));
  E3D_CUDA_TRY(cudaMemcpyAsync(s.pos, h.data(), h.size() * sizeof(long long), cudaMemcpyHostToDevice, c->st));
  E3D_CUDA_TRY(cudaStreamSynchronize(c->st));  // h is a local buffer
  s.set.pos = s.pos;
  return E3D_OK;
}

// Copy planes [from, from + FAT) of the nine fields of `src` into planes [to, to + FAT) of `dst`
// on dst's stream (peer copies between devices through unified addressing).
int copyGhostPlanes(const SlabRun& dst, long long to, const SlabRun& src, long long from) {
  const long long ys = dst.c->g.yStride;
  const size_t bytes = (size_t)FAT * ys * sizeof(float);
  for (int k = 0; k < NCOMP; k++)
    E3D_CUDA_TRY(cudaMemcpyAsync(dst.c->w1.p[k] + to * ys, src.c->w1.p[k] + from * ys, bytes, cudaMemcpyDefault,
                                 dst.c->st));
  return E3D_OK;
}
}  // namespace

int nlPropagateSlabsHost(Context* const* slabs, int nSlabs, int nyGlobal, bool adjoint, float* const* model,
                         float* const* data, const HostGeom& src, const HostGeom& rec) {
  E3D_ARG(slabs && nSlabs >= 1 && nSlabs <= 64 && model && data, "bad slab arguments");
  std::vector<SlabRun> sl(nSlabs);
  const Context* c0 = slabs[0];
  E3D_ARG(c0 && c0->haveMedium, "slab 0 has no medium");
  long long y = 0;
  for (int i = 0; i < nSlabs; i++) {
    Context* c = slabs[i];
    E3D_ARG(c && c->haveMedium, "a slab has no medium");
    const ContextDesc &d = c->d, &d0 = c0->d;
    E3D_ARG(d.nz == d0.nz && d.nx == d0.nx && d.nts == d0.nts && d.sub == d0.sub && d.minPad == d0.minPad &&
                d.dz == d0.dz && d.dx == d0.dx && d.dy == d0.dy && d.dts == d0.dts && d.alphaCos == d0.alphaCos &&
                d.fixQ1 == d0.fixQ1 && d.q2compat == d0.q2compat && d.freeSurface == d0.freeSurface,
            "slabs of one grid must share every parameter but ny");
    // each slab sends FAT of its own planes to each neighbour
    E3D_ARG(d.ny >= 3 * FAT, "a slab needs at least FAT planes of its own (ny_domDec >= 3*FAT)");
    for (int j = 0; j < i; j++) E3D_ARG(slabs[j] != c, "a context appears twice among the slabs");
    sl[i].c = c;
    sl[i].y0 = y;
    y += d.ny - 2 * FAT;
  }
  E3D_ARG(y + 2 * FAT == nyGlobal, "slab sizes do not add up to ny (sum of ny_domDec - 2*FAT*(n-1) != ny)");
  const long long ys = c0->g.yStride;
  const long long nG = ys * nyGlobal;

  // deal the acquisition points to the slabs that update them
  for (int side = 0; side < 2; side++) {
    const HostGeom& g = side ? rec : src;
    for (int k = 0; k < NCOMP; k++) {
      const long long* tab = nullptr;
      long long n = 0;
      E3D_RET(componentTable(c0, g, side == 1, k, &tab, &n));
      for (long long i = 0; i < n; i++) {
        const long long p = tab[i];
        E3D_ARG(p >= 0 && p < nG, "acquisition point outside the grid");
        const long long iy = p / ys;
        int owner = -1;
        for (int t = 0; t < nSlabs && owner < 0; t++)
          if (iy >= sl[t].y0 + FAT && iy < sl[t].y0 + sl[t].c->d.ny - FAT) owner = t;
        if (owner < 0) {
          setLastError("acquisition point inside the FAT ring", __FILE__, __LINE__);
          return E3D_ERR_BOUNDS;
        }
        sl[owner].pos[side][k].push_back(p - sl[owner].y0 * ys);
        sl[owner].rows[side][k].push_back(i);
      }
    }
  }
  const int nts = c0->d.nts, sub = c0->d.sub;
  const int inSide = adjoint ? 1 : 0;
  float* const* inHost = adjoint ? data : model;
  float* const* outHost = adjoint ? model : data;
  int st = E3D_OK;
  // a failed CUDA call of the slab orchestration: its message and E3D_ERR_CUDA
  auto cu = [&](cudaError_t e) {
    if (e != cudaSuccess && st == E3D_OK) {
      setLastError(cudaGetErrorString(e), __FILE__, __LINE__);
      st = E3D_ERR_CUDA;
    }
    return st == E3D_OK;
  };
  for (int i = 0; i < nSlabs && st == E3D_OK; i++) {
    SlabRun& r = sl[i];
    Context* c = r.c;
    cu(cudaSetDevice(c->d.device));
    if (st == E3D_OK) {
      c->g.yOff = (int)r.y0;
      c->g.nyTaper = nyGlobal;
    }
    // input rows gathered into slab-local blocks, [n_k][nts] as the host layout
    const float* in[NCOMP];
    for (int k = 0; k < NCOMP && st == E3D_OK; k++) {
      const auto& rows = r.rows[inSide][k];
      r.sig[inSide][k].resize(std::max<size_t>(rows.size(), 1) * nts);
      for (size_t j = 0; j < rows.size(); j++) {
        if (!inHost[k]) {
          setLastError("null signal block", __FILE__, __LINE__);
          st = E3D_ERR_ARG;
          break;
        }
        std::copy(inHost[k] + rows[j] * nts, inHost[k] + (rows[j] + 1) * nts, r.sig[inSide][k].begin() + j * nts);
      }
      in[k] = r.sig[inSide][k].data();
    }
    if (st == E3D_OK) st = stageSlabTables(c, r.pos[0], r.S);
    if (st == E3D_OK) st = stageSlabTables(c, r.pos[1], r.R);
    if (st == E3D_OK) st = adjoint ? stageSignalsZero(c, r.S) : stageSignalsIn(c, r.S, in);
    if (st == E3D_OK) st = adjoint ? stageSignalsIn(c, r.R, in) : stageSignalsZero(c, r.R);
    if (st == E3D_OK) st = allocFields(c, c->w0, true);
    if (st == E3D_OK) st = allocFields(c, c->w1, true);
    if (st == E3D_OK) cu(cudaEventCreateWithFlags(&r.stepped, cudaEventDisableTiming));
    if (st == E3D_OK) cu(cudaEventCreateWithFlags(&r.copied, cudaEventDisableTiming));
  }
  // the time loop: every slab steps, then every slab fetches its ghost planes
  for (int b = 0; b < nts - 1 && st == E3D_OK; b++) {
    const int its = adjoint ? nts - 2 - b : b;
    for (int s = 0; s < sub && st == E3D_OK; s++) {
      const bool first = b == 0 && s == 0;
      for (int i = 0; i < nSlabs && st == E3D_OK; i++) {
        SlabRun& r = sl[i];
        Context* c = r.c;
        if (!cu(cudaSetDevice(c->d.device))) break;
        // the neighbours have read this slab's previous level before it is overwritten
        if (!first) {
          if (i > 0) cu(cudaStreamWaitEvent(c->st, sl[i - 1].copied, 0));
          if (i + 1 < nSlabs) cu(cudaStreamWaitEvent(c->st, sl[i + 1].copied, 0));
        }
        if (st == E3D_OK) st = nlSubStep(c, adjoint, r.S.set, r.R.set, r.S.sig, r.R.sig, its, s, nullptr);
        if (st == E3D_OK) cu(cudaEventRecord(r.stepped, c->st));
      }
      for (int i = 0; i < nSlabs && st == E3D_OK; i++) {
        SlabRun& r = sl[i];
        Context* c = r.c;
        if (!cu(cudaSetDevice(c->d.device))) break;
        const long long ny = c->d.ny;
        if (i > 0) {
          const SlabRun& lo = sl[i - 1];
          cu(cudaStreamWaitEvent(c->st, lo.stepped, 0));
          // the lower neighbour's top own planes into this slab's bottom ghost planes
          if (st == E3D_OK) st = copyGhostPlanes(r, 0, lo, lo.c->d.ny - 2 * FAT);
        }
        if (i + 1 < nSlabs && st == E3D_OK) {
          const SlabRun& hi = sl[i + 1];
          cu(cudaStreamWaitEvent(c->st, hi.stepped, 0));
          // the upper neighbour's bottom own planes into this slab's top ghost planes
          if (st == E3D_OK) st = copyGhostPlanes(r, ny - FAT, hi, FAT);
        }
        if (st == E3D_OK) cu(cudaEventRecord(r.copied, c->st));
      }
    }
  }
  // outputs back to the host rows they came from
  for (int i = 0; i < nSlabs; i++) {
    SlabRun& r = sl[i];
    Context* c = r.c;
    cudaSetDevice(c->d.device);
    const int outSide = 1 - inSide;
    float* out[NCOMP];
    for (int k = 0; k < NCOMP; k++) {
      r.sig[outSide][k].assign(std::max<size_t>(r.rows[outSide][k].size(), 1) * nts, 0.f);
      out[k] = r.sig[outSide][k].data();
    }
    if (st == E3D_OK) st = stageSignalsOut(c, adjoint ? r.S : r.R, out);
    if (st == E3D_OK) st = checkPipeError(c);  // synchronizes the slab's stream
    if (st == E3D_OK)
      for (int k = 0; k < NCOMP && st == E3D_OK; k++) {
        const auto& rows = r.rows[outSide][k];
        if (!rows.empty() && !outHost[k]) {
          setLastError("null output block", __FILE__, __LINE__);
          st = E3D_ERR_ARG;
        }
        for (size_t j = 0; j < rows.size() && st == E3D_OK; j++)
          std::copy(out[k] + j * nts, out[k] + (j + 1) * nts, outHost[k] + rows[j] * nts);
      }
  }
  for (int i = 0; i < nSlabs; i++) {
    SlabRun& r = sl[i];
    Context* c = r.c;
    cudaSetDevice(c->d.device);
    cudaStreamSynchronize(c->st);
    releaseStaged(c, r.S);
    releaseStaged(c, r.R);
    if (r.stepped) cudaEventDestroy(r.stepped);
    if (r.copied) cudaEventDestroy(r.copied);
    c->g.yOff = 0;
    c->g.nyTaper = c->d.ny;
  }
  return st;
}

int stepOnly(Context* c, int mode, int nSteps) {
  E3D_ARG(c && c->haveMedium, "medium not set");
  E3D_ARG(mode >= 0 && mode <= 5, "bad mode");
  // modes 3..5: modes 0..2 with the new level decimated into two coarse
  // accumulators, as the fused-accumulator passes run them (3 velocity fields for
  // the source recompute, 9 fields for the adjoint).  The ring passes' exact
  // adjoint on the premultiplied-only state is mode 1 on premultiplied levels.
  const bool fused = mode >= 3;
  const int m = fused ? mode - 3 : mode;
  E3D_RET(allocFields(c, c->w0, false));
  E3D_RET(allocFields(c, c->w1, false));
  if (fused) {
    E3D_RET(allocFields(c, c->ss[0], true));
    E3D_RET(allocFields(c, c->ss[1], true));
  }
  // the exact adjoint runs on the dual state, as in the adjoint pass, with the TMA loader
  const bool dual = m == STEP_ADJ_EXACT && c->loader >= 2 && c->d.nz % 4 == 0;
  if (dual) {
    E3D_RET(allocFields(c, c->q0, false));
    E3D_RET(allocFields(c, c->q1, false));
  }
  for (int i = 0; i < nSteps; i++) {
    StepPtrs p = makeStep(c, c->w0, c->w1);
    if (dual)
      for (int k = 0; k < NCOMP; k++) {
        p.c[k] = c->q1.p[k];
        p.oP[k] = c->q0.p[k];
      }
    if (fused) {
      p.nAcc = m == STEP_ADJ_EXACT ? NCOMP : 3;
      for (int k = 0; k < p.nAcc; k++) {
        p.accL[k] = c->ss[0].p[k];
        p.accR[k] = c->ss[1].p[k];
      }
      p.accWl = c->filt[1];
      p.accWr = c->filt[c->hfilt + 1];
    }
    E3D_RET(launchStep(c, m, p));
    swapF(c->w0, c->w1);
    if (dual) swapF(c->q0, c->q1);
  }
  return E3D_OK;
}

int checkpointSegment(const Context* c) { return c->ckptSegLen; }

// ---------------------------------------------------------------------------
// Born
// ---------------------------------------------------------------------------
static int ensureVSlots(Context* c, int nslots) {
  while ((int)c->vSlots.size() < nslots) {
    float* v = nullptr;
    E3D_RET(devAlloc(c, (void**)&v, (size_t)3 * c->g.n * sizeof(float)));
    c->vSlots.push_back(v);
  }
  return E3D_OK;
}

static float* vComp(float* slot, int k, long long n) { return slot ? slot + (size_t)k * n : nullptr; }

// Decimation of the damped velocity of fine step it2 of a source block into
// vLeft (weight f[it2]) and vRight (weight f[h+it2]); with vLeft null only the
// right slot accumulates (interpWavefieldVxVyVz_3D, kernelsElaGpu_3D.cu:1646-1672).
static void setSourceAcc(const Context* c, StepPtrs& p, int it2, float* vLeft, float* vRight) {
  const long long n = c->g.n;
  for (int k = 0; k < 3; k++) {
    p.accL[k] = vComp(vLeft, k, n);
    p.accR[k] = vComp(vRight, k, n);
  }
  if (!vLeft) {  // only the right accumulator is wanted
    for (int k = 0; k < 3; k++) {
      p.accL[k] = p.accR[k];
      p.accR[k] = nullptr;
    }
    p.accWl = c->filt[c->hfilt + it2];
  } else {
    p.accWl = c->filt[it2];
    p.accWr = c->filt[c->hfilt + it2];
  }
  p.nAcc = 3;
}

// One coarse block (its) of the source-side forward propagation on state
// (s0,s1), injecting srcSig and decimating into vLeft / vRight.
static int sourceBlock(Context* c, int its, const DevSignals& srcSet, const float* srcSig, float* vLeft,
                       float* vRight) {
  for (int it2 = 1; it2 <= c->d.sub; it2++) {
    StepPtrs p = makeStep(c, c->s0, c->s1);
    setSourceAcc(c, p, it2, vLeft, vRight);
    E3D_RET(launchStep(c, STEP_FWD, p));
    E3D_RET(launchInject(c, p, srcSet, srcSig, its, it2 - 1));
    swapF(c->s0, c->s1);
  }
  return E3D_OK;
}

static int launchImaging(Context* c, bool adjoint, int t, float* vPrev, float* vCur, float* vNext, Fields9& ss) {
  ImagingPtrs q{};
  const long long n = c->g.n;
  for (int k = 0; k < 3; k++) {
    q.vPrev[k] = vComp(vPrev, k, n);
    q.vCur[k] = vComp(vCur, k, n);
    q.vNext[k] = vComp(vNext, k, n);
  }
  for (int k = 0; k < NCOMP; k++) q.ss[k] = ss.p[k];
  for (int k = 0; k < NMED; k++) q.pert[k] = c->pertDev[k];
  q.dtsInv = c->dtsInv;
  q.q3compat = c->d.q3compat;
  dim3 block(32, 8);
  dim3 grid((c->d.nz - 2 * FAT + 31) / 32, (c->d.nx - 2 * FAT + 7) / 8, c->d.ny - 2 * FAT);
  c->launches++;
  if (adjoint) kImaging<true><<<grid, block, 0, c->st>>>(q, c->g);
  else kImaging<false><<<grid, block, 0, c->st>>>(q, c->g);
  E3D_LAUNCH_CHECK();
  (void)t;
  return E3D_OK;
}

// ---------------------------------------------------------------------------
// Rings of fine time levels (the gradient's passes).  With a ring the stepper
// writes level m+1 into its own slot, so the sub levels of a coarse block are
// all still there when the block ends, and one launch per block decimates them
// (source velocity) or decimates and images them (adjoint) instead of the
// stepper reading and writing two accumulators at every fine step.
// ---------------------------------------------------------------------------
static int ringLevels(const Context* c) {
  return (c->ringMode && c->d.sub <= RING_SUB_MAX) ? std::max(c->d.sub + 1, 3) : 0;
}

// The ring passes' exact adjoint runs on the premultiplied-only state where the
// medium's premultiplication is this well conditioned (the normal-stress block's
// eigenvalue ratio; every density and shear plane positive): its stepper needs no
// inverse, but the block imaging recovers the raw decimated fields with one, at
// a cost of a few float roundings times this ratio.
constexpr double kPremCondMax = 100.0;

static int premultipliedAdjoint(Context* c, bool& use) {
  use = false;
  if (!c->premMode || c->loader < 2 || c->d.nz % 4 != 0 || !c->haveMedium) return E3D_OK;
  if (c->premCond < 0) {
    if (!c->posFlag) E3D_RET(devAlloc(c, (void**)&c->posFlag, sizeof(unsigned)));
    E3D_CUDA_TRY(cudaMemsetAsync(c->posFlag, 0, sizeof(unsigned), c->st));
    StepPtrs p{};
    for (int k = 0; k < NMED; k++) p.m[k] = c->med[k];
    c->launches++;
    kPremultiplyCondition<<<c->numSMs * 4, 256, 0, c->st>>>(p, c->g, c->posFlag);
    E3D_LAUNCH_CHECK();
    unsigned bits = 0;
    E3D_CUDA_TRY(cudaMemcpyAsync(&bits, c->posFlag, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
    E3D_CUDA_TRY(cudaStreamSynchronize(c->st));
    float cond;
    std::memcpy(&cond, &bits, sizeof(float));
    c->premCond = std::isfinite(cond) ? (double)cond : 1e30;
  }
  use = c->premCond <= kPremCondMax;
  return E3D_OK;
}

int setPremultipliedAdjoint(Context* c, int on) {
  E3D_ARG(c && (on == 0 || on == 1), "bad adjoint state mode");
  c->premMode = on;
  return E3D_OK;
}

static Fields9& ringAt(std::vector<Fields9>& r, long long m) {
  const long long R = (long long)r.size();
  return r[(size_t)(((m % R) + R) % R)];
}

// Allocate a ring of `levels` levels whose first two are a and b; every level zeroed.
static int ensureRing(Context* c, std::vector<Fields9>& ring, Fields9& a, Fields9& b, int levels) {
  if (ring.empty()) {
    E3D_RET(allocFields(c, a, false));
    E3D_RET(allocFields(c, b, false));
    ring.push_back(a);
    ring.push_back(b);
    while ((int)ring.size() < levels) {
      Fields9 f;
      E3D_RET(allocFields(c, f, false));
      ring.push_back(f);
    }
  }
  E3D_ARG((int)ring.size() == levels, "ring size changed");
  for (auto& f : ring) E3D_RET(zeroFields(c, f));
  return E3D_OK;
}

// Source velocity of the block whose last fine level is mEnd (fine steps 1..sub
// are levels mEnd-sub+1..mEnd): the left part into vLeft (leftMode 1 added to
// the right part of the previous block already there, 2 written, 0 skipped)
// and the right part written into vRight (may be null).
static int launchDecimate(Context* c, long long mEnd, float* vLeft, int leftMode, float* vRight) {
  DecimatePtrs d{};
  const int sub = c->d.sub;
  d.nlev = sub;
  for (int t = 0; t < sub; t++) {
    Fields9& L = ringAt(c->srcRing, mEnd - sub + 1 + t);
    for (int k = 0; k < 3; k++) d.lev[t][k] = L.p[k];
    d.wl[t] = c->filt[t + 1];
    d.wr[t] = c->filt[c->hfilt + t + 1];
  }
  d.vl = leftMode ? vLeft : nullptr;
  d.vlMode = leftMode;
  d.vr = vRight;
  d.n = c->g.n;
  if (!d.vl && !d.vr) return E3D_OK;
  bool vec = c->g.n % 4 == 0;
  for (int t = 0; t < sub; t++)
    for (int k = 0; k < 3; k++) vec = vec && ((uintptr_t)d.lev[t][k] % 16 == 0);
  vec = vec && (!d.vl || (uintptr_t)d.vl % 16 == 0) && (!d.vr || (uintptr_t)d.vr % 16 == 0);
  const long long items = vec ? c->g.n / 4 : c->g.n;
  const unsigned gx = (unsigned)std::min<long long>((items + 255) / 256, (long long)c->numSMs * 8);
  c->launches++;
  TimedLaunch tl(c, 7);
  if (vec) kDecimateVelocity<true><<<dim3(gx, 3), 256, 0, c->st>>>(d);
  else kDecimateVelocity<false><<<dim3(gx, 3), 256, 0, c->st>>>(d);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

// Adjoint imaging of block its from the adjoint ring; the block's last fine
// level (it2 = 0) is mEnd, so level it2 is mEnd - it2.  v[0..3] = V(its-1..its+2).
// Halo and lead maps of the source velocities at the two coarse times a block images
// (time 0 absent without a left image: any valid field stands in, it is not loaded).
static int imagingVelocityMaps(Context* c, const ImagingBlockPtrs& q, CUtensorMap halo[2][3], CUtensorMap lead[2][3],
                               int itx = IMG_TX) {
  const CUtensorMap* m = nullptr;
  for (int t = 0; t < 2; t++)
    for (int k = 0; k < 3; k++) {
      const float* src = q.v[t + 1][k] ? q.v[t + 1][k] : q.v[2][k];
      E3D_RET(tensorMap(c, src, SZ, itx + 2 * HALO, &m));
      halo[t][k] = *m;
      E3D_RET(tensorMap(c, src, TZ, itx, &m));
      lead[t][k] = *m;
    }
  return E3D_OK;
}

// Block imaging with the levels and the medium staged by TMA (kImagingLev): ITX = 8, one CTA
// per SM; ITX = 4, three.
template <int NLEV, int ITX>
static int launchImagingLev(Context* c, const ImagingBlockPtrs& q, int tiz, int nyi) {
  constexpr int STAGES = imgLevStages(NLEV, ITX);
  constexpr size_t smem = (size_t)STAGES * imgLevStageF(NLEV, ITX) * sizeof(float);
  static std::atomic<unsigned long long> configured{0};
  E3D_RET(ensureSmemAttr((const void*)kImagingLev<NLEV, STAGES, ITX>, smem, configured));
  ImagingLevMaps<NLEV> mp;
  E3D_RET(imagingVelocityMaps(c, q, mp.halo, mp.lead, ITX));
  const CUtensorMap* m = nullptr;
  for (int j = 0; j < NLEV; j++)
    for (int k = 0; k < NCOMP; k++) {
      E3D_RET(tensorMap(c, q.lev[j][k], TZ, ITX, &m));
      mp.lev[j][k] = *m;
    }
  for (int k = 0; k < NMED; k++) {
    E3D_RET(tensorMap(c, q.med[k], TZ, ITX, &m));
    mp.med[k] = *m;
  }
  const int tix = (c->g.nx - 2 * FAT + ITX - 1) / ITX;
  const int perSM = ITX == 4 ? 3 : 1;
  const int chunks0 =
      c->imgChunks > 0 ? std::min(c->imgChunks, nyi) : chooseChunks(c, (long long)tiz * tix, nyi, perSM);
  const int yChunk = (nyi + chunks0 - 1) / chunks0;
  const int chunks = (nyi + yChunk - 1) / yChunk;
  kImagingLev<NLEV, STAGES, ITX><<<dim3(tiz, tix, chunks), dim3(TZ, ITX), smem, c->st>>>(mp, q, c->g, yChunk);
  return E3D_OK;
}

template <int ITX>
static int launchImagingLevSub(Context* c, const ImagingBlockPtrs& q, int tiz, int nyi, int sub) {
  switch (sub) {
    case 1: return launchImagingLev<1, ITX>(c, q, tiz, nyi);
    case 2: return launchImagingLev<2, ITX>(c, q, tiz, nyi);
    case 3: return launchImagingLev<3, ITX>(c, q, tiz, nyi);
    case 4: return launchImagingLev<4, ITX>(c, q, tiz, nyi);
    case 5: return launchImagingLev<5, ITX>(c, q, tiz, nyi);
    case 6: return launchImagingLev<6, ITX>(c, q, tiz, nyi);
    case 7: return launchImagingLev<7, ITX>(c, q, tiz, nyi);
    default: return launchImagingLev<8, ITX>(c, q, tiz, nyi);
  }
}

static int launchImagingBlock(Context* c, long long mEnd, float* const v[4], bool carryIn, bool leftImage,
                              Fields9& carry, bool prem) {
  ImagingBlockPtrs q{};
  q.prem = prem ? 1 : 0;
  for (int k = 0; k < NMED; k++) q.med[k] = c->med[k];
  const int sub = c->d.sub;
  q.nlev = sub;
  // in the order the fine steps ran (it2 = sub-1 first), as the fused decimation summed them
  for (int j = 0; j < sub; j++) {
    const int it2 = sub - 1 - j;
    Fields9& L = ringAt(c->adjRing, mEnd - it2);
    for (int k = 0; k < NCOMP; k++) q.lev[j][k] = L.p[k];
    q.wl[j] = c->filt[it2];
    q.wr[j] = c->filt[c->hfilt + it2];
  }
  const long long n = c->g.n;
  for (int t = 0; t < 4; t++)
    for (int k = 0; k < 3; k++) q.v[t][k] = vComp(v[t], k, n);
  for (int k = 0; k < NCOMP; k++) q.carry[k] = carry.p[k];
  q.carryIn = carryIn ? 1 : 0;
  q.leftImage = leftImage ? 1 : 0;
  for (int k = 0; k < NMED; k++) q.pert[k] = c->pertDev[k];
  q.dtsInv = c->dtsInv;
  q.q3compat = c->d.q3compat;
  c->launches++;
  TimedLaunch tl(c, 6);
  const bool tma = c->d.nz % 4 == 0 && c->loader >= 2;
  int variant = c->imgVariant;
  // automatic: the y-march with velocity tiles staged by TMA.  Measured on B200 in the 288^3
  // gradient: 1.46 ms per block against 1.88 ms with the levels staged too (one CTA per SM)
  if (variant == 0) variant = tma ? 2 : 1;
  if (variant >= 2 && c->d.nz % 4 != 0) variant = 1;  // the TMA forms need 16-byte rows
  const int tiz = (c->g.nz - 2 * FAT + TZ - 1) / TZ;
  const int tix = (c->g.nx - 2 * FAT + IMG_TX - 1) / IMG_TX;
  const int nyi = c->g.ny - 2 * FAT;
  if (variant == 3) {
    E3D_RET(launchImagingLevSub<8>(c, q, tiz, nyi, sub));
  } else if (variant == 4) {
    E3D_RET(launchImagingLevSub<4>(c, q, tiz, nyi, sub));
  } else if (variant == 2) {
    // y-marching TMA form: tensor maps of the velocity fields (cached per pointer)
    ImagingMaps mp;
    E3D_RET(imagingVelocityMaps(c, q, mp.halo, mp.lead));
    constexpr size_t smem = (size_t)2 * IMG_STAGE_F * sizeof(float);
    static std::atomic<unsigned long long> configured{0};
    E3D_RET(ensureSmemAttr((const void*)kImagingTma, smem, configured));
    const int chunks0 = c->imgChunks > 0 ? std::min(c->imgChunks, nyi) : chooseChunks(c, (long long)tiz * tix, nyi);
    const int yChunk = (nyi + chunks0 - 1) / chunks0;
    const int chunks = (nyi + yChunk - 1) / yChunk;
    kImagingTma<<<dim3(tiz, tix, chunks), dim3(TZ, IMG_TX), smem, c->st>>>(mp, q, c->g, yChunk);
  } else {
    dim3 block(32, 8);
    dim3 grid((c->d.nz - 2 * FAT + 31) / 32, (c->d.nx - 2 * FAT + 7) / 8, c->d.ny - 2 * FAT);
    kImagingBlock<<<grid, block, 0, c->st>>>(q, c->g);
  }
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

static int ensurePert(Context* c) {
  for (int k = 0; k < NMED; k++)
    if (!c->pertDev[k]) E3D_RET(devAlloc(c, (void**)&c->pertDev[k], (size_t)c->g.n * sizeof(float)));
  return E3D_OK;
}

// Born forward: the source propagation runs two coarse blocks ahead of the
// scattered propagation so that S[t] (needs V[t-1..t+1]) is ready when the
// scattered block t-1 starts.  Four velocity slots and two secondary-source
// slots rotate; nothing leaves the device.
static int bornForwardDevice(Context* c, const DevSignals& srcSet, const DevSignals& recSet, const float* srcSig,
                             float* recSig) {
  const int nts = c->d.nts, sub = c->d.sub;
  E3D_RET(allocFields(c, c->s0, true));
  E3D_RET(allocFields(c, c->s1, true));
  E3D_RET(allocFields(c, c->w0, true));
  E3D_RET(allocFields(c, c->w1, true));
  E3D_RET(allocFields(c, c->ss[0], true));
  E3D_RET(allocFields(c, c->ss[1], true));
  E3D_RET(ensureVSlots(c, 4));
  c->tailValid = false;  // the rotating slots overwrite a kept source segment
  for (int i = 0; i < 4; i++)
    E3D_CUDA_TRY(cudaMemsetAsync(c->vSlots[i], 0, (size_t)3 * c->g.n * sizeof(float), c->st));
  E3D_CUDA_TRY(cudaMemsetAsync(recSig, 0, (size_t)std::max(recSet.off[NCOMP], 1) * nts * sizeof(float), c->st));
  auto V = [&](int t) -> float* { return (t < 0 || t >= nts) ? nullptr : c->vSlots[t % 4]; };
  auto SS = [&](int t) -> Fields9& { return c->ss[t % 2]; };
  int nextS = 0;        // next secondary source to compute
  int nextScatter = 0;  // next scattered block
  auto scatterBlock = [&](int its) -> int {
    for (int it2 = 1; it2 <= sub; it2++) {
      StepPtrs p = makeStep(c, c->w0, c->w1);
      for (int k = 0; k < NCOMP; k++) {
        p.ssL[k] = SS(its).p[k];
        p.ssR[k] = SS(its + 1).p[k];
      }
      p.ssWl = c->filt[it2 - 1];
      p.ssWr = c->filt[c->hfilt + it2 - 1];
      E3D_RET(launchStep(c, STEP_FWD, p));
      E3D_RET(launchRecord(c, p, recSet, recSig, its, it2));
      swapF(c->w0, c->w1);
    }
    return E3D_OK;
  };
  auto computeS = [&](int t) -> int { return launchImaging(c, false, t, V(t - 1), V(t), V(t + 1), SS(t)); };
  for (int b = 0; b < nts - 1; b++) {
    // slot of V[b+1] was last used by V[b-3]; clear it before accumulating
    E3D_CUDA_TRY(cudaMemsetAsync(V(b + 1), 0, (size_t)3 * c->g.n * sizeof(float), c->st));
    E3D_RET(sourceBlock(c, b, srcSet, srcSig, V(b), V(b + 1)));
    // V[b] is complete: S[b-1] can be formed
    while (nextS <= b - 1) E3D_RET(computeS(nextS++));
    while (nextScatter + 1 < nextS) E3D_RET(scatterBlock(nextScatter++));
  }
  // tail: each S[t] overwrites S[t-2], so finish the scattered block that
  // still needs it before forming the next one
  while (nextS < nts) {
    E3D_RET(computeS(nextS++));
    while (nextScatter + 1 < nextS && nextScatter < nts - 1) E3D_RET(scatterBlock(nextScatter++));
  }
  while (nextScatter < nts - 1) E3D_RET(scatterBlock(nextScatter++));
  return E3D_OK;
}

// ---------------------------------------------------------------------------
// Checkpointed source wavefield for the Born adjoint / FWI gradient.
// The blocks are cut into segments of L blocks aligned to the END of the
// record: segment s covers [segStart(s), segStart(s+1)) and the first segment
// holds the remainder.  A checkpoint for segment s >= 1 holds the source-side
// state at the start of block segStart(s)-1; recomputing from it yields
// V[segStart(s)] complete (its right-weight part comes from that block).
// The forward pass decimates the last segment's velocity into the slots as it
// goes, so the adjoint pass recomputes every segment but the last (which is
// the longest, hence the end alignment).
// The plan (segment length, checkpoint storage, velocity-slot storage) is
// schedule::choosePlan's for the memory budget autoBudget gives.
// ---------------------------------------------------------------------------
enum { V_F32 = 0, V_F16 = 1 };

using schedule::segStart;

static size_t ckptBytesPerState(const Context* c, int type) {
  return (size_t)schedule::stateBytes(c->g.n, c->d.ny, type);
}
static size_t vHalfBytes(const Context* c) { return schedule::halfSlotValuesBytes(c->g.n); }
static size_t vStoreBytes(const Context* c) { return schedule::halfSlotBytes(c->g.n, c->d.ny); }
static double vSlotBytes(const Context* c, int vt) { return schedule::slotBytes(c->g.n, c->d.ny, vt); }

static double heldBytes(const Context* c) {
  double b = 0;
  for (void* p : c->ckpt)
    if (p) b += ckptBytesPerState(c, c->ckptAllocType);
  b += (double)c->vSlots.size() * vSlotBytes(c, V_F32) + (double)c->vStore.size() * vSlotBytes(c, V_F16);
  return b;
}

// Device bytes the adjoint pass will still allocate (adjoint levels, decimation
// slots, premultiplied levels).
static double pendingAdjointBytes(const Context* c) {
  const double f = (double)c->g.n * sizeof(float);
  double b = 0;
  const int R = ringLevels(c);
  if (R) {
    // the adjoint ring (w0, w1 and R-2 more levels) and the carried decimation
    if (c->adjRing.empty()) b += (double)(R - 2) * NCOMP * f + (c->w0.p[0] ? 0 : 18 * f);
    if (!c->ss[0].p[0]) b += NCOMP * f;
  } else {
    if (!c->w0.p[0]) b += 18 * f;
    if (!c->ss[0].p[0]) b += 18 * f;
  }
  const bool prem = R && c->premMode && c->premCond >= 0 && c->premCond <= kPremCondMax;
  if (!c->q0.p[0] && c->loader >= 2 && !prem) b += 18 * f;
  return b;
}

// Bytes available for checkpoints and velocity slots: the explicit budget, or
// 85% of the free memory left after the caller's reserve (negative budget)
// and the adjoint pass's pending allocations.
static double autoBudget(const Context* c, size_t free) {
  if (c->budget > 0) return c->budget;
  const double reserve = c->budget < 0 ? -c->budget : 0.0;
  return 0.85 * ((double)free - reserve) - pendingAdjointBytes(c);
}

static int choosePlan(Context* c, int& L) {
  size_t free = 0, total = 0;
  E3D_CUDA_TRY(cudaMemGetInfo(&free, &total));
  // memory this context already holds for checkpoints and velocity slots counts as available
  const double budget = autoBudget(c, free) + heldBytes(c);
  schedule::Plan plan{};
  if (!schedule::choosePlan(c->g.n, c->d.ny, c->d.nts, budget, c->ckptType, c->vType, c->segment, plan)) {
    setLastError("wavefield checkpoints do not fit in device memory", __FILE__, __LINE__);
    return E3D_ERR_OOM;
  }
  c->ckptUsed = plan.ck;
  c->vUsed = plan.vt;
  L = plan.L;
  return E3D_OK;
}

static int resizeVStorage(Context* c, int nF32, int nF16) {
  while ((int)c->vSlots.size() > nF32) {
    devFree(c, c->vSlots.back());
    c->vSlots.pop_back();
  }
  while ((int)c->vStore.size() > nF16) {
    devFree(c, c->vStore.back());
    c->vStore.pop_back();
  }
  E3D_RET(ensureVSlots(c, nF32));
  while ((int)c->vStore.size() < nF16) {
    void* p = nullptr;
    E3D_RET(devAlloc(c, &p, vStoreBytes(c)));
    c->vStore.push_back(p);
  }
  return E3D_OK;
}

// Grid of the slice kernels for nf consecutive fields: each block covers
// kSliceThreads * kSliceVecPerThread * 4 values of one y slice.
static dim3 sliceGrid(const Context* c, int nf) {
  const long long per = (long long)kSliceThreads * kSliceVecPerThread * 4;
  return dim3((unsigned)((c->g.yStride + per - 1) / per), (unsigned)c->d.ny, (unsigned)nf);
}

// Four-wide slice access: slices and fields start on 4-value boundaries and
// the FP32 and 16-bit arrays are 16- and 8-byte aligned.
static bool sliceVec(const Context* c, const void* f32, const void* h16) {
  return c->g.yStride % 4 == 0 && c->g.n % 4 == 0 && (uintptr_t)f32 % 16 == 0 && (uintptr_t)h16 % 8 == 0;
}

// Scaled 16-bit copy of nf consecutive fields of n values: slice maxima into
// the scratch, then the packed values and one unscaling factor per (field, y).
template <typename H>
static int packSlices(Context* c, const float* a, int nf, int topExp, H* out, float* scales) {
  const long long n = c->g.n, ys = c->g.yStride;
  float* smax = (float*)c->scratch;
  const dim3 grid = sliceGrid(c, nf);
  const bool vec = sliceVec(c, a, out);
  E3D_CUDA_TRY(cudaMemsetAsync(smax, 0, (size_t)nf * c->d.ny * sizeof(float), c->st));
  c->launches += 2;
  if (vec) kSliceMaxAbs<true><<<grid, kSliceThreads, 0, c->st>>>(a, n, ys, smax);
  else kSliceMaxAbs<false><<<grid, kSliceThreads, 0, c->st>>>(a, n, ys, smax);
  E3D_LAUNCH_CHECK();
  if (vec) kPackSlices<H, true><<<grid, kSliceThreads, 0, c->st>>>(a, n, ys, smax, topExp, out, scales);
  else kPackSlices<H, false><<<grid, kSliceThreads, 0, c->st>>>(a, n, ys, smax, topExp, out, scales);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

template <typename H>
static int unpackSlices(Context* c, const H* in, int nf, const float* scales, float* a) {
  const long long n = c->g.n, ys = c->g.yStride;
  const dim3 grid = sliceGrid(c, nf);
  c->launches++;
  if (sliceVec(c, a, in)) kUnpackSlices<H, true><<<grid, kSliceThreads, 0, c->st>>>(in, n, ys, scales, a);
  else kUnpackSlices<H, false><<<grid, kSliceThreads, 0, c->st>>>(in, n, ys, scales, a);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

// Per-(field, y-slice) scaled FP16 copy of the three velocity fields of slot v.
static int packVelocity(Context* c, const float* v, void* store) {
  float* scales = (float*)((char*)store + vHalfBytes(c));
  return packSlices(c, v, 3, 14, (__half*)store, scales);
}

static int unpackVelocity(Context* c, const void* store, float* v) {
  const float* scales = (const float*)((const char*)store + vHalfBytes(c));
  return unpackSlices(c, (const __half*)store, 3, scales, v);
}

static int packState(Context* c, int seg) {
  const long long n = c->g.n;
  const int ny = c->d.ny;
  Fields9* parts[2] = {&c->s0, &c->s1};
  if (c->ckptUsed == CKPT_F32) {
    float* dst = (float*)c->ckpt[seg];
    for (int h = 0; h < 2; h++)
      for (int k = 0; k < NCOMP; k++)
        E3D_CUDA_TRY(cudaMemcpyAsync(dst + (size_t)(h * NCOMP + k) * n, parts[h]->p[k], n * sizeof(float),
                                     cudaMemcpyDeviceToDevice, c->st));
    return E3D_OK;
  }
  float* scales = c->ckptScale[seg];
  for (int h = 0; h < 2; h++)
    for (int k = 0; k < NCOMP; k++) {
      const int f = h * NCOMP + k;
      if (c->ckptUsed == CKPT_F16)
        E3D_RET(packSlices(c, parts[h]->p[k], 1, 14, (__half*)c->ckpt[seg] + (size_t)f * n, scales + (size_t)f * ny));
      else
        E3D_RET(packSlices(c, parts[h]->p[k], 1, 0, (__nv_bfloat16*)c->ckpt[seg] + (size_t)f * n,
                           scales + (size_t)f * ny));
    }
  return E3D_OK;
}

static int unpackState(Context* c, int seg) {
  const long long n = c->g.n;
  const int ny = c->d.ny;
  Fields9* parts[2] = {&c->s0, &c->s1};
  for (int h = 0; h < 2; h++)
    for (int k = 0; k < NCOMP; k++) {
      const int f = h * NCOMP + k;
      if (c->ckptUsed == CKPT_F32)
        E3D_CUDA_TRY(cudaMemcpyAsync(parts[h]->p[k], (float*)c->ckpt[seg] + (size_t)f * n, n * sizeof(float),
                                     cudaMemcpyDeviceToDevice, c->st));
      else if (c->ckptUsed == CKPT_F16)
        E3D_RET(unpackSlices(c, (const __half*)c->ckpt[seg] + (size_t)f * n, 1, c->ckptScale[seg] + (size_t)f * ny,
                             parts[h]->p[k]));
      else
        E3D_RET(unpackSlices(c, (const __nv_bfloat16*)c->ckpt[seg] + (size_t)f * n, 1,
                             c->ckptScale[seg] + (size_t)f * ny, parts[h]->p[k]));
    }
  return E3D_OK;
}

static int prepareCheckpoints(Context* c, int& L, int& nseg) {
  const int blocks = c->d.nts - 1;
  E3D_RET(choosePlan(c, L));
  nseg = (blocks + L - 1) / L;
  if (c->ckptSegLen != L || (int)c->ckpt.size() != nseg || c->ckptAllocType != c->ckptUsed ||
      c->vAllocType != c->vUsed) {
    for (void* p : c->ckpt) devFree(c, p);
    for (float* p : c->ckptScale) devFree(c, p);
    c->ckpt.assign(nseg, nullptr);
    c->ckptScale.assign(nseg, nullptr);
    c->ckptAllocType = c->ckptUsed;
    E3D_RET(resizeVStorage(c, c->vUsed == V_F32 ? L + 3 : 4, c->vUsed == V_F32 ? 0 : L + 2));
    c->vAllocType = c->vUsed;
    for (int s = 1; s < nseg; s++) {
      const size_t eb = c->ckptUsed == CKPT_F32 ? 4 : 2;
      E3D_RET(devAlloc(c, &c->ckpt[s], (size_t)18 * c->g.n * eb));
      if (c->ckptUsed != CKPT_F32)
        E3D_RET(devAlloc(c, (void**)&c->ckptScale[s], (size_t)18 * c->d.ny * sizeof(float)));
    }
    c->ckptSegLen = L;
  }
  E3D_RET(scratchAtLeast(c, (size_t)3 * c->d.ny * sizeof(float)));  // slice maxima of three fields
  return E3D_OK;
}

// Receiver slices between the regular acquisition points and irregular traces.
static int traceRingAtLeast(Context* c, size_t floats) {
  if (c->traceRingFloats >= floats) return E3D_OK;
  devFree(c, c->traceRing);
  c->traceRing = nullptr;
  c->traceRingFloats = 0;
  E3D_RET(devAlloc(c, (void**)&c->traceRing, std::max<size_t>(floats, 1) * sizeof(float)));
  c->traceRingFloats = floats;
  return E3D_OK;
}

static int traceGather(Context* c, const TraceMap& m, int nReg, const float* reg, float* irr) {
  const int rows = NCOMP * m.nIrreg;
  if (rows == 0) return E3D_OK;
  c->launches++;
  kTraceGather<<<(rows + 127) / 128, 128, 0, c->st>>>(reg, irr, rows, m.nTaps, m.slot, m.weight, nReg);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

static int traceSpread(Context* c, const TraceMap& m, int nReg, const float* irr, float* reg) {
  if (nReg == 0) return E3D_OK;
  c->launches++;
  kTraceSpread<<<(nReg + 127) / 128, 128, 0, c->st>>>(irr, reg, nReg, m.rowPtr, m.idx, m.w, NCOMP * m.nIrreg);
  E3D_LAUNCH_CHECK();
  return E3D_OK;
}

// Source-side forward pass over all coarse blocks, saving the state at the
// start of block segStart(s)-1 for every segment s >= 1 and decimating the
// velocity of the last segment into the velocity slots (the adjoint pass
// then starts without recomputing it).  When recSig is non-null the
// receivers are recorded too (this is the nonlinear forward of FWI): into a
// time-major regular-grid array, or, with a trace map, through a two-slice
// ring converted to irregular traces as each coarse slice completes.
static int sourcePassRing(Context* c, const DevSignals& srcSet, const DevSignals* recSet, const float* srcSig,
                          float* recSig, const TraceMap* map);

static int sourcePassWithCheckpoints(Context* c, const DevSignals& srcSet, const DevSignals* recSet,
                                     const float* srcSig, float* recSig, const TraceMap* map) {
  if (ringLevels(c)) return sourcePassRing(c, srcSet, recSet, srcSig, recSig, map);
  int L = 0, nseg = 0;
  c->ckptValid = false;
  c->tailValid = false;
  E3D_RET(prepareCheckpoints(c, L, nseg));
  E3D_RET(allocFields(c, c->s0, true));
  E3D_RET(allocFields(c, c->s1, true));
  const int nts = c->d.nts, sub = c->d.sub, blocks = nts - 1;
  const long long n = c->g.n;
  const size_t nr = recSet ? (size_t)recSet->off[NCOMP] : 0;
  const size_t rows = map ? (size_t)NCOMP * map->nIrreg : 0;
  float* ring = nullptr;
  if (recSig && map) {
    E3D_RET(traceRingAtLeast(c, 2 * nr));
    ring = c->traceRing;
    E3D_CUDA_TRY(cudaMemsetAsync(ring, 0, std::max<size_t>(2 * nr, 1) * sizeof(float), c->st));
  } else if (recSig) {
    E3D_CUDA_TRY(cudaMemsetAsync(recSig, 0, std::max<size_t>(nr, 1) * nts * sizeof(float), c->st));
  }
  // the last segment's velocity V[tailBeg .. nts-1], laid out as the adjoint
  // pass's recomputation lays it out (FP32: one slot per time; FP16: a
  // two-slot FP32 ring packed into the FP16 slots as each time completes)
  const bool vc = c->vUsed == V_F16;
  const int tailBeg = segStart(blocks, L, nseg, nseg - 1);
  auto A = [&](int t) -> float* {
    if (t < tailBeg || t >= nts) return nullptr;
    return vc ? c->vSlots[(t - tailBeg) % 2] : c->vSlots[t - tailBeg];
  };
  const int nClear = vc ? 2 : nts - tailBeg;
  for (int i = 0; i < nClear; i++)
    E3D_CUDA_TRY(cudaMemsetAsync(c->vSlots[i], 0, (size_t)3 * n * sizeof(float), c->st));
  int nextCk = 1;
  for (int b = 0; b < blocks; b++) {
    if (nextCk < nseg && b == segStart(blocks, L, nseg, nextCk) - 1) E3D_RET(packState(c, nextCk++));
    const bool decimate = b >= tailBeg - 1;  // block tailBeg-1 feeds V[tailBeg] through its right weights
    for (int it2 = 1; it2 <= sub; it2++) {
      StepPtrs p = makeStep(c, c->s0, c->s1);
      if (decimate) setSourceAcc(c, p, it2, A(b), A(b + 1));
      E3D_RET(launchStep(c, STEP_FWD, p));
      E3D_RET(launchInject(c, p, srcSet, srcSig, b, it2 - 1));
      if (ring) E3D_RET(launchRecordSlices(c, p, *recSet, ring + (b % 2) * nr, ring + ((b + 1) % 2) * nr, it2));
      else if (recSig) E3D_RET(launchRecord(c, p, *recSet, recSig, b, it2));
      swapF(c->s0, c->s1);
    }
    if (vc && b >= tailBeg) {
      // V[b] is complete: store it and reuse its slot for V[b+2]
      E3D_RET(packVelocity(c, A(b), c->vStore[b - tailBeg]));
      E3D_CUDA_TRY(cudaMemsetAsync(A(b), 0, (size_t)3 * n * sizeof(float), c->st));
    }
    if (ring) {
      // slice b is complete; its ring slot is reused for slice b+2
      E3D_RET(traceGather(c, *map, (int)nr, ring + (b % 2) * nr, recSig + (size_t)b * rows));
      if (nr) E3D_CUDA_TRY(cudaMemsetAsync(ring + (b % 2) * nr, 0, nr * sizeof(float), c->st));
    }
  }
  // V[nts-1] has no block of its own: complete after block nts-2
  if (vc) E3D_RET(packVelocity(c, A(nts - 1), c->vStore[nts - 1 - tailBeg]));
  if (ring) E3D_RET(traceGather(c, *map, (int)nr, ring + ((nts - 1) % 2) * nr, recSig + (size_t)(nts - 1) * rows));
  c->ckptValid = true;
  c->tailValid = true;
  return E3D_OK;
}

// Adjoint pass (BornElasticAdjGpu_3D phase B) consuming the checkpoints:
// segments are processed last to first; each recomputes its velocity slots
// from its checkpoint (the last one only when the forward pass's copy has been
// overwritten since), then runs its adjoint blocks and imaging.  With a
// trace map the residual is irregular and time-major; each coarse slice is
// spread to the regular acquisition points just before the block that
// injects it.
static int adjointPassRing(Context* c, const DevSignals& srcSet, const DevSignals& recSet, const float* srcSig,
                           const float* resid, const TraceMap* map, float* srcAdj);

static int adjointPassFromCheckpoints(Context* c, const DevSignals& srcSet, const DevSignals& recSet,
                                      const float* srcSig, const float* resid, const TraceMap* map,
                                      float* srcAdj = nullptr) {
  E3D_ARG(c->ckptValid, "no checkpoints for this shot");
  if (ringLevels(c)) return adjointPassRing(c, srcSet, recSet, srcSig, resid, map, srcAdj);
  const int nts = c->d.nts, sub = c->d.sub, L = c->ckptSegLen;
  const int blocks = nts - 1;
  const int nseg = (blocks + L - 1) / L;
  const long long n = c->g.n;
  const bool vc = c->vUsed == V_F16;
  E3D_RET(resizeVStorage(c, std::max<int>(vc ? 4 : L + 3, (int)c->vSlots.size()),
                         std::max<int>(vc ? L + 2 : 0, (int)c->vStore.size())));
  E3D_RET(allocFields(c, c->w0, true));
  E3D_RET(allocFields(c, c->w1, true));
  E3D_RET(allocFields(c, c->ss[0], true));
  E3D_RET(allocFields(c, c->ss[1], true));
  // the TMA stepper runs the exact adjoint on a dual state (raw + premultiplied)
  const bool dual = c->loader >= 2 && c->d.nz % 4 == 0;
  if (dual) {
    E3D_RET(allocFields(c, c->q0, true));
    E3D_RET(allocFields(c, c->q1, true));
  }
  const size_t nr = (size_t)recSet.off[NCOMP];
  const size_t rows = map ? (size_t)NCOMP * map->nIrreg : 0;
  if (srcAdj)
    E3D_CUDA_TRY(cudaMemsetAsync(srcAdj, 0, (size_t)std::max(srcSet.off[NCOMP], 1) * nts * sizeof(float), c->st));
  if (map) {
    E3D_RET(traceRingAtLeast(c, 2 * nr));
    E3D_RET(traceSpread(c, *map, (int)nr, resid + (size_t)(nts - 1) * rows, c->traceRing + ((nts - 1) % 2) * nr));
  }
  auto dataSlice = [&](int t) -> const float* {
    return map ? c->traceRing + (t % 2) * nr : resid + (size_t)t * nr;
  };
  // adjoint decimation slots: A[its] (left, fresh per block) and A[its+1] (right)
  Fields9* aLeft = &c->ss[0];
  Fields9* aRight = &c->ss[1];
  int winStart = 0;
  // FP32 velocity of coarse time t for the imaging condition
  auto V = [&](int t) -> float* {
    if (t < 0 || t >= nts) return nullptr;
    if (vc) return c->vSlots[t % 3];
    const int i = t - winStart;
    return (i >= 0 && i < (int)c->vSlots.size()) ? c->vSlots[i] : nullptr;
  };
  // accumulation slot of V[t] while the segment is recomputed
  auto A = [&](int t) -> float* {
    if (t < 0 || t >= nts) return nullptr;
    return vc ? c->vSlots[(t - winStart) % 2] : c->vSlots[t - winStart];
  };
  // the forward pass left the last segment's velocity in the slots; processing
  // any earlier segment overwrites them
  const bool tailKept = c->tailValid;
  if (nseg > 1) c->tailValid = false;
  for (int s = nseg - 1; s >= 0; s--) {
    const int bBeg = segStart(blocks, L, nseg, s);
    const int bEnd = segStart(blocks, L, nseg, s + 1);  // adjoint blocks [bBeg, bEnd)
    const int lastBlock = std::min(bEnd + 1, blocks - 1);
    winStart = bBeg;
    if (!(tailKept && s == nseg - 1)) {
      // recompute V[bBeg .. min(bEnd+1, nts-1)] from the checkpoint
      const int nClear = vc ? 2 : std::min(bEnd + 2, nts - 1) - bBeg + 1;
      for (int i = 0; i < nClear; i++)
        E3D_CUDA_TRY(cudaMemsetAsync(c->vSlots[i], 0, (size_t)3 * n * sizeof(float), c->st));
      int firstBlock = 0;
      if (s == 0) {
        E3D_RET(zeroFields(c, c->s0));
        E3D_RET(zeroFields(c, c->s1));
      } else {
        E3D_RET(unpackState(c, s));
        // block bBeg-1 only feeds V[bBeg] through its right weights
        E3D_RET(sourceBlock(c, bBeg - 1, srcSet, srcSig, nullptr, A(bBeg)));
        firstBlock = bBeg;
      }
      for (int b = firstBlock; b <= lastBlock; b++) {
        E3D_RET(sourceBlock(c, b, srcSet, srcSig, A(b), A(b + 1)));
        if (vc) {
          // V[b] is complete: store it and reuse its slot for V[b+2]
          E3D_RET(packVelocity(c, A(b), c->vStore[b - bBeg]));
          E3D_CUDA_TRY(cudaMemsetAsync(A(b), 0, (size_t)3 * n * sizeof(float), c->st));
        }
      }
      // V[nts-1] has no block of its own: complete after block nts-2
      if (vc && lastBlock + 1 == nts - 1 && nts - 1 <= bEnd + 1)
        E3D_RET(packVelocity(c, A(nts - 1), c->vStore[nts - 1 - bBeg]));
    }
    if (vc)
      for (int t = bEnd; t <= std::min(bEnd + 1, nts - 1); t++)
        E3D_RET(unpackVelocity(c, c->vStore[t - bBeg], V(t)));
    // adjoint blocks, last to first
    for (int its = bEnd - 1; its >= bBeg; its--) {
      if (vc) E3D_RET(unpackVelocity(c, c->vStore[its - bBeg], V(its)));
      if (map) E3D_RET(traceSpread(c, *map, (int)nr, resid + (size_t)its * rows, c->traceRing + (its % 2) * nr));
      for (int it2 = sub - 1; it2 >= 0; it2--) {
        StepPtrs p = makeStep(c, c->w0, c->w1);
        for (int k = 0; k < NCOMP; k++) {
          p.accL[k] = aLeft->p[k];
          p.accR[k] = aRight->p[k];
        }
        p.accWl = c->filt[it2];
        p.accWr = c->filt[c->hfilt + it2];
        p.nAcc = NCOMP;
        if (dual) {
          for (int k = 0; k < NCOMP; k++) {
            p.c[k] = c->q1.p[k];
            p.oP[k] = c->q0.p[k];
          }
        }
        // A[its] starts with this block: the TMA stepper writes it on the first
        // fine step instead of accumulating onto a cleared slot
        if (it2 == sub - 1) {
          if (dual) p.accInitL = 1;
          else E3D_RET(zeroFields(c, *aLeft));
        }
        E3D_RET(launchStep(c, STEP_ADJ_EXACT, p));
        E3D_RET(launchInjectSlices(c, p, recSet, dataSlice(its), dataSlice(its + 1), it2 + 1));
        if (dual) E3D_RET(launchRefresh(c, p, recSet));
        // transpose of the source injection of forward step (its, it2+1): the exact
        // adjoint of the nonlinear propagation with respect to the scaled source signals
        if (srcAdj) E3D_RET(launchExtractSource(c, p, srcSet, srcAdj, its, it2));
        swapF(c->w0, c->w1);
        if (dual) swapF(c->q0, c->q1);
      }
      // imaging condition at its+1 (A[its+1] complete)
      E3D_RET(launchImaging(c, true, its + 1, V(its), V(its + 1), V(its + 2), *aRight));
      std::swap(aLeft, aRight);  // A[its] becomes the right accumulator of block its-1
    }
  }
  // final imaging at t = 0 (uses V[0], V[1] of the first segment window)
  E3D_RET(launchImaging(c, true, 0, nullptr, V(0), V(1), *aRight));
  return E3D_OK;
}

// ---------------------------------------------------------------------------
// The checkpointed passes with rings of fine levels (the same schedule, loop
// order and checkpoints as the two functions above; only the decimation
// moves out of the stepper into one launch per coarse block).
// ---------------------------------------------------------------------------

// One coarse block (its) of the source-side forward propagation on the source
// ring from level m, injecting srcSig; then the block's velocity decimated
// into vLeft (leftMode as launchDecimate) and vRight.  m advances by sub.
static int sourceBlockRing(Context* c, long long& m, int its, const DevSignals& srcSet, const float* srcSig,
                           float* vLeft, int leftMode, float* vRight) {
  auto S = [&](long long k) -> Fields9& { return ringAt(c->srcRing, k); };
  for (int it2 = 1; it2 <= c->d.sub; it2++) {
    StepPtrs p = makeRingStep(c, S(m - 1), S(m), S(m + 1));
    E3D_RET(launchStep(c, STEP_FWD, p));
    E3D_RET(launchInject(c, afterStep(p), srcSet, srcSig, its, it2 - 1));
    m++;
  }
  if ((vLeft && leftMode) || vRight) E3D_RET(launchDecimate(c, m, vLeft, leftMode, vRight));
  c->s0 = S(m - 1);
  c->s1 = S(m);
  return E3D_OK;
}

static int sourcePassRing(Context* c, const DevSignals& srcSet, const DevSignals* recSet, const float* srcSig,
                          float* recSig, const TraceMap* map) {
  int L = 0, nseg = 0;
  c->ckptValid = false;
  c->tailValid = false;
  // the ring is allocated before the plan, so that the free memory the plan sees excludes it
  E3D_RET(ensureRing(c, c->srcRing, c->s0, c->s1, ringLevels(c)));
  {
    bool prem = false;  // known before the plan, which then leaves out the dual state's levels
    E3D_RET(premultipliedAdjoint(c, prem));
  }
  E3D_RET(prepareCheckpoints(c, L, nseg));
  const int nts = c->d.nts, sub = c->d.sub, blocks = nts - 1;
  const size_t nr = recSet ? (size_t)recSet->off[NCOMP] : 0;
  const size_t rows = map ? (size_t)NCOMP * map->nIrreg : 0;
  float* ring = nullptr;
  if (recSig && map) {
    E3D_RET(traceRingAtLeast(c, 2 * nr));
    ring = c->traceRing;
    E3D_CUDA_TRY(cudaMemsetAsync(ring, 0, std::max<size_t>(2 * nr, 1) * sizeof(float), c->st));
  } else if (recSig) {
    E3D_CUDA_TRY(cudaMemsetAsync(recSig, 0, std::max<size_t>(nr, 1) * nts * sizeof(float), c->st));
  }
  // the last segment's velocity V[tailBeg .. nts-1] (FP32: one slot per time;
  // FP16: a two-slot FP32 ring packed into the FP16 slots as each time completes)
  const bool vc = c->vUsed == V_F16;
  const int tailBeg = segStart(blocks, L, nseg, nseg - 1);
  auto A = [&](int t) -> float* {
    if (t < tailBeg || t >= nts) return nullptr;
    return vc ? c->vSlots[(t - tailBeg) % 2] : c->vSlots[t - tailBeg];
  };
  auto S = [&](long long k) -> Fields9& { return ringAt(c->srcRing, k); };
  long long m = 0;  // levels -1 and 0 are the zero initial state
  int nextCk = 1;
  for (int b = 0; b < blocks; b++) {
    if (nextCk < nseg && b == segStart(blocks, L, nseg, nextCk) - 1) {
      c->s0 = S(m - 1);
      c->s1 = S(m);
      E3D_RET(packState(c, nextCk++));
    }
    for (int it2 = 1; it2 <= sub; it2++) {
      StepPtrs p = makeRingStep(c, S(m - 1), S(m), S(m + 1));
      E3D_RET(launchStep(c, STEP_FWD, p));
      const StepPtrs q = afterStep(p);
      E3D_RET(launchInject(c, q, srcSet, srcSig, b, it2 - 1));
      if (ring) E3D_RET(launchRecordSlices(c, q, *recSet, ring + (b % 2) * nr, ring + ((b + 1) % 2) * nr, it2));
      else if (recSig) E3D_RET(launchRecord(c, q, *recSet, recSig, b, it2));
      m++;
    }
    // block tailBeg-1 feeds V[tailBeg] through its right weights only; V[0] has no earlier block
    if (b >= tailBeg - 1) E3D_RET(launchDecimate(c, m, A(b), b < tailBeg ? 0 : (b == 0 ? 2 : 1), A(b + 1)));
    if (vc && b >= tailBeg) {
      // V[b] is complete: store it; its slot next receives V[b+2], written by block b+1
      E3D_RET(packVelocity(c, A(b), c->vStore[b - tailBeg]));
    }
    if (ring) {
      // slice b is complete; its ring slot is reused for slice b+2
      E3D_RET(traceGather(c, *map, (int)nr, ring + (b % 2) * nr, recSig + (size_t)b * rows));
      if (nr) E3D_CUDA_TRY(cudaMemsetAsync(ring + (b % 2) * nr, 0, nr * sizeof(float), c->st));
    }
  }
  // V[nts-1] has no block of its own: complete after block nts-2
  if (vc) E3D_RET(packVelocity(c, A(nts - 1), c->vStore[nts - 1 - tailBeg]));
  if (ring) E3D_RET(traceGather(c, *map, (int)nr, ring + ((nts - 1) % 2) * nr, recSig + (size_t)(nts - 1) * rows));
  c->s0 = S(m - 1);
  c->s1 = S(m);
  c->ckptValid = true;
  c->tailValid = true;
  return E3D_OK;
}

// Adjoint pass with the adjoint levels in a ring: after the last fine step of
// block its, one launch decimates its levels into the right part R (coarse
// sample its+1) and the left part L (its) and images both.  V(its-1) belongs
// to the segment's window except at its first block, whose L is carried to the
// next block processed (the last block of the previous segment), as the fused
// decimation carried its accumulator.
static int adjointPassRing(Context* c, const DevSignals& srcSet, const DevSignals& recSet, const float* srcSig,
                           const float* resid, const TraceMap* map, float* srcAdj) {
  const int nts = c->d.nts, sub = c->d.sub, L = c->ckptSegLen;
  const int blocks = nts - 1;
  const int nseg = (blocks + L - 1) / L;
  const bool vc = c->vUsed == V_F16;
  E3D_RET(resizeVStorage(c, std::max<int>(vc ? 4 : L + 3, (int)c->vSlots.size()),
                         std::max<int>(vc ? L + 2 : 0, (int)c->vStore.size())));
  E3D_RET(ensureRing(c, c->adjRing, c->w0, c->w1, ringLevels(c)));
  Fields9& carry = c->ss[0];
  E3D_RET(allocFields(c, carry, true));  // L of the block after the last one: zero
  const bool dual = c->loader >= 2 && c->d.nz % 4 == 0;
  // the premultiplied-only state: the ring holds premultiplied levels and no raw level is kept
  bool prem = false;
  const int ncn = recSet.off[SXX + 1] - recSet.off[SXX];
  if (dual && !srcAdj && recSet.off[SYY + 1] - recSet.off[SYY] == ncn && recSet.off[SZZ + 1] - recSet.off[SZZ] == ncn)
    E3D_RET(premultipliedAdjoint(c, prem));
  if (dual && !prem) {
    E3D_RET(allocFields(c, c->q0, true));
    E3D_RET(allocFields(c, c->q1, true));
  }
  const size_t nr = (size_t)recSet.off[NCOMP];
  const size_t rows = map ? (size_t)NCOMP * map->nIrreg : 0;
  if (srcAdj)
    E3D_CUDA_TRY(cudaMemsetAsync(srcAdj, 0, (size_t)std::max(srcSet.off[NCOMP], 1) * nts * sizeof(float), c->st));
  if (map) {
    E3D_RET(traceRingAtLeast(c, 2 * nr));
    E3D_RET(traceSpread(c, *map, (int)nr, resid + (size_t)(nts - 1) * rows, c->traceRing + ((nts - 1) % 2) * nr));
  }
  auto dataSlice = [&](int t) -> const float* {
    return map ? c->traceRing + (t % 2) * nr : resid + (size_t)t * nr;
  };
  int winStart = 0, winEnd = -1;  // velocity window [winStart, winEnd] of the current segment
  int held[4] = {-1, -1, -1, -1};  // FP16 slots: the time unpacked in FP32 slot t % 4
  // FP32 velocity of coarse time t for the imaging condition
  auto V = [&](int t) -> float* {
    if (t < 0 || t >= nts) return nullptr;
    if (vc) return held[t % 4] == t ? c->vSlots[t % 4] : nullptr;
    const int i = t - winStart;
    return (i >= 0 && i < (int)c->vSlots.size()) ? c->vSlots[i] : nullptr;
  };
  auto unpackV = [&](int t) -> int {
    if (!vc || t < winStart || t > winEnd || held[t % 4] == t) return E3D_OK;
    E3D_RET(unpackVelocity(c, c->vStore[t - winStart], c->vSlots[t % 4]));
    held[t % 4] = t;
    return E3D_OK;
  };
  // accumulation slot of V[t] while the segment is recomputed
  auto Acc = [&](int t) -> float* {
    if (t < 0 || t >= nts) return nullptr;
    return vc ? c->vSlots[(t - winStart) % 2] : c->vSlots[t - winStart];
  };
  auto W = [&](long long k) -> Fields9& { return ringAt(c->adjRing, k); };
  long long ma = 0;  // adjoint levels -1 and 0: the zero final state
  const bool tailKept = c->tailValid;
  if (nseg > 1) c->tailValid = false;
  for (int s = nseg - 1; s >= 0; s--) {
    const int bBeg = segStart(blocks, L, nseg, s);
    const int bEnd = segStart(blocks, L, nseg, s + 1);  // adjoint blocks [bBeg, bEnd)
    const int lastBlock = std::min(bEnd + 1, blocks - 1);
    winStart = bBeg;
    winEnd = std::min(bEnd + 1, nts - 1);
    if (!(tailKept && s == nseg - 1)) {
      // recompute V[bBeg .. min(bEnd+1, nts-1)] from the checkpoint
      long long m = 0;
      int firstBlock = 0;
      auto S = [&](long long k) -> Fields9& { return ringAt(c->srcRing, k); };
      if (s == 0) {
        E3D_RET(zeroFields(c, S(-1)));
        E3D_RET(zeroFields(c, S(0)));
      } else {
        c->s0 = S(-1);
        c->s1 = S(0);
        E3D_RET(unpackState(c, s));
        // block bBeg-1 only feeds V[bBeg] through its right weights
        E3D_RET(sourceBlockRing(c, m, bBeg - 1, srcSet, srcSig, nullptr, 0, Acc(bBeg)));
        firstBlock = bBeg;
      }
      for (int b = firstBlock; b <= lastBlock; b++) {
        E3D_RET(sourceBlockRing(c, m, b, srcSet, srcSig, Acc(b), b == 0 ? 2 : 1, Acc(b + 1)));
        // V[b] is complete: store it; its slot next receives V[b+2], written by block b+1
        if (vc) E3D_RET(packVelocity(c, Acc(b), c->vStore[b - bBeg]));
      }
      // V[nts-1] has no block of its own: complete after block nts-2
      if (vc && lastBlock + 1 == nts - 1 && nts - 1 <= bEnd + 1)
        E3D_RET(packVelocity(c, Acc(nts - 1), c->vStore[nts - 1 - bBeg]));
    }
    for (int i = 0; i < 4; i++) held[i] = -1;  // the recompute used the FP32 slots
    // adjoint blocks, last to first
    for (int its = bEnd - 1; its >= bBeg; its--) {
      const bool leftImage = its > bBeg;
      for (int t = its + 2; t >= (leftImage ? its - 1 : its); t--) E3D_RET(unpackV(t));
      if (map) E3D_RET(traceSpread(c, *map, (int)nr, resid + (size_t)its * rows, c->traceRing + (its % 2) * nr));
      for (int it2 = sub - 1; it2 >= 0; it2--) {
        StepPtrs p = makeRingStep(c, W(ma - 1), W(ma), W(ma + 1));
        if (dual && !prem) {
          for (int k = 0; k < NCOMP; k++) {
            p.c[k] = c->q1.p[k];
            p.oP[k] = c->q0.p[k];
          }
        }
        // On premultiplied levels P = M a the exact adjoint's update
        // a_new = G (G a_old - D(P_cur)), P_new = M a_new reads
        // P_new = G (G P_old - M D(P_cur)) with M applied term by term: the
        // time-reversed stepper (stepAdjGpu_3D's update) on P.
        E3D_RET(launchStep(c, prem ? STEP_ADJ_REVERSED : STEP_ADJ_EXACT, p));
        const StepPtrs q = afterStep(p);
        if (prem) E3D_RET(launchInjectPremultiplied(c, q, recSet, dataSlice(its), dataSlice(its + 1), it2 + 1));
        else if (dual) E3D_RET(launchInjectRefresh(c, q, recSet, dataSlice(its), dataSlice(its + 1), it2 + 1));
        else E3D_RET(launchInjectSlices(c, q, recSet, dataSlice(its), dataSlice(its + 1), it2 + 1));
        // transpose of the source injection of forward step (its, it2+1): the exact
        // adjoint of the nonlinear propagation with respect to the scaled source signals
        if (srcAdj) E3D_RET(launchExtractSource(c, q, srcSet, srcAdj, its, it2));
        ma++;
        if (dual && !prem) swapF(c->q0, c->q1);
      }
      float* const v[4] = {leftImage ? V(its - 1) : nullptr, V(its), V(its + 1), V(its + 2)};
      E3D_RET(launchImagingBlock(c, ma, v, its == bEnd - 1, leftImage, carry, prem));
    }
  }
  // final imaging at t = 0: the carried left part of block 0
  E3D_RET(launchImaging(c, true, 0, nullptr, V(0), V(1), carry));
  c->w0 = W(ma - 1);
  c->w1 = W(ma);
  return E3D_OK;
}

static int bornAdjointDevice(Context* c, const DevSignals& srcSet, const DevSignals& recSet, const float* srcSig,
                             const float* resid) {
  E3D_RET(sourcePassWithCheckpoints(c, srcSet, nullptr, srcSig, nullptr, nullptr));
  return adjointPassFromCheckpoints(c, srcSet, recSet, srcSig, resid, nullptr);
}

int bornForwardHost(Context* c, const float* const* srcSig, float* const* data, const HostGeom& src,
                    const HostGeom& rec, const float* const* pert) {
  E3D_ARG(c && c->haveMedium, "medium not set");
  E3D_RET(rejectFreeSurface(c));
  E3D_ARG(srcSig && data && pert, "null argument");
  E3D_CUDA_TRY(cudaSetDevice(c->d.device));
  E3D_RET(ensurePert(c));
  for (int k = 0; k < NMED; k++)
    E3D_CUDA_TRY(cudaMemcpyAsync(c->pertDev[k], pert[k], (size_t)c->g.n * sizeof(float), cudaMemcpyHostToDevice,
                                 c->st));
  Staged S, R;
  int st = stageGeom(c, src, false, S);
  if (st == E3D_OK) st = stageGeom(c, rec, true, R);
  if (st == E3D_OK) st = stageSignalsIn(c, S, srcSig);
  if (st == E3D_OK) st = stageSignalsZero(c, R);
  if (st == E3D_OK) st = bornForwardDevice(c, S.set, R.set, S.sig, R.sig);
  if (st == E3D_OK) st = stageSignalsOut(c, R, data);
  if (st == E3D_OK) st = checkPipeError(c);
  if (st == E3D_OK && cudaStreamSynchronize(c->st) != cudaSuccess) {
    setLastError("stream failure", __FILE__, __LINE__);
    st = E3D_ERR_CUDA;
  }
  releaseStaged(c, S);
  releaseStaged(c, R);
  return st;
}

int bornAdjointHost(Context* c, const float* const* srcSig, const float* const* data, const HostGeom& src,
                    const HostGeom& rec, float* const* pert) {
  E3D_ARG(c && c->haveMedium, "medium not set");
  E3D_RET(rejectFreeSurface(c));
  E3D_ARG(srcSig && data && pert, "null argument");
  E3D_CUDA_TRY(cudaSetDevice(c->d.device));
  E3D_RET(ensurePert(c));
  // the reference copies the caller's planes to the device and accumulates
  // the image onto them (BornElasticGpuFunctions_3D.cu:2110-2114)
  for (int k = 0; k < NMED; k++)
    E3D_CUDA_TRY(cudaMemcpyAsync(c->pertDev[k], pert[k], (size_t)c->g.n * sizeof(float), cudaMemcpyHostToDevice,
                                 c->st));
  Staged S, R;
  int st = stageGeom(c, src, false, S);
  if (st == E3D_OK) st = stageGeom(c, rec, true, R);
  if (st == E3D_OK) st = stageSignalsIn(c, S, srcSig);
  if (st == E3D_OK) st = stageSignalsIn(c, R, const_cast<float* const*>(data));
  if (st == E3D_OK) st = bornAdjointDevice(c, S.set, R.set, S.sig, R.sig);
  if (st == E3D_OK) st = checkPipeError(c);
  if (st == E3D_OK) {
    for (int k = 0; k < NMED && st == E3D_OK; k++) {
      cudaError_t e = cudaMemcpyAsync(pert[k], c->pertDev[k], (size_t)c->g.n * sizeof(float),
                                      cudaMemcpyDeviceToHost, c->st);
      if (e != cudaSuccess) st = E3D_ERR_CUDA;
    }
    if (st == E3D_OK && cudaStreamSynchronize(c->st) != cudaSuccess) st = E3D_ERR_CUDA;
    if (st != E3D_OK) setLastError("copy-out failure", __FILE__, __LINE__);
  }
  releaseStaged(c, S);
  releaseStaged(c, R);
  return st;
}

// ---------------------------------------------------------------------------
// FWI (device API)
// ---------------------------------------------------------------------------
int fwiForwardDevice(Context* c, const DevSignals& srcSet, const DevSignals& recSet, const float* srcSig,
                     float* recSig, const TraceMap* map) {
  E3D_ARG(c && c->haveMedium, "medium not set");
  E3D_ARG(c->d.nts >= 2, "FWI needs at least two coarse samples");
  E3D_RET(rejectFreeSurface(c));
  E3D_CUDA_TRY(cudaSetDevice(c->d.device));
  return sourcePassWithCheckpoints(c, srcSet, &recSet, srcSig, recSig, map);
}

int fwiGradientDevice(Context* c, const DevSignals& srcSet, const DevSignals& recSet, const float* srcSig,
                      const float* residual, float* const* pert8, const TraceMap* map, float* srcAdj) {
  E3D_ARG(c && c->haveMedium, "medium not set");
  E3D_ARG(pert8 != nullptr, "null gradient planes");
  E3D_RET(rejectFreeSurface(c));
  E3D_CUDA_TRY(cudaSetDevice(c->d.device));
  for (int k = 0; k < NMED; k++) {
    E3D_ARG(pert8[k] != nullptr, "null gradient plane");
    c->pertDev[k] = pert8[k];  // accumulate straight into the caller's planes
  }
  int st = adjointPassFromCheckpoints(c, srcSet, recSet, srcSig, residual, map, srcAdj);
  for (int k = 0; k < NMED; k++) c->pertDev[k] = nullptr;
  return st;
}

int setVelocityStorage(Context* c, int type) {
  E3D_ARG(c && type >= -1 && type <= 1, "bad velocity slot storage type");
  c->vType = type;
  c->ckptValid = false;
  c->tailValid = false;
  return E3D_OK;
}

int velocityStorage(const Context* c) { return c->vUsed; }

int setDecimationRing(Context* c, int on) {
  E3D_ARG(c && (on == 0 || on == 1), "bad decimation mode");
  c->ringMode = on;
  c->ckptValid = false;
  c->tailValid = false;
  return E3D_OK;
}

int checkpointType(const Context* c) { return c->ckptUsed; }

// ---------------------------------------------------------------------------
// Allocation-free nonlinear propagation.  Some callers cannot allocate device
// memory while they propagate: a host framework may already hold nearly all of
// the device's memory in its own pool, or a caller may not be allowed to make
// cudaMalloc/cudaFree calls (which can synchronize the whole device) inside its
// time-critical loop.  For them the two wavefield levels and the sponge taper
// live in one fixed device array, sized for small grids; the caller passes the
// medium planes, positions and signals as device pointers.  The array is a
// module global, so every GPU that loads this library reserves it until the
// process exits, and every call on a device uses the same array.
// ---------------------------------------------------------------------------
constexpr size_t kStaticWorkBytes = (size_t)64 << 20;  // 64 MiB: 18 fields of up to ~0.93 M cells + taper
constexpr int kStaticMaxDevices = 64;
static __device__ __align__(256) unsigned char g_e3dStaticWork[kStaticWorkBytes];
static std::mutex g_staticWorkMutex;
static void* g_staticWorkAddr[kStaticMaxDevices] = {};
static CUcontext g_staticWorkCtx[kStaticMaxDevices] = {};  // context the cached address belongs to

size_t staticWorkBytes() { return kStaticWorkBytes; }

// cuCtxGetCurrent through the runtime's driver entry point (no libcuda link dependency)
static CUresult (*ctxGetCurrent())(CUcontext*) {
  static CUresult (*fn)(CUcontext*) = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (CUresult(*)(CUcontext*))f;
  }
  return fn;
}

// Device address of the static work array on the current device.  The name
// g_e3dStaticWork is a host-side stand-in in host code, so its device address
// is looked up once per device (with that device current) and cached, and
// looked up again when the device's primary context is no longer the one the
// address was taken in (after cudaDeviceReset).
static int staticWorkAddress(int dev, float** out) {
  if (dev < 0 || dev >= kStaticMaxDevices) {
    setLastError("device ordinal beyond the static work table", __FILE__, __LINE__);
    return E3D_ERR_ARG;
  }
  E3D_CUDA_TRY(cudaSetDevice(dev));  // makes the device's primary context current
  CUcontext cur = nullptr;
  if (auto fn = ctxGetCurrent()) fn(&cur);
  std::lock_guard<std::mutex> lock(g_staticWorkMutex);
  if (!g_staticWorkAddr[dev] || g_staticWorkCtx[dev] != cur) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_e3dStaticWork);
    if (e != cudaSuccess || !p) {
      setLastError(e != cudaSuccess ? cudaGetErrorString(e) : "null static work address", __FILE__, __LINE__);
      return E3D_ERR_CUDA;
    }
    g_staticWorkAddr[dev] = p;
    g_staticWorkCtx[dev] = cur;
  }
  *out = (float*)g_staticWorkAddr[dev];
  return E3D_OK;
}

int nlPropagateStatic(const ContextDesc& d, const float* const* planes, bool adjoint, const DevSignals& srcSet,
                      const DevSignals& recSet, float* srcSig, float* recSig, cudaStream_t st) {
  E3D_ARG(planes != nullptr, "null medium planes");
  for (int k = 0; k < NMED; k++) E3D_ARG(planes[k] != nullptr, "null medium plane");
  E3D_ARG(d.nz > 2 * FAT && d.nx > 2 * FAT && d.ny > 2 * FAT, "grid must exceed 2*FAT on every axis");
  E3D_ARG(d.nts >= 3, "nts must be at least 3");
  E3D_ARG(d.sub >= 1 && d.sub < SUB_MAX, "sub must be in [1, SUB_MAX)");
  E3D_ARG(d.minPad >= 0 && d.minPad < PAD_MAX, "minPad must be in [0, PAD_MAX)");
  E3D_ARG(d.dz > 0 && d.dx > 0 && d.dy > 0 && d.dts > 0, "sampling must be positive");
  E3D_ARG(srcSet.off[NCOMP] == 0 || srcSig, "null source signals");
  E3D_ARG(recSet.off[NCOMP] == 0 || recSig, "null receiver signals");
  const long long n = (long long)d.nz * d.nx * d.ny;
  const size_t fieldsBytes = ((size_t)2 * NCOMP * n * sizeof(float) + 255) / 256 * 256;
  // the two levels, the taper and one word for the position-table check
  const size_t need = fieldsBytes + (size_t)PAD_MAX * sizeof(float) + 256;
  if (n >= (1LL << 34) || need > kStaticWorkBytes) {
    char msg[256];
    snprintf(msg, sizeof(msg),
             "grid of %lld cells needs %zu bytes of static work memory; the allocation-free entry point holds "
             "%zu bytes (18 fields of at most %zu cells)",
             n, need, kStaticWorkBytes, (kStaticWorkBytes - (size_t)PAD_MAX * sizeof(float) - 256) / (18 * sizeof(float)));
    setLastError(msg, __FILE__, __LINE__);
    return E3D_ERR_ARG;
  }
  int dev = 0;
  E3D_CUDA_TRY(cudaGetDevice(&dev));
  float* work = nullptr;
  E3D_RET(staticWorkAddress(dev, &work));
  // grid constants as in createContext
  GridConst g{};
  g.nz = d.nz; g.nx = d.nx; g.ny = d.ny; g.minPad = d.minPad;
  g.yOff = 0; g.nyTaper = d.ny;
  g.yStride = (long long)d.nz * d.nx;
  g.n = n;
  const double kc[4] = {1.196289062541883, -0.079752604188901, 0.009570312506634, -6.975446437140719e-04};
  for (int i = 0; i < 4; i++) {
    g.cz[i] = (float)(kc[i] / d.dz);
    g.cx[i] = (float)(kc[i] / d.dx);
    g.cy[i] = (float)(kc[i] / (d.fixQ1 ? d.dy : d.dx));
  }
  const int ntw = (d.nts - 1) * d.sub + 1;
  const int hfilt = d.sub + 1;
  std::vector<float> filt(2 * hfilt, 0.f);
  const double scale = 1.0 / std::sqrt((float)ntw / (float)d.nts);
  for (int i = 0; i < hfilt; i++) {
    float left = (float)(1.0 - 1.0 * i / d.sub);
    float right = (float)(1.0 - left);
    filt[i] = (float)(left * scale);
    filt[i + hfilt] = (float)(right * scale);
  }
  TaperArg taper;
  for (int i = 0; i < PAD_MAX; i++) taper.v[i] = 1.f;
  for (int i = 0; i < d.minPad; i++) {
    float arg = (float)(M_PI / (1.0 * d.minPad) * 1.0 * (d.minPad - i));
    taper.v[i] = (float)(d.alphaCos + (1.0 - d.alphaCos) * std::cos(arg));
  }
  float* taperDev = (float*)((char*)work + fieldsBytes);
  unsigned* flagDev = (unsigned*)((char*)work + fieldsBytes + (size_t)PAD_MAX * sizeof(float));
  {
    // device positions: every entry an updated cell, checked before anything is written
    const DevSignals* sets[2] = {&srcSet, &recSet};
    E3D_RET(checkDevicePositions(sets, 2, d.nz, d.nx, d.ny, flagDev, st));
  }
  // the taper travels as a kernel argument; the array keeps the previous call's
  // contents, so both levels start at zero
  kWriteTaper<<<1, 128, 0, st>>>(taper, taperDev);
  E3D_LAUNCH_CHECK();
  E3D_CUDA_TRY(cudaMemsetAsync(work, 0, (size_t)2 * NCOMP * n * sizeof(float), st));
  g.taper = taperDev;
  Fields9 a, b;
  for (int k = 0; k < NCOMP; k++) {
    a.p[k] = work + (size_t)k * n;
    b.p[k] = work + (size_t)(NCOMP + k) * n;
  }
  constexpr int TXS = 8;
  const int tiz = (g.nz - 2 * FAT + TZ - 1) / TZ;
  const int tix = (g.nx - 2 * FAT + TXS - 1) / TXS;
  const int nyi = g.ny - 2 * FAT;
  const long long tiles = (long long)tiz * tix;
  int sms = 148;
  E3D_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int chunks = (int)std::min<long long>((4LL * sms + tiles - 1) / tiles, std::max(1, nyi / 32));
  chunks = std::max(chunks, 1);
  const int yChunk = (nyi + chunks - 1) / chunks;
  chunks = (nyi + yChunk - 1) / yChunk;
  const dim3 grid(tiz, tix, chunks), block(TZ, TXS);
  auto sparse = [](const DevSignals& s) {
    SparseSet ss;
    ss.pos = s.pos;
    for (int i = 0; i <= NCOMP; i++) ss.off[i] = s.off[i];
    return ss;
  };
  const SparseSet S = sparse(srcSet), R = sparse(recSet);
  const int nS = srcSet.off[NCOMP], nR = recSet.off[NCOMP];
  const size_t ns = (size_t)nS, nr = (size_t)nR;
  auto makeP = [&](Fields9& o, const Fields9& cur) {
    StepPtrs p{};
    for (int k = 0; k < NCOMP; k++) {
      p.o[k] = o.p[k];
      p.c[k] = cur.p[k];
    }
    for (int k = 0; k < NMED; k++) p.m[k] = planes[k];
    return p;
  };
  const int nts = d.nts, sub = d.sub;
  if (!adjoint) {
    if (nR) E3D_CUDA_TRY(cudaMemsetAsync(recSig, 0, nr * nts * sizeof(float), st));
    for (int its = 0; its < nts - 1; its++)
      for (int it2 = 1; it2 <= sub; it2++) {
        StepPtrs p = makeP(a, b);
        kStep<STEP_FWD, TXS><<<grid, block, 0, st>>>(p, g, yChunk);
        E3D_LAUNCH_CHECK();
        if (nS) {
          kInject<<<(nS + 127) / 128, 128, 0, st>>>(p, g, S, srcSig + its * ns, srcSig + (its + 1) * ns,
                                                   filt[it2 - 1], filt[hfilt + it2 - 1]);
          E3D_LAUNCH_CHECK();
        }
        if (nR) {
          kRecord<<<(nR + 127) / 128, 128, 0, st>>>(p, R, recSig + its * nr, recSig + (its + 1) * nr, filt[it2],
                                                   filt[hfilt + it2]);
          E3D_LAUNCH_CHECK();
        }
        swapF(a, b);
      }
  } else {
    if (nS) E3D_CUDA_TRY(cudaMemsetAsync(srcSig, 0, ns * nts * sizeof(float), st));
    for (int its = nts - 2; its >= 0; its--)
      for (int it2 = sub - 1; it2 >= 0; it2--) {
        StepPtrs p = makeP(a, b);
        kStep<STEP_ADJ_REVERSED, TXS><<<grid, block, 0, st>>>(p, g, yChunk);
        E3D_LAUNCH_CHECK();
        if (nR) {
          kInject<<<(nR + 127) / 128, 128, 0, st>>>(p, g, R, recSig + its * nr, recSig + (its + 1) * nr,
                                                   filt[it2 + 1], filt[hfilt + it2 + 1]);
          E3D_LAUNCH_CHECK();
        }
        if (nS) {
          kRecord<<<(nS + 127) / 128, 128, 0, st>>>(p, S, srcSig + its * ns, srcSig + (its + 1) * ns, filt[it2],
                                                   filt[hfilt + it2]);
          E3D_LAUNCH_CHECK();
        }
        swapF(a, b);
      }
  }
  return E3D_OK;
}

}  // namespace e3d
