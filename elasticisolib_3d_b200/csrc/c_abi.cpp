// C ABI over the engine: the reference-named seam (per-iGpu slots, the
// reference's process-global state) and the explicit-context API.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "../../include/elastic3d_b200.h"
#include "engine.h"
#include "schedule.h"

using namespace e3d;

struct e3d_context {
  Context* c = nullptr;
};

namespace {

constexpr int N_SLOTS = 16;  // varElaDeclare_3D.h:15 (N_GPU_MAX)

// Parameters recorded by init*Gpu_3D until allocate*Gpu_3D creates the context.
struct Slot {
  bool inited = false;
  ContextDesc desc;
  Context* ctx = nullptr;
  int ny = 0;      // planes of the allocated context (a y-slab's when below desc.ny)
  int device = 0;  // its device
};

std::mutex g_mutex;
Slot g_nl[N_SLOTS];
Slot g_born[N_SLOTS];

int fail(int code, const char* msg) {
  setLastError(msg, __FILE__, __LINE__);
  return code;
}

int initSlot(Slot* table, float dz, float dx, float dy, int nz, int nx, int ny, int nts, float dts, int sub,
             int minPad, int blockSize, float alphaCos, int nGpu, int iGpuId) {
  (void)blockSize;  // the reference required 16; the engine picks its own tiles
  if (nGpu < 1 || nGpu > N_SLOTS) return fail(E3D_ERR_ARG, "nGpu out of range");
  if (sub >= SUB_MAX) return fail(E3D_ERR_ARG, "sub must be below SUB_MAX");
  if (minPad >= PAD_MAX) return fail(E3D_ERR_ARG, "minPad must be below PAD_MAX");
  std::lock_guard<std::mutex> lock(g_mutex);
  // init is called once per GPU thread; every slot shares the same parameters
  for (int i = 0; i < nGpu; i++) {
    Slot& s = table[i];
    s.desc.nz = nz; s.desc.nx = nx; s.desc.ny = ny; s.desc.nts = nts; s.desc.sub = sub;
    s.desc.minPad = minPad; s.desc.dz = dz; s.desc.dx = dx; s.desc.dy = dy; s.desc.dts = dts;
    s.desc.alphaCos = alphaCos;
    s.inited = true;
  }
  (void)iGpuId;
  return E3D_OK;
}

int allocSlot(Slot* table, const float* const* planes, int nx, int ny, int nz, int iGpu, int iGpuId) {
  if (iGpu < 0 || iGpu >= N_SLOTS) return fail(E3D_ERR_ARG, "iGpu out of range");
  Slot& s = table[iGpu];
  if (!s.inited) return fail(E3D_ERR_STATE, "allocate before init");
  // ny below the init's ny: a y-slab of a decomposed grid (the reference allocates ny_domDec[iGpu]
  // planes of the shifted medium, nonlinearPropElasticGpu_3D.cpp:37-48)
  if (s.desc.nx != nx || ny > s.desc.ny || (ny < s.desc.ny && ny < 3 * FAT) || s.desc.nz != nz)
    return fail(E3D_ERR_ARG, "grid differs from init");
  if (s.ctx) {
    destroyContext(s.ctx);
    s.ctx = nullptr;
  }
  ContextDesc d = s.desc;
  d.ny = ny;
  d.device = iGpuId;
  Context* c = nullptr;
  int st = createContext(d, &c);
  if (st != E3D_OK) return st;
  st = setMedium(c, planes, false);
  if (st != E3D_OK) {
    destroyContext(c);
    return st;
  }
  s.ctx = c;
  s.ny = ny;
  s.device = iGpuId;
  return E3D_OK;
}

int freeSlot(Slot* table, int iGpu) {
  if (iGpu < 0 || iGpu >= N_SLOTS) return fail(E3D_ERR_ARG, "iGpu out of range");
  if (table[iGpu].ctx) destroyContext(table[iGpu].ctx);
  table[iGpu].ctx = nullptr;
  return E3D_OK;
}

Context* slotCtx(Slot* table, int iGpu, int nx, int ny, int nz) {
  if (iGpu < 0 || iGpu >= N_SLOTS || !table[iGpu].ctx) return nullptr;
  const ContextDesc& d = table[iGpu].desc;
  if (d.nx != nx || d.ny != ny || d.nz != nz || table[iGpu].ny != ny) return nullptr;
  return table[iGpu].ctx;
}

// The slab contexts of a decomposed propagation: slots 0..n-1 allocated with ny_domDec[i] planes
// on gpuList[i], the init's ny the whole grid's.
int slabCtxs(Slot* table, int nx, int ny, int nz, const int* nyDomDec, int nDomDec, const int* gpuList, int nGpu,
             std::vector<Context*>& out) {
  if (!nyDomDec || !gpuList || nDomDec < 2 || nDomDec != nGpu || nDomDec > N_SLOTS)
    return fail(E3D_ERR_ARG, "domain decomposition needs one ny_domDec entry per GPU and at least two");
  out.clear();
  for (int i = 0; i < nDomDec; i++) {
    const Slot& s = table[i];
    if (!s.ctx || s.desc.nx != nx || s.desc.ny != ny || s.desc.nz != nz || s.ny != nyDomDec[i] ||
        s.device != gpuList[i])
      return fail(E3D_ERR_STATE, "slab slot not allocated with ny_domDec[iGpu] planes on gpuList[iGpu]");
    out.push_back(s.ctx);
  }
  return E3D_OK;
}

HostGeom geom14(long long* p0, long long n0, long long* p1, long long n1, long long* p2, long long n2,
                long long* p3, long long n3, long long* p4, long long n4, long long* p5, long long n5,
                long long* p6, long long n6) {
  HostGeom g;
  long long* p[7] = {p0, p1, p2, p3, p4, p5, p6};
  long long n[7] = {n0, n1, n2, n3, n4, n5, n6};
  for (int i = 0; i < 7; i++) {
    g.pos[i] = p[i];
    g.n[i] = n[i];
  }
  return g;
}

HostGeom geomArrays(const long long* const* pos, const long long* n) {
  HostGeom g;
  for (int i = 0; i < 7; i++) {
    g.pos[i] = pos[i];
    g.n[i] = n[i];
  }
  return g;
}

}  // namespace

extern "C" {

const char* e3d_last_error(void) { return lastError(); }
const char* e3d_version(void) { return "elastic3d_b200 0.1.0 (sm_100a)"; }

int getGpuInfo_3D(const int* gpuList, int nGpuList, int info, int deviceNumberInfo) {
  (void)info;
  (void)deviceNumberInfo;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) return fail(E3D_ERR_CUDA, "cudaGetDeviceCount failed");
  if (nGpuList < 1 || !gpuList) return fail(E3D_ERR_ARG, "empty GPU list");
  for (int i = 0; i < nGpuList; i++)
    if (gpuList[i] < 0 || gpuList[i] >= count) return fail(E3D_ERR_ARG, "GPU id not present");
  return E3D_OK;
}

int setGpuP2P(int nGpu, int info, const int* gpuList) {
  (void)info;
  if (nGpu < 1 || !gpuList) return fail(E3D_ERR_ARG, "empty GPU list");
  for (int i = 0; i < nGpu; i++)
    for (int j = 0; j < nGpu; j++) {
      if (i == j) continue;
      int can = 0;
      if (cudaDeviceCanAccessPeer(&can, gpuList[i], gpuList[j]) != cudaSuccess) return fail(E3D_ERR_CUDA, "peer query");
      if (!can) continue;
      if (cudaSetDevice(gpuList[i]) != cudaSuccess) return fail(E3D_ERR_CUDA, "cudaSetDevice");
      cudaError_t e = cudaDeviceEnablePeerAccess(gpuList[j], 0);
      if (e != cudaSuccess && e != cudaErrorPeerAccessAlreadyEnabled) return fail(E3D_ERR_CUDA, "peer enable");
      cudaGetLastError();
    }
  return E3D_OK;
}

int initNonlinearElasticGpu_3D(float dz, float dx, float dy, int nz, int nx, int ny, int nts, float dts, int sub,
                               int minPad, int blockSize, float alphaCos, int nGpu, int iGpuId, int iGpuAlloc) {
  (void)iGpuAlloc;
  return initSlot(g_nl, dz, dx, dy, nz, nx, ny, nts, dts, sub, minPad, blockSize, alphaCos, nGpu, iGpuId);
}

int allocateNonlinearElasticGpu_3D(float* rhoxDtw, float* rhoyDtw, float* rhozDtw, float* lamb2MuDtw,
                                   float* lambDtw, float* muxzDtw, float* muxyDtw, float* muyzDtw, int nx, int ny,
                                   int nz, int iGpu, int iGpuId) {
  const float* planes[8] = {rhoxDtw, rhoyDtw, rhozDtw, lamb2MuDtw, lambDtw, muxzDtw, muxyDtw, muyzDtw};
  return allocSlot(g_nl, planes, nx, ny, nz, iGpu, iGpuId);
}

int deallocateNonlinearElasticGpu_3D(int iGpu, int iGpuId) {
  (void)iGpuId;
  return freeSlot(g_nl, iGpu);
}

#define E3D_SEAM_SIGNALS                                                                                          \
  float *m0, float *m1, float *m2, float *m3, float *m4, float *m5, float *m6, float *m7, float *m8, float *d0,  \
      float *d1, float *d2, float *d3, float *d4, float *d5, float *d6, float *d7, float *d8, long long *s0,       \
      long long ns0, long long *s1, long long ns1, long long *s2, long long ns2, long long *s3, long long ns3,    \
      long long *s4, long long ns4, long long *s5, long long ns5, long long *s6, long long ns6, long long *r0,    \
      long long nr0, long long *r1, long long nr1, long long *r2, long long nr2, long long *r3, long long nr3,    \
      long long *r4, long long nr4, long long *r5, long long nr5, long long *r6, long long nr6

int propElasticFwdGpu_3D(E3D_SEAM_SIGNALS, int nx, int ny, int nz, int iGpu, int iGpuId) {
  (void)iGpuId;
  Context* c = slotCtx(g_nl, iGpu, nx, ny, nz);
  if (!c) return fail(E3D_ERR_STATE, "propagator slot not allocated (or grid mismatch)");
  float* model[9] = {m0, m1, m2, m3, m4, m5, m6, m7, m8};
  float* data[9] = {d0, d1, d2, d3, d4, d5, d6, d7, d8};
  return nlPropagateHost(c, false, model, data, geom14(s0, ns0, s1, ns1, s2, ns2, s3, ns3, s4, ns4, s5, ns5, s6, ns6),
                         geom14(r0, nr0, r1, nr1, r2, nr2, r3, nr3, r4, nr4, r5, nr5, r6, nr6));
}

int propElasticAdjGpu_3D(E3D_SEAM_SIGNALS, int nx, int ny, int nz, int iGpu, int iGpuId) {
  (void)iGpuId;
  Context* c = slotCtx(g_nl, iGpu, nx, ny, nz);
  if (!c) return fail(E3D_ERR_STATE, "propagator slot not allocated (or grid mismatch)");
  float* model[9] = {m0, m1, m2, m3, m4, m5, m6, m7, m8};
  float* data[9] = {d0, d1, d2, d3, d4, d5, d6, d7, d8};
  return nlPropagateHost(c, true, model, data, geom14(s0, ns0, s1, ns1, s2, ns2, s3, ns3, s4, ns4, s5, ns5, s6, ns6),
                         geom14(r0, nr0, r1, nr1, r2, nr2, r3, nr3, r4, nr4, r5, nr5, r6, nr6));
}

int propElasticFwdGpudomDec_3D(E3D_SEAM_SIGNALS, int nx, int ny, int nz, const int* ny_domDec, int nDomDec,
                               const int* gpuList, int nGpu) {
  std::vector<Context*> slabs;
  int st = slabCtxs(g_nl, nx, ny, nz, ny_domDec, nDomDec, gpuList, nGpu, slabs);
  if (st != E3D_OK) return st;
  float* model[9] = {m0, m1, m2, m3, m4, m5, m6, m7, m8};
  float* data[9] = {d0, d1, d2, d3, d4, d5, d6, d7, d8};
  return nlPropagateSlabsHost(slabs.data(), (int)slabs.size(), ny, false, model, data,
                              geom14(s0, ns0, s1, ns1, s2, ns2, s3, ns3, s4, ns4, s5, ns5, s6, ns6),
                              geom14(r0, nr0, r1, nr1, r2, nr2, r3, nr3, r4, nr4, r5, nr5, r6, nr6));
}

int propElasticAdjGpudomDec_3D(E3D_SEAM_SIGNALS, int nx, int ny, int nz, const int* ny_domDec, int nDomDec,
                               const int* gpuList, int nGpu) {
  std::vector<Context*> slabs;
  int st = slabCtxs(g_nl, nx, ny, nz, ny_domDec, nDomDec, gpuList, nGpu, slabs);
  if (st != E3D_OK) return st;
  float* model[9] = {m0, m1, m2, m3, m4, m5, m6, m7, m8};
  float* data[9] = {d0, d1, d2, d3, d4, d5, d6, d7, d8};
  return nlPropagateSlabsHost(slabs.data(), (int)slabs.size(), ny, true, model, data,
                              geom14(s0, ns0, s1, ns1, s2, ns2, s3, ns3, s4, ns4, s5, ns5, s6, ns6),
                              geom14(r0, nr0, r1, nr1, r2, nr2, r3, nr3, r4, nr4, r5, nr5, r6, nr6));
}

int initBornElasticGpu_3D(float dz, float dx, float dy, int nz, int nx, int ny, int nts, float dts, int sub,
                          int minPad, int blockSize, float alphaCos, int nGpu, int iGpuId, int iGpuAlloc) {
  (void)iGpuAlloc;
  return initSlot(g_born, dz, dx, dy, nz, nx, ny, nts, dts, sub, minPad, blockSize, alphaCos, nGpu, iGpuId);
}

int allocateBornElasticGpu_3D(float* rhoxDtw, float* rhoyDtw, float* rhozDtw, float* lamb2MuDtw, float* lambDtw,
                              float* muxzDtw, float* muxyDtw, float* muyzDtw, int nx, int ny, int nz, int iGpu,
                              int iGpuId) {
  const float* planes[8] = {rhoxDtw, rhoyDtw, rhozDtw, lamb2MuDtw, lambDtw, muxzDtw, muxyDtw, muyzDtw};
  return allocSlot(g_born, planes, nx, ny, nz, iGpu, iGpuId);
}

int deallocateBornElasticGpu_3D(int iGpu, int iGpuId) {
  (void)iGpuId;
  return freeSlot(g_born, iGpu);
}

int allocatePinBornElasticGpu_3D(int nx, int ny, int nz, int nts, int nGpu, int iGpuId, int iGpu, int iGpuAlloc) {
  (void)iGpuId;
  (void)iGpuAlloc;
  if (nx <= 0 || ny <= 0 || nz <= 0 || nts < 3 || nGpu < 1 || iGpu < 0 || iGpu >= N_SLOTS)
    return fail(E3D_ERR_ARG, "bad Born wavefield allocation arguments");
  return E3D_OK;
}

int deallocatePinBornElasticGpu_3D(int iGpu, int iGpuId) {
  (void)iGpuId;
  if (iGpu < 0 || iGpu >= N_SLOTS) return fail(E3D_ERR_ARG, "iGpu out of range");
  return E3D_OK;
}

#define E3D_SEAM_PERT \
  float *p0, float *p1, float *p2, float *p3, float *p4, float *p5, float *p6, float *p7

int BornElasticFwdGpu_3D(E3D_SEAM_SIGNALS, E3D_SEAM_PERT, int nx, int ny, int nz, int iGpu, int iGpuId) {
  (void)iGpuId;
  Context* c = slotCtx(g_born, iGpu, nx, ny, nz);
  if (!c) return fail(E3D_ERR_STATE, "Born slot not allocated (or grid mismatch)");
  const float* src[9] = {m0, m1, m2, m3, m4, m5, m6, m7, m8};
  float* data[9] = {d0, d1, d2, d3, d4, d5, d6, d7, d8};
  const float* pert[8] = {p0, p1, p2, p3, p4, p5, p6, p7};
  return bornForwardHost(c, src, data, geom14(s0, ns0, s1, ns1, s2, ns2, s3, ns3, s4, ns4, s5, ns5, s6, ns6),
                         geom14(r0, nr0, r1, nr1, r2, nr2, r3, nr3, r4, nr4, r5, nr5, r6, nr6), pert);
}

int BornElasticAdjGpu_3D(E3D_SEAM_SIGNALS, E3D_SEAM_PERT, int nx, int ny, int nz, int iGpu, int iGpuId) {
  (void)iGpuId;
  Context* c = slotCtx(g_born, iGpu, nx, ny, nz);
  if (!c) return fail(E3D_ERR_STATE, "Born slot not allocated (or grid mismatch)");
  const float* src[9] = {m0, m1, m2, m3, m4, m5, m6, m7, m8};
  const float* data[9] = {d0, d1, d2, d3, d4, d5, d6, d7, d8};
  float* pert[8] = {p0, p1, p2, p3, p4, p5, p6, p7};
  return bornAdjointHost(c, src, data, geom14(s0, ns0, s1, ns1, s2, ns2, s3, ns3, s4, ns4, s5, ns5, s6, ns6),
                         geom14(r0, nr0, r1, nr1, r2, nr2, r3, nr3, r4, nr4, r5, nr5, r6, nr6), pert);
}

// ---------------------------------------------------------------------------
int e3d_context_create(const e3d_desc* desc, e3d_context** out) {
  if (!desc || !out) return fail(E3D_ERR_ARG, "null argument");
  ContextDesc d;
  d.device = desc->device;
  d.nz = desc->nz; d.nx = desc->nx; d.ny = desc->ny;
  d.nts = desc->nts; d.sub = desc->sub; d.minPad = desc->minPad;
  d.dz = desc->dz; d.dx = desc->dx; d.dy = desc->dy; d.dts = desc->dts; d.alphaCos = desc->alphaCos;
  d.fixQ1 = desc->fix_q1; d.q2compat = desc->q2compat; d.q3compat = desc->q3compat;
  d.freeSurface = desc->free_surface;
  Context* c = nullptr;
  int st = createContext(d, &c);
  if (st != E3D_OK) return st;
  *out = new e3d_context();
  (*out)->c = c;
  return E3D_OK;
}

int e3d_context_destroy(e3d_context* ctx) {
  if (!ctx) return E3D_OK;
  destroyContext(ctx->c);
  delete ctx;
  return E3D_OK;
}

#define CTX_OR_FAIL(ctx) \
  if (!(ctx) || !(ctx)->c) return fail(E3D_ERR_ARG, "null context")

int e3d_set_medium(e3d_context* ctx, const float* const* planes8, int on_device) {
  CTX_OR_FAIL(ctx);
  return setMedium(ctx->c, planes8, on_device != 0);
}

int e3d_set_stepper_variant(e3d_context* ctx, int tx, int stages, int loader) {
  CTX_OR_FAIL(ctx);
  return setStepperVariant(ctx->c, tx, stages, loader);
}

int e3d_set_graph_loop(e3d_context* ctx, int on) {
  CTX_OR_FAIL(ctx);
  return setGraphLoop(ctx->c, on);
}

int e3d_set_stepper_chunks(e3d_context* ctx, int chunks) {
  CTX_OR_FAIL(ctx);
  return setStepperChunks(ctx->c, chunks);
}

int e3d_set_checkpoint_policy(e3d_context* ctx, int type, int segment, double budget_bytes) {
  CTX_OR_FAIL(ctx);
  return setCheckpointPolicy(ctx->c, type, segment, budget_bytes);
}

int e3d_synchronize(e3d_context* ctx) {
  CTX_OR_FAIL(ctx);
  cudaError_t e = cudaStreamSynchronize(stream(ctx->c));
  if (e != cudaSuccess) return fail(E3D_ERR_CUDA, cudaGetErrorString(e));
  return checkPipeError(ctx->c);
}

void* e3d_stream(e3d_context* ctx) { return (ctx && ctx->c) ? (void*)stream(ctx->c) : nullptr; }

int e3d_set_stream(e3d_context* ctx, void* s, int use_own) {
  CTX_OR_FAIL(ctx);
  return setStream(ctx->c, (cudaStream_t)s, use_own != 0);
}

long long e3d_cells_per_step(const e3d_context* ctx) { return (ctx && ctx->c) ? cellsPerStep(ctx->c) : 0; }

int e3d_checkpoint_segment(const e3d_context* ctx) { return (ctx && ctx->c) ? checkpointSegment(ctx->c) : 0; }

int e3d_checkpoint_schedule(int blocks, int segment_len, int* seg_start, int max_segments, int* recomputed) {
  if (blocks < 1 || segment_len < 1) return -E3D_ERR_ARG;
  const int L = std::min(segment_len, blocks);
  const int nseg = e3d::schedule::segments(blocks, L);
  if (seg_start) {
    if (max_segments < nseg) return -E3D_ERR_ARG;
    for (int s = 0; s <= nseg; s++) seg_start[s] = e3d::schedule::segStart(blocks, L, nseg, s);
  }
  if (recomputed) *recomputed = e3d::schedule::recomputedBlocks(blocks, L);
  return nseg;
}

int e3d_checkpoint_plan(long long n_cells, int ny, int nts, double budget_bytes, int ckpt_type, int velocity_type,
                        int segment, int* ckpt_used, int* velocity_used, int* segment_len, double* plan_bytes) {
  if (n_cells < 1 || ny < 1 || nts < 2 || ckpt_type < -1 || ckpt_type > 2 || velocity_type < -1 ||
      velocity_type > 1 || segment < 0)
    return E3D_ERR_ARG;
  e3d::schedule::Plan p{};
  if (!e3d::schedule::choosePlan(n_cells, ny, nts, budget_bytes, ckpt_type, velocity_type, segment, p))
    return E3D_ERR_OOM;
  if (ckpt_used) *ckpt_used = p.ck;
  if (velocity_used) *velocity_used = p.vt;
  if (segment_len) *segment_len = p.L;
  if (plan_bytes) *plan_bytes = e3d::schedule::planBytes(n_cells, ny, nts, p.ck, p.vt, p.L);
  return E3D_OK;
}

int e3d_nl_forward(e3d_context* ctx, const float* const* model9, float* const* data9, const long long* const* src_pos,
                   const long long* n_src, const long long* const* rec_pos, const long long* n_rec) {
  CTX_OR_FAIL(ctx);
  if (!src_pos || !n_src || !rec_pos || !n_rec) return fail(E3D_ERR_ARG, "null geometry");
  return nlPropagateHost(ctx->c, false, const_cast<float* const*>(model9), data9, geomArrays(src_pos, n_src),
                         geomArrays(rec_pos, n_rec));
}

int e3d_nl_adjoint(e3d_context* ctx, float* const* model9, const float* const* data9, const long long* const* src_pos,
                   const long long* n_src, const long long* const* rec_pos, const long long* n_rec) {
  CTX_OR_FAIL(ctx);
  if (!src_pos || !n_src || !rec_pos || !n_rec) return fail(E3D_ERR_ARG, "null geometry");
  return nlPropagateHost(ctx->c, true, model9, const_cast<float* const*>(data9), geomArrays(src_pos, n_src),
                         geomArrays(rec_pos, n_rec));
}

int e3d_nl_propagate_slabs(e3d_context* const* slabs, int n_slabs, int ny_global, int adjoint, float* const* model9,
                           float* const* data9, const long long* const* src_pos, const long long* n_src,
                           const long long* const* rec_pos, const long long* n_rec) {
  if (!slabs || n_slabs < 1 || n_slabs > 64) return fail(E3D_ERR_ARG, "bad slab list");
  if (!src_pos || !n_src || !rec_pos || !n_rec) return fail(E3D_ERR_ARG, "null geometry");
  std::vector<Context*> cs;
  for (int i = 0; i < n_slabs; i++) {
    if (!slabs[i] || !slabs[i]->c) return fail(E3D_ERR_ARG, "null slab context");
    cs.push_back(slabs[i]->c);
  }
  return nlPropagateSlabsHost(cs.data(), n_slabs, ny_global, adjoint != 0, model9, data9,
                              geomArrays(src_pos, n_src), geomArrays(rec_pos, n_rec));
}

int e3d_born_forward(e3d_context* ctx, const float* const* src9, float* const* data9, const long long* const* src_pos,
                     const long long* n_src, const long long* const* rec_pos, const long long* n_rec,
                     const float* const* pert8) {
  CTX_OR_FAIL(ctx);
  if (!src_pos || !n_src || !rec_pos || !n_rec) return fail(E3D_ERR_ARG, "null geometry");
  return bornForwardHost(ctx->c, src9, data9, geomArrays(src_pos, n_src), geomArrays(rec_pos, n_rec), pert8);
}

int e3d_born_adjoint(e3d_context* ctx, const float* const* src9, const float* const* data9,
                     const long long* const* src_pos, const long long* n_src, const long long* const* rec_pos,
                     const long long* n_rec, float* const* pert8) {
  CTX_OR_FAIL(ctx);
  if (!src_pos || !n_src || !rec_pos || !n_rec) return fail(E3D_ERR_ARG, "null geometry");
  return bornAdjointHost(ctx->c, src9, data9, geomArrays(src_pos, n_src), geomArrays(rec_pos, n_rec), pert8);
}

static int devSet(const long long* pos, const int* off10, DevSignals& s) {
  if (!off10) return fail(E3D_ERR_ARG, "null offsets");
  s.pos = pos;
  for (int k = 0; k <= NCOMP; k++) {
    s.off[k] = off10[k];
    if (k > 0 && off10[k] < off10[k - 1]) return fail(E3D_ERR_ARG, "offsets must be non-decreasing");
  }
  if (off10[0] != 0) return fail(E3D_ERR_ARG, "offsets must start at 0");
  if (off10[NCOMP] > 0 && !pos) return fail(E3D_ERR_ARG, "null position table");
  return E3D_OK;
}

int e3d_nl_propagate_device(e3d_context* ctx, int adjoint, const long long* src_pos_dev, const int* src_off10,
                            const long long* rec_pos_dev, const int* rec_off10, float* src_sig_dev,
                            float* rec_sig_dev) {
  CTX_OR_FAIL(ctx);
  DevSignals S, R;
  int st = devSet(src_pos_dev, src_off10, S);
  if (st == E3D_OK) st = devSet(rec_pos_dev, rec_off10, R);
  if (st == E3D_OK) st = validateDeviceSets(ctx->c, S, R);
  if (st != E3D_OK) return st;
  return nlPropagateDevice(ctx->c, adjoint != 0, S, R, src_sig_dev, rec_sig_dev);
}

static int traceMap(const e3d_trace_map* m, TraceMap& t) {
  if (!m) return E3D_OK;
  if (m->n_irreg < 0 || m->n_taps < 1 || m->n_taps > 64) {
    setLastError("bad trace map sizes", __FILE__, __LINE__);
    return E3D_ERR_ARG;
  }
  if (!m->row_ptr || (m->n_irreg > 0 && (!m->slot || !m->weight || !m->idx || !m->w))) {
    setLastError("null trace map table", __FILE__, __LINE__);
    return E3D_ERR_ARG;
  }
  t.nIrreg = m->n_irreg;
  t.nTaps = m->n_taps;
  t.slot = m->slot;
  t.weight = m->weight;
  t.rowPtr = m->row_ptr;
  t.idx = m->idx;
  t.w = m->w;
  return E3D_OK;
}

int e3d_fwi_forward_device(e3d_context* ctx, const long long* src_pos_dev, const int* src_off10,
                           const long long* rec_pos_dev, const int* rec_off10, const float* src_sig_dev,
                           float* rec_sig_dev, const e3d_trace_map* map) {
  CTX_OR_FAIL(ctx);
  DevSignals S, R;
  TraceMap T;
  int st = devSet(src_pos_dev, src_off10, S);
  if (st == E3D_OK) st = devSet(rec_pos_dev, rec_off10, R);
  if (st == E3D_OK) st = traceMap(map, T);
  if (st == E3D_OK) st = validateDeviceSets(ctx->c, S, R);
  if (st != E3D_OK) return st;
  return fwiForwardDevice(ctx->c, S, R, src_sig_dev, rec_sig_dev, map ? &T : nullptr);
}

int e3d_fwi_gradient_device(e3d_context* ctx, const long long* src_pos_dev, const int* src_off10,
                            const long long* rec_pos_dev, const int* rec_off10, const float* src_sig_dev,
                            const float* residual_dev, float* const* grad8_dev, const e3d_trace_map* map,
                            float* src_adj_dev) {
  CTX_OR_FAIL(ctx);
  DevSignals S, R;
  TraceMap T;
  int st = devSet(src_pos_dev, src_off10, S);
  if (st == E3D_OK) st = devSet(rec_pos_dev, rec_off10, R);
  if (st == E3D_OK) st = traceMap(map, T);
  if (st == E3D_OK) st = validateDeviceSets(ctx->c, S, R);
  if (st != E3D_OK) return st;
  return fwiGradientDevice(ctx->c, S, R, src_sig_dev, residual_dev, grad8_dev, map ? &T : nullptr, src_adj_dev);
}

int e3d_set_velocity_storage(e3d_context* ctx, int type) {
  CTX_OR_FAIL(ctx);
  return setVelocityStorage(ctx->c, type);
}

int e3d_velocity_storage(const e3d_context* ctx) { return (ctx && ctx->c) ? velocityStorage(ctx->c) : -1; }

int e3d_checkpoint_type(const e3d_context* ctx) { return (ctx && ctx->c) ? checkpointType(ctx->c) : -1; }

int e3d_nl_forward_batch_device(e3d_context* ctx, int shots, const long long* src_pos_dev, const int* src_off10,
                                const long long* rec_pos_dev, const int* rec_off10, const float* src_sig_dev,
                                float* rec_sig_dev) {
  CTX_OR_FAIL(ctx);
  DevSignals S, R;
  int st = devSet(src_pos_dev, src_off10, S);
  if (st == E3D_OK) st = devSet(rec_pos_dev, rec_off10, R);
  if (st == E3D_OK && shots < 1) st = fail(E3D_ERR_ARG, "shots must be positive");
  if (st == E3D_OK) st = validateDeviceSets(ctx->c, S, R, shots);
  if (st != E3D_OK) return st;
  return nlForwardBatchDevice(ctx->c, shots, S, R, src_sig_dev, rec_sig_dev);
}

int e3d_set_premultiplied_adjoint(e3d_context* ctx, int on) {
  CTX_OR_FAIL(ctx);
  return setPremultipliedAdjoint(ctx->c, on);
}

int e3d_set_imaging_chunks(e3d_context* ctx, int chunks) {
  CTX_OR_FAIL(ctx);
  return setImagingChunks(ctx->c, chunks);
}

int e3d_set_imaging_variant(e3d_context* ctx, int variant) {
  CTX_OR_FAIL(ctx);
  return setImagingVariant(ctx->c, variant);
}

int e3d_set_decimation_ring(e3d_context* ctx, int on) {
  CTX_OR_FAIL(ctx);
  return setDecimationRing(ctx->c, on);
}

int e3d_nl_propagate_device_noalloc(const e3d_desc* desc, const float* const* planes8_dev, int adjoint,
                                    const long long* src_pos_dev, const int* src_off10,
                                    const long long* rec_pos_dev, const int* rec_off10, float* src_sig_dev,
                                    float* rec_sig_dev, void* stream) {
  if (!desc) return fail(E3D_ERR_ARG, "null descriptor");
  if (desc->free_surface) return fail(E3D_ERR_ARG, "the allocation-free entry point has no free surface");
  ContextDesc d;
  d.device = desc->device;
  d.nz = desc->nz; d.nx = desc->nx; d.ny = desc->ny;
  d.nts = desc->nts; d.sub = desc->sub; d.minPad = desc->minPad;
  d.dz = desc->dz; d.dx = desc->dx; d.dy = desc->dy; d.dts = desc->dts; d.alphaCos = desc->alphaCos;
  d.fixQ1 = desc->fix_q1; d.q2compat = desc->q2compat; d.q3compat = desc->q3compat;
  DevSignals S, R;
  int st = devSet(src_pos_dev, src_off10, S);
  if (st == E3D_OK) st = devSet(rec_pos_dev, rec_off10, R);
  if (st != E3D_OK) return st;
  return nlPropagateStatic(d, planes8_dev, adjoint != 0, S, R, src_sig_dev, rec_sig_dev, (cudaStream_t)stream);
}

size_t e3d_noalloc_work_bytes(void) { return staticWorkBytes(); }

int e3d_kernel_timing(e3d_context* ctx, int every) {
  CTX_OR_FAIL(ctx);
  return setKernelTiming(ctx->c, every);
}

int e3d_kernel_timing_read(e3d_context* ctx, int mode, double* avg_ms, long long* count) {
  CTX_OR_FAIL(ctx);
  return readKernelTiming(ctx->c, mode, avg_ms, count);
}

long long e3d_launch_count(const e3d_context* ctx) { return (ctx && ctx->c) ? launchCount(ctx->c) : 0; }

int e3d_step_only(e3d_context* ctx, int mode, int n_steps) {
  CTX_OR_FAIL(ctx);
  return stepOnly(ctx->c, mode, n_steps);
}

}  // extern "C"
