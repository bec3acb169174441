// C++ engine behind the C ABI: one Context per (device, propagation grid,
// time axis).  A Context owns its device buffers and its CUDA stream; the
// C ABI maps the reference's process-global, per-iGpu state onto Contexts.
#pragma once
#include <cstddef>
#include <string>
#include <vector>
#include "common.cuh"

namespace e3d {

// Regular-grid acquisition points of the seven grids (center, x, y, z, xz, xy, yz).
struct HostGeom {
  const long long* pos[NGRID];
  long long n[NGRID];
};

// Storage type of saved wavefield states.
enum CkptType { CKPT_AUTO = -1, CKPT_F32 = 0, CKPT_F16 = 1, CKPT_BF16 = 2 };

struct ContextDesc {
  int device = 0;
  int nz = 0, nx = 0, ny = 0;
  int nts = 0;       // coarse samples
  int sub = 0;       // internal (2x parfile) subsampling
  int minPad = 0;
  float dz = 0, dx = 0, dy = 0, dts = 0, alphaCos = 0.99f;
  int fixQ1 = 0;     // 1: y derivatives use dy (the reference uses dx)
  int q2compat = 1;  // 1: sxz receivers use the z-grid positions (reference behaviour)
  int q3compat = 1;  // 1: Born yz shear term uses the xz derivative pair (reference behaviour)
  int freeSurface = 0;  // 1: stress-free surface at z = FAT (nonlinear propagation only)
};

struct Context;

int createContext(const ContextDesc& d, Context** out);
void destroyContext(Context* c);
// medium: 8 planes of nz*nx*ny floats; onDevice selects host or device pointers
int setMedium(Context* c, const float* const* planes, bool onDevice);
// Stepper variant for the autotuner: tile width along x (8 or 16), shared
// memory pipeline depth (2 or 3) and plane loader (0 plain loads, 1 cp.async,
// 2 TMA bulk tensor copies).
int setStepperVariant(Context* c, int tx, int stages, int loader);
// Number of y chunks the stepper grid splits each (z, x) tile column into (0: automatic).
int setStepperChunks(Context* c, int chunks);
// Reads and clears the device flag set when a bounded pipeline wait expired.
int checkPipeError(Context* c);
// Sampled stepper timing: bracket every n-th stepper launch with CUDA events (0 = off).
int setKernelTiming(Context* c, int every);
// Average duration (ms) of the sampled stepper launches of one mode since the last read.
int readKernelTiming(Context* c, int mode, double* avgMs, long long* count);
// Kernel launches issued by this context so far.
long long launchCount(const Context* c);
int setCheckpointPolicy(Context* c, int ckptType, int segment, double budgetBytes);

// Reference-layout host entry points ([nDevice][nts] per component).
int nlPropagateHost(Context* c, bool adjoint, float* const* model, float* const* data, const HostGeom& src,
                    const HostGeom& rec);
int bornForwardHost(Context* c, const float* const* srcSig, float* const* data, const HostGeom& src,
                    const HostGeom& rec, const float* const* pert);
int bornAdjointHost(Context* c, const float* const* srcSig, const float* const* data, const HostGeom& src,
                    const HostGeom& rec, float* const* pert);

// Device entry points: signals are time-major and concatenated over the nine
// components ([nts][sum of per-component counts]); positions are device
// arrays concatenated the same way with per-component offsets off[0..9].
struct DevSignals {
  const long long* pos;
  int off[NCOMP + 1];
};
// y-slab domain decomposition: `slabs` are contexts over consecutive y-slabs of one grid of
// nyGlobal planes (slab s over ny_s planes, neighbours overlapping by 2*FAT), each with its slab
// of the medium; host geometry in global positions, host signals as nlPropagateHost.
int nlPropagateSlabsHost(Context* const* slabs, int nSlabs, int nyGlobal, bool adjoint, float* const* model,
                         float* const* data, const HostGeom& src, const HostGeom& rec);
int nlPropagateDevice(Context* c, bool adjoint, const DevSignals& srcSet, const DevSignals& recSet,
                      float* srcSig, float* recSig);
// Device position tables: every entry an updated cell (E3D_ERR_BOUNDS otherwise); waits on the
// context's stream.  The device-pointer entry points call it before any propagation.
int validateDeviceSets(Context* c, const DevSignals& a, const DevSignals& b, int shots = 1);
// Batched nonlinear forward of `shots` shots of the context's medium (stacked per field); the
// position tables index the stacked grids (shot s at offset s*nz*nx*ny), signals time-major over
// the combined tables.
int nlForwardBatchDevice(Context* c, int shots, const DevSignals& srcSet, const DevSignals& recSet,
                         const float* srcSig, float* recSig);
// 1 (default): nonlinear propagation replays captured coarse blocks as CUDA graphs.
int setGraphLoop(Context* c, int on);
// Irregular receivers as linear combinations of the regular acquisition
// points (device arrays).  Receiver row r = k*nIrreg + i (component k).
//   gather (regular -> irregular): irr[r] = sum_f weight[r*nTaps+f] * reg[slot[r*nTaps+f]]
//   spread (irregular -> regular): reg[j] = sum_{e in [rowPtr[j], rowPtr[j+1])} w[e] * irr[idx[e]]
// slot and j index the concatenated regular list of the receiver DevSignals.
struct TraceMap {
  int nIrreg = 0;
  int nTaps = 0;
  const int* slot = nullptr;
  const float* weight = nullptr;
  const int* rowPtr = nullptr;
  const int* idx = nullptr;
  const float* w = nullptr;
};
// FWI: nonlinear forward that saves wavefield checkpoints for a later
// gradient; the gradient call consumes them (Born adjoint of the residual).
// Without a trace map recSig/residual are regular-grid and time-major
// ([nts][recSet.off[9]]); with one they are irregular and time-major
// ([nts][9*nIrreg]) and no regular-grid trace array is ever allocated.
int fwiForwardDevice(Context* c, const DevSignals& srcSet, const DevSignals& recSet, const float* srcSig,
                     float* recSig, const TraceMap* map);
// srcAdj (optional, time-major [nts][srcSet.off[9]]): the exact adjoint of the nonlinear
// propagation with respect to the scaled source signals, sampled during the same pass.
int fwiGradientDevice(Context* c, const DevSignals& srcSet, const DevSignals& recSet, const float* srcSig,
                      const float* residual, float* const* pert8, const TraceMap* map, float* srcAdj);
// Source velocity slot storage of the checkpoint plan: -1 auto, 0 FP32, 1 FP16 per-slice scaled.
int setVelocityStorage(Context* c, int type);
int velocityStorage(const Context* c);
int checkpointType(const Context* c);
// Decimation of the gradient's passes: 1 (default) from rings of fine levels, one
// launch per coarse block; 0 through accumulators fused into every fine step.
int setDecimationRing(Context* c, int on);
// y chunks of the y-marching block imaging launch (0: automatic).
int setImagingChunks(Context* c, int chunks);
int setImagingVariant(Context* c, int variant);
// Exact adjoint of the ring passes: 1 (default) the premultiplied-only state where the
// medium allows it, 0 always the dual raw + premultiplied state.
int setPremultipliedAdjoint(Context* c, int on);

// Allocation-free nonlinear propagation on the current device: the wavefield
// levels and the taper live in a fixed 64 MiB device array (staticWorkBytes());
// planes are the eight medium planes on the device.  Calls on one device share
// the array, so calls that overlap on the GPU race.
int nlPropagateStatic(const ContextDesc& d, const float* const* planes, bool adjoint, const DevSignals& srcSet,
                      const DevSignals& recSet, float* srcSig, float* recSig, cudaStream_t st);
size_t staticWorkBytes();

// Timing/inspection helpers
int stepOnly(Context* c, int mode, int nSteps);  // run nSteps bare steps on the working state
long long cellsPerStep(const Context* c);
int checkpointSegment(const Context* c);  // coarse blocks per checkpoint segment (0 before first use)
double deviceBytesInUse(const Context* c);
cudaStream_t stream(Context* c);
int setStream(Context* c, cudaStream_t s, bool useOwn);

const char* lastError();
}  // namespace e3d
