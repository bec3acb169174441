/* elastic3d_b200.h -- C ABI of the B200 elastic 3D propagation library.
 *
 * Two layers, both plain C (pointers and sizes, no C++ or torch types):
 *
 * 1. The drop-in seam.  Same names and argument meaning as the reference's
 *    raw-pointer driver functions, which its C++ operator classes call:
 *      elastic_iso_float/include/nonlinearPropElasticGpuFunctions_3D.h:9-18
 *      elastic_iso_float/include/BornElasticGpuFunctions_3D.h:9-21
 *    Every function returns an int status (0 = success) instead of void;
 *    the reference printed and called exit(-1) on CUDA errors
 *    (elastic_iso_float/src/cudaErrors_3D.cu:4-27).  Host arrays are owned
 *    by the caller; outputs are overwritten, as in the reference.  The
 *    functions that took std::vector take a pointer and a count.
 *
 * 2. An explicit-context API (e3d_*) for new callers: several grids per
 *    process, device-resident signals, checkpointed FWI gradients.
 *
 * Conventions: a field has nz*nx*ny floats, z fastest
 * (index = iy*nz*nx + ix*nz + iz).  Acquisition positions are int64 indices
 * into that layout, one table per grid in the order
 * center, x, y, z, xz, xy, yz.  Signal blocks follow the reference:
 * one block per wavefield component vx, vy, vz, sxx, syy, szz, sxz, sxy, syz,
 * each [nDevice][nts] with time fastest.  `sub` is always the internal value
 * (twice the parameter-file value), as the reference drivers receive it.
 */
#ifndef ELASTIC3D_B200_H
#define ELASTIC3D_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes */
#define E3D_OK 0
#define E3D_ERR_ARG 1
#define E3D_ERR_CUDA 2
#define E3D_ERR_STATE 3
#define E3D_ERR_OOM 4
#define E3D_ERR_BOUNDS 5

/* Human-readable description of the last error on the calling thread. */
const char* e3d_last_error(void);
/* Library version string. */
const char* e3d_version(void);

/* ------------------------------------------------------------------------
 * 1. Drop-in seam -- nonlinear propagator
 * ---------------------------------------------------------------------- */

/* Replaces bool getGpuInfo_3D(std::vector<int> gpuList, int info, int deviceNumber)
 * (nonlinearPropElasticGpuFunctions_3D.h:8).  Returns 0 when every listed
 * device exists, E3D_ERR_ARG otherwise. */
int getGpuInfo_3D(const int* gpuList, int nGpuList, int info, int deviceNumberInfo);

/* Replaces void setGpuP2P(int nGpu, int info, std::vector<int> gpuList)
 * (nonlinearPropElasticGpuFunctions_3D.h:9).  Enables peer access between
 * the listed devices where the hardware allows it. */
int setGpuP2P(int nGpu, int info, const int* gpuList);

/* Replaces initNonlinearElasticGpu_3D (nonlinearPropElasticGpuFunctions_3D.h:10).
 * Records grid, time axis, taper and filter constants for slot iGpu. */
int initNonlinearElasticGpu_3D(float dz, float dx, float dy, int nz, int nx, int ny, int nts, float dts, int sub,
                               int minPad, int blockSize, float alphaCos, int nGpu, int iGpuId, int iGpuAlloc);

/* Replaces allocateNonlinearElasticGpu_3D (nonlinearPropElasticGpuFunctions_3D.h:11).
 * Copies the eight scaled medium planes (host) to device iGpuId. */
int allocateNonlinearElasticGpu_3D(float* rhoxDtw, float* rhoyDtw, float* rhozDtw, float* lamb2MuDtw,
                                   float* lambDtw, float* muxzDtw, float* muxyDtw, float* muyzDtw, int nx, int ny,
                                   int nz, int iGpu, int iGpuId);

/* Replaces deallocateNonlinearElasticGpu_3D (nonlinearPropElasticGpuFunctions_3D.h:12). */
int deallocateNonlinearElasticGpu_3D(int iGpu, int iGpuId);

/* Replaces propElasticFwdGpu_3D (nonlinearPropElasticGpuFunctions_3D.h:15).
 * model*: nine source blocks (in); data*: nine receiver blocks (out, overwritten). */
int propElasticFwdGpu_3D(float* modelRegDts_vx, float* modelRegDts_vy, float* modelRegDts_vz,
                         float* modelRegDts_sigmaxx, float* modelRegDts_sigmayy, float* modelRegDts_sigmazz,
                         float* modelRegDts_sigmaxz, float* modelRegDts_sigmaxy, float* modelRegDts_sigmayz,
                         float* dataRegDts_vx, float* dataRegDts_vy, float* dataRegDts_vz,
                         float* dataRegDts_sigmaxx, float* dataRegDts_sigmayy, float* dataRegDts_sigmazz,
                         float* dataRegDts_sigmaxz, float* dataRegDts_sigmaxy, float* dataRegDts_sigmayz,
                         long long* sourcesPositionRegCenterGrid, long long nSourcesRegCenterGrid,
                         long long* sourcesPositionRegXGrid, long long nSourcesRegXGrid,
                         long long* sourcesPositionRegYGrid, long long nSourcesRegYGrid,
                         long long* sourcesPositionRegZGrid, long long nSourcesRegZGrid,
                         long long* sourcesPositionRegXZGrid, long long nSourcesRegXZGrid,
                         long long* sourcesPositionRegXYGrid, long long nSourcesRegXYGrid,
                         long long* sourcesPositionRegYZGrid, long long nSourcesRegYZGrid,
                         long long* receiversPositionRegCenterGrid, long long nReceiversRegCenterGrid,
                         long long* receiversPositionRegXGrid, long long nReceiversRegXGrid,
                         long long* receiversPositionRegYGrid, long long nReceiversRegYGrid,
                         long long* receiversPositionRegZGrid, long long nReceiversRegZGrid,
                         long long* receiversPositionRegXZGrid, long long nReceiversRegXZGrid,
                         long long* receiversPositionRegXYGrid, long long nReceiversRegXYGrid,
                         long long* receiversPositionRegYZGrid, long long nReceiversRegYZGrid, int nx, int ny,
                         int nz, int iGpu, int iGpuId);

/* Replaces propElasticAdjGpu_3D (nonlinearPropElasticGpuFunctions_3D.h:19).
 * data*: nine receiver blocks (in); model*: nine source blocks (out, overwritten).
 * Uses the reference's time-reversed stepper (not an exact transpose). */
int propElasticAdjGpu_3D(float* modelRegDts_vx, float* modelRegDts_vy, float* modelRegDts_vz,
                         float* modelRegDts_sigmaxx, float* modelRegDts_sigmayy, float* modelRegDts_sigmazz,
                         float* modelRegDts_sigmaxz, float* modelRegDts_sigmaxy, float* modelRegDts_sigmayz,
                         float* dataRegDts_vx, float* dataRegDts_vy, float* dataRegDts_vz,
                         float* dataRegDts_sigmaxx, float* dataRegDts_sigmayy, float* dataRegDts_sigmazz,
                         float* dataRegDts_sigmaxz, float* dataRegDts_sigmaxy, float* dataRegDts_sigmayz,
                         long long* sourcesPositionRegCenterGrid, long long nSourcesRegCenterGrid,
                         long long* sourcesPositionRegXGrid, long long nSourcesRegXGrid,
                         long long* sourcesPositionRegYGrid, long long nSourcesRegYGrid,
                         long long* sourcesPositionRegZGrid, long long nSourcesRegZGrid,
                         long long* sourcesPositionRegXZGrid, long long nSourcesRegXZGrid,
                         long long* sourcesPositionRegXYGrid, long long nSourcesRegXYGrid,
                         long long* sourcesPositionRegYZGrid, long long nSourcesRegYZGrid,
                         long long* receiversPositionRegCenterGrid, long long nReceiversRegCenterGrid,
                         long long* receiversPositionRegXGrid, long long nReceiversRegXGrid,
                         long long* receiversPositionRegYGrid, long long nReceiversRegYGrid,
                         long long* receiversPositionRegZGrid, long long nReceiversRegZGrid,
                         long long* receiversPositionRegXZGrid, long long nReceiversRegXZGrid,
                         long long* receiversPositionRegXYGrid, long long nReceiversRegXYGrid,
                         long long* receiversPositionRegYZGrid, long long nReceiversRegYZGrid, int nx, int ny,
                         int nz, int iGpu, int iGpuId);

/* Replaces propElasticFwdGpudomDec_3D (nonlinearPropElasticGpuFunctions_3D.h:15, driver
 * nonlinearPropElasticGpuFunctions_3D.cu:976-1297): the forward over y-slabs of one grid.  Slot
 * iGpu (0..nGpu-1) holds slab iGpu, allocated by allocateNonlinearElasticGpu_3D with
 * ny_domDec[iGpu] planes of the medium shifted by the planes of the slabs before it less 2*FAT
 * each (neighbours overlap by 2*FAT), on gpuList[iGpu]; init takes the whole grid's ny.
 * The slab sizes follow nonlinearPropElasticShotsGpu_3D.cpp:48-76: slab 0 ny/nGpu + FAT, middle
 * slabs ny/nGpu + 2*FAT, the last the rest + FAT; every slab needs at least 3*FAT planes.
 * Positions are global.  Each slab updates its own planes; after every fine step and its
 * injection the nine fields' FAT boundary planes go to the neighbours (peer copies between
 * GPUs).  The result equals propElasticFwdGpu_3D on the whole grid.  The reference's
 * std::vector arguments become a pointer and a count. */
int propElasticFwdGpudomDec_3D(float* modelRegDts_vx, float* modelRegDts_vy, float* modelRegDts_vz,
                               float* modelRegDts_sigmaxx, float* modelRegDts_sigmayy, float* modelRegDts_sigmazz,
                               float* modelRegDts_sigmaxz, float* modelRegDts_sigmaxy, float* modelRegDts_sigmayz,
                               float* dataRegDts_vx, float* dataRegDts_vy, float* dataRegDts_vz,
                               float* dataRegDts_sigmaxx, float* dataRegDts_sigmayy, float* dataRegDts_sigmazz,
                               float* dataRegDts_sigmaxz, float* dataRegDts_sigmaxy, float* dataRegDts_sigmayz,
                               long long* sourcesPositionRegCenterGrid, long long nSourcesRegCenterGrid,
                               long long* sourcesPositionRegXGrid, long long nSourcesRegXGrid,
                               long long* sourcesPositionRegYGrid, long long nSourcesRegYGrid,
                               long long* sourcesPositionRegZGrid, long long nSourcesRegZGrid,
                               long long* sourcesPositionRegXZGrid, long long nSourcesRegXZGrid,
                               long long* sourcesPositionRegXYGrid, long long nSourcesRegXYGrid,
                               long long* sourcesPositionRegYZGrid, long long nSourcesRegYZGrid,
                               long long* receiversPositionRegCenterGrid, long long nReceiversRegCenterGrid,
                               long long* receiversPositionRegXGrid, long long nReceiversRegXGrid,
                               long long* receiversPositionRegYGrid, long long nReceiversRegYGrid,
                               long long* receiversPositionRegZGrid, long long nReceiversRegZGrid,
                               long long* receiversPositionRegXZGrid, long long nReceiversRegXZGrid,
                               long long* receiversPositionRegXYGrid, long long nReceiversRegXYGrid,
                               long long* receiversPositionRegYZGrid, long long nReceiversRegYZGrid, int nx,
                               int ny, int nz, const int* ny_domDec, int nDomDec, const int* gpuList, int nGpu);

/* Replaces propElasticAdjGpudomDec_3D (nonlinearPropElasticGpuFunctions_3D.h:19, driver
 * nonlinearPropElasticGpuFunctions_3D.cu:1396-1719): the time-reversed adjoint over the same
 * slabs; equals propElasticAdjGpu_3D on the whole grid. */
int propElasticAdjGpudomDec_3D(float* modelRegDts_vx, float* modelRegDts_vy, float* modelRegDts_vz,
                               float* modelRegDts_sigmaxx, float* modelRegDts_sigmayy, float* modelRegDts_sigmazz,
                               float* modelRegDts_sigmaxz, float* modelRegDts_sigmaxy, float* modelRegDts_sigmayz,
                               float* dataRegDts_vx, float* dataRegDts_vy, float* dataRegDts_vz,
                               float* dataRegDts_sigmaxx, float* dataRegDts_sigmayy, float* dataRegDts_sigmazz,
                               float* dataRegDts_sigmaxz, float* dataRegDts_sigmaxy, float* dataRegDts_sigmayz,
                               long long* sourcesPositionRegCenterGrid, long long nSourcesRegCenterGrid,
                               long long* sourcesPositionRegXGrid, long long nSourcesRegXGrid,
                               long long* sourcesPositionRegYGrid, long long nSourcesRegYGrid,
                               long long* sourcesPositionRegZGrid, long long nSourcesRegZGrid,
                               long long* sourcesPositionRegXZGrid, long long nSourcesRegXZGrid,
                               long long* sourcesPositionRegXYGrid, long long nSourcesRegXYGrid,
                               long long* sourcesPositionRegYZGrid, long long nSourcesRegYZGrid,
                               long long* receiversPositionRegCenterGrid, long long nReceiversRegCenterGrid,
                               long long* receiversPositionRegXGrid, long long nReceiversRegXGrid,
                               long long* receiversPositionRegYGrid, long long nReceiversRegYGrid,
                               long long* receiversPositionRegZGrid, long long nReceiversRegZGrid,
                               long long* receiversPositionRegXZGrid, long long nReceiversRegXZGrid,
                               long long* receiversPositionRegXYGrid, long long nReceiversRegXYGrid,
                               long long* receiversPositionRegYZGrid, long long nReceiversRegYZGrid, int nx,
                               int ny, int nz, const int* ny_domDec, int nDomDec, const int* gpuList, int nGpu);

/* ------------------------------------------------------------------------
 * 1b. Drop-in seam -- Born propagator
 * ---------------------------------------------------------------------- */

/* Replaces initBornElasticGpu_3D (BornElasticGpuFunctions_3D.h:10). */
int initBornElasticGpu_3D(float dz, float dx, float dy, int nz, int nx, int ny, int nts, float dts, int sub,
                          int minPad, int blockSize, float alphaCos, int nGpu, int iGpuId, int iGpuAlloc);
/* Replaces allocateBornElasticGpu_3D (BornElasticGpuFunctions_3D.h:11). */
int allocateBornElasticGpu_3D(float* rhoxDtw, float* rhoyDtw, float* rhozDtw, float* lamb2MuDtw, float* lambDtw,
                              float* muxzDtw, float* muxyDtw, float* muyzDtw, int nx, int ny, int nz, int iGpu,
                              int iGpuId);
/* Replaces deallocateBornElasticGpu_3D (BornElasticGpuFunctions_3D.h:12). */
int deallocateBornElasticGpu_3D(int iGpu, int iGpuId);
/* Replaces allocatePinBornElasticGpu_3D (BornElasticGpuFunctions_3D.h:14).  The
 * source wavefield stays on the device (checkpoints), so no pinned host
 * memory is taken; the call only validates its arguments. */
int allocatePinBornElasticGpu_3D(int nx, int ny, int nz, int nts, int nGpu, int iGpuId, int iGpu, int iGpuAlloc);
/* Replaces deallocatePinBornElasticGpu_3D (BornElasticGpuFunctions_3D.h:15). */
int deallocatePinBornElasticGpu_3D(int iGpu, int iGpuId);

/* Replaces BornElasticFwdGpu_3D (BornElasticGpuFunctions_3D.h:18).  source*:
 * nine source blocks; data*: nine receiver blocks (out); drho*..dmuyz: the
 * eight staggered, scaled perturbation planes (in). */
int BornElasticFwdGpu_3D(float* sourceRegDts_vx, float* sourceRegDts_vy, float* sourceRegDts_vz,
                         float* sourceRegDts_sigmaxx, float* sourceRegDts_sigmayy, float* sourceRegDts_sigmazz,
                         float* sourceRegDts_sigmaxz, float* sourceRegDts_sigmaxy, float* sourceRegDts_sigmayz,
                         float* dataRegDts_vx, float* dataRegDts_vy, float* dataRegDts_vz,
                         float* dataRegDts_sigmaxx, float* dataRegDts_sigmayy, float* dataRegDts_sigmazz,
                         float* dataRegDts_sigmaxz, float* dataRegDts_sigmaxy, float* dataRegDts_sigmayz,
                         long long* sourcesPositionRegCenterGrid, long long nSourcesRegCenterGrid,
                         long long* sourcesPositionRegXGrid, long long nSourcesRegXGrid,
                         long long* sourcesPositionRegYGrid, long long nSourcesRegYGrid,
                         long long* sourcesPositionRegZGrid, long long nSourcesRegZGrid,
                         long long* sourcesPositionRegXZGrid, long long nSourcesRegXZGrid,
                         long long* sourcesPositionRegXYGrid, long long nSourcesRegXYGrid,
                         long long* sourcesPositionRegYZGrid, long long nSourcesRegYZGrid,
                         long long* receiversPositionRegCenterGrid, long long nReceiversRegCenterGrid,
                         long long* receiversPositionRegXGrid, long long nReceiversRegXGrid,
                         long long* receiversPositionRegYGrid, long long nReceiversRegYGrid,
                         long long* receiversPositionRegZGrid, long long nReceiversRegZGrid,
                         long long* receiversPositionRegXZGrid, long long nReceiversRegXZGrid,
                         long long* receiversPositionRegXYGrid, long long nReceiversRegXYGrid,
                         long long* receiversPositionRegYZGrid, long long nReceiversRegYZGrid, float* drhox,
                         float* drhoy, float* drhoz, float* dlame, float* dmu, float* dmuxz, float* dmuxy,
                         float* dmuyz, int nx, int ny, int nz, int iGpu, int iGpuId);

/* Replaces BornElasticAdjGpu_3D (BornElasticGpuFunctions_3D.h:21).  The image
 * is accumulated onto the caller's eight planes (the reference copies them
 * to the device first and copies the sum back). */
int BornElasticAdjGpu_3D(float* sourceRegDts_vx, float* sourceRegDts_vy, float* sourceRegDts_vz,
                         float* sourceRegDts_sigmaxx, float* sourceRegDts_sigmayy, float* sourceRegDts_sigmazz,
                         float* sourceRegDts_sigmaxz, float* sourceRegDts_sigmaxy, float* sourceRegDts_sigmayz,
                         float* dataRegDts_vx, float* dataRegDts_vy, float* dataRegDts_vz,
                         float* dataRegDts_sigmaxx, float* dataRegDts_sigmayy, float* dataRegDts_sigmazz,
                         float* dataRegDts_sigmaxz, float* dataRegDts_sigmaxy, float* dataRegDts_sigmayz,
                         long long* sourcesPositionRegCenterGrid, long long nSourcesRegCenterGrid,
                         long long* sourcesPositionRegXGrid, long long nSourcesRegXGrid,
                         long long* sourcesPositionRegYGrid, long long nSourcesRegYGrid,
                         long long* sourcesPositionRegZGrid, long long nSourcesRegZGrid,
                         long long* sourcesPositionRegXZGrid, long long nSourcesRegXZGrid,
                         long long* sourcesPositionRegXYGrid, long long nSourcesRegXYGrid,
                         long long* sourcesPositionRegYZGrid, long long nSourcesRegYZGrid,
                         long long* receiversPositionRegCenterGrid, long long nReceiversRegCenterGrid,
                         long long* receiversPositionRegXGrid, long long nReceiversRegXGrid,
                         long long* receiversPositionRegYGrid, long long nReceiversRegYGrid,
                         long long* receiversPositionRegZGrid, long long nReceiversRegZGrid,
                         long long* receiversPositionRegXZGrid, long long nReceiversRegXZGrid,
                         long long* receiversPositionRegXYGrid, long long nReceiversRegXYGrid,
                         long long* receiversPositionRegYZGrid, long long nReceiversRegYZGrid, float* drhox,
                         float* drhoy, float* drhoz, float* dlame, float* dmu, float* dmuxz, float* dmuxy,
                         float* dmuyz, int nx, int ny, int nz, int iGpu, int iGpuId);

/* ------------------------------------------------------------------------
 * 2. Explicit-context API
 * ---------------------------------------------------------------------- */
typedef struct e3d_context e3d_context;

typedef struct e3d_desc {
  int device;
  int nz, nx, ny;
  int nts;        /* coarse samples */
  int sub;        /* internal subsampling (2x the parameter-file value) */
  int minPad;
  float dz, dx, dy, dts, alphaCos;
  int fix_q1;     /* 1: y derivatives divide by dy (the reference divides by dx) */
  int q2compat;   /* 1: sxz receivers read the z-grid table (reference behaviour) */
  int q3compat;   /* 1: Born yz shear term uses the xz derivative pair (reference behaviour) */
  int free_surface; /* 1: stress-free surface at z = FAT, the top face not tapered; nonlinear
                       propagation only (the reference parses freeSurface but implements none,
                       fdParamElastic_3D.cpp:44-45); 0: the reference's sponge on all faces */
} e3d_desc;

/* Counterpart of initNonlinearElasticGpu_3D + allocateNonlinearElasticGpu_3D
 * with an explicit handle instead of process-global slots. */
int e3d_context_create(const e3d_desc* desc, e3d_context** out);
int e3d_context_destroy(e3d_context* ctx);
/* Eight medium planes (see allocateNonlinearElasticGpu_3D); on_device != 0 for device pointers. */
int e3d_set_medium(e3d_context* ctx, const float* const* planes8, int on_device);
/* Stepper variant (autotuner hook): tile width along x (8 or 16), shared-memory
 * pipeline depth (2 or 3 stages; 2 to 4 with loaders 6 to 8) and plane loader (0 plain
 * loads, 1 cp.async, 2 TMA bulk tensor copies, 3-5 TMA with a rotating y-window,
 * 6 TMA with the velocity and stress updates of a step as two CTA roles of one
 * launch, 8-wide tiles, 7 the same for the forward and time-reversed steps with
 * the exact adjoint on loader 2's stepper, 8 as 7 with each thread updating two
 * consecutive z cells from paired shared-memory loads; 1 to 8 need nz % 4 == 0). */
int e3d_set_stepper_variant(e3d_context* ctx, int tx, int stages, int loader);
/* Nonlinear propagation (e3d_nl_* and the seam's propElastic*Gpu_3D): on = 1
 * (default) captures one coarse block as a CUDA graph after running the first
 * block eagerly and replays it for the others, the coarse time index living on
 * the device; 0 launches every kernel from the host.  Graphs are not used on
 * the legacy default stream or while stepper timing samples are being taken. */
int e3d_set_graph_loop(e3d_context* ctx, int on);
/* Autotuner hook: the number of y chunks each (z, x) tile column of the
 * stepper grid is split into (CTAs = z tiles * x tiles * chunks); 0 = automatic. */
int e3d_set_stepper_chunks(e3d_context* ctx, int chunks);
/* Checkpoint storage: type -1 = chosen among fp32 states with fp32 velocity
 * slots, fp16 states with fp32 slots, fp16 states with fp16 slots (default);
 * 0 = fp32, 1 = fp16, 2 = bf16 (16-bit types carry one scale per y-slice and
 * field).  Each candidate takes the longest segment that fits; the one that
 * recomputes the fewest source blocks wins, a 16-bit plan only where it saves
 * more than 5% (states) / 5% (velocity slots) of the blocks.  The forward pass
 * keeps the last segment's velocity, so only the earlier segments are recomputed;
 * segment = coarse blocks per segment (0 = automatic), segments aligned to the
 * end of the record;
 * budget_bytes > 0: device bytes for checkpoints and velocity slots; 0: 85% of the
 * free memory; < 0: 85% of the free memory minus |budget_bytes| kept for the caller. */
int e3d_set_checkpoint_policy(e3d_context* ctx, int type, int segment, double budget_bytes);
/* Wait for all work queued on the context's stream; reports an expired
 * bounded pipeline wait inside the stepper as E3D_ERR_CUDA. */
int e3d_synchronize(e3d_context* ctx);
/* cudaStream_t of the context, as void*. */
void* e3d_stream(e3d_context* ctx);
/* Queue the context's work on an existing cudaStream_t (passed as void*), e.g. the
 * caller's framework stream; a NULL handle is the legacy default stream.
 * use_own != 0 returns to the context's own stream (stream is then ignored). */
int e3d_set_stream(e3d_context* ctx, void* stream, int use_own);
/* Updated cells per fine step ((nz-8)(nx-8)(ny-8)). */
long long e3d_cells_per_step(const e3d_context* ctx);
/* Coarse blocks per checkpoint segment chosen by the last checkpointed forward (0 before). */
int e3d_checkpoint_segment(const e3d_context* ctx);
/* Storage of the decimated source velocity kept per segment for the imaging
 * condition: -1 = as the checkpoint plan chooses (default), 0 = fp32,
 * 1 = fp16 with one scale per y-slice and field. */
int e3d_set_velocity_storage(e3d_context* ctx, int type);
/* Velocity slot storage of the current plan (0 fp32, 1 fp16). */
int e3d_velocity_storage(const e3d_context* ctx);
/* State storage of the current checkpoints (0 fp32, 1 fp16, 2 bf16). */
int e3d_checkpoint_type(const e3d_context* ctx);
/* How the checkpointed passes decimate fine levels into coarse samples (the
 * reference's interpWavefieldVxVyVz_3D and extractInterpAdjointWavefield_3D,
 * kernelsElaGpu_3D.cu:1646-1672, 1694-1714, which run at every fine step):
 * on = 1 (default): the fine levels of a coarse block stay in a ring of
 * sub+1 levels and one launch per block decimates them (the adjoint's launch
 * also applies the imaging condition); on = 0: two coarse accumulators are
 * read and written by the stepper at every fine step.  Blocks longer than 8
 * fine steps always use the accumulators.  Invalidates the checkpoints. */
int e3d_set_decimation_ring(e3d_context* ctx, int on);
/* y chunks of the block imaging launch of the decimation ring (0 = automatic:
 * the rule of the stepper grids).  A tuning knob; no counterpart in the reference. */
int e3d_set_imaging_chunks(e3d_context* ctx, int chunks);
/* Kernel of that block imaging: 0 = automatic (2 where the TMA forms apply:
 * nz % 4 == 0 and a TMA stepper loader, else 1), 1 = one thread per cell
 * reading every operand from global memory, 2 = y-march with the velocity
 * tiles staged by TMA and the adjoint levels read per cell, 3 = y-march with
 * the velocity tiles, the adjoint levels and the medium staged by TMA (one
 * CTA per SM; measured slower than 2 on B200 at sub = 4), 4 = 3 on 4-wide
 * tiles (three CTAs per SM).  The same sums in the same order; a tuning knob
 * with no counterpart in the reference. */
int e3d_set_imaging_variant(e3d_context* ctx, int variant);
/* State of the exact adjoint (the transpose of stepFwdGpu_3D's update, as
 * stepAdjGpuBorn_3D, kernelsElaGpu_3D.cu:825-1177) in the checkpointed passes
 * with a decimation ring.  on = 1 (default): where the medium allows it -- all
 * density and shear planes positive and the normal-stress block of the
 * premultiplication conditioned within 100 -- only the medium-premultiplied
 * levels P = M a are stored (140 B per cell and step): the update
 * a_new = G(G a_old - D(P_cur)) then reads P_new = G(G P_old - M D(P_cur)), the
 * reference's time-reversed stepper (stepAdjGpu_3D) applied to P, and the
 * imaging converts its decimated sums back to raw values once per coarse
 * block; otherwise, and with on = 0, the raw and the premultiplied levels both
 * (176 B).  The choice is made per medium. */
int e3d_set_premultiplied_adjoint(e3d_context* ctx, int on);
/* The checkpoint schedule of a record of `blocks` coarse blocks (nts - 1) cut
 * into segments of `segment_len` blocks, as the checkpointed passes run it:
 * returns the segment count nseg, or -E3D_ERR_ARG.  seg_start (room for
 * max_segments + 1 values, may be NULL) receives the first block of each
 * segment and then `blocks`: segments are aligned to the end of the record
 * and the first holds the remainder.  *recomputed (may be NULL) receives the
 * source blocks the adjoint pass recomputes (every segment but the last, whose
 * velocity the forward pass keeps).  No device work; no counterpart in the
 * reference, whose Born adjoint stores the whole source wavefield on the host
 * (BornElasticGpuFunctions_3D.cu:1268-1316). */
int e3d_checkpoint_schedule(int blocks, int segment_len, int* seg_start, int max_segments, int* recomputed);
/* The checkpoint plan the checkpointed passes choose for a padded grid of
 * n_cells cells in ny y slices, nts coarse samples and budget_bytes of device
 * memory for checkpoints and velocity slots (the passes use 85% of the free
 * memory, less the caller's reserve and the adjoint pass's working fields):
 * ckpt_type / velocity_type / segment as in e3d_set_checkpoint_policy and
 * e3d_set_velocity_storage.  Outputs (each may be NULL): the state and slot
 * storage types, the segment length and the plan's bytes.  E3D_ERR_OOM when
 * nothing fits.  No device work. */
int e3d_checkpoint_plan(long long n_cells, int ny, int nts, double budget_bytes, int ckpt_type, int velocity_type,
                        int segment, int* ckpt_used, int* velocity_used, int* segment_len, double* plan_bytes);

/* Host-buffer propagations.  src_pos/rec_pos: 7 tables; n_src/n_rec: 7 counts. */
int e3d_nl_forward(e3d_context* ctx, const float* const* model9, float* const* data9,
                   const long long* const* src_pos, const long long* n_src, const long long* const* rec_pos,
                   const long long* n_rec);
int e3d_nl_adjoint(e3d_context* ctx, float* const* model9, const float* const* data9,
                   const long long* const* src_pos, const long long* n_src, const long long* const* rec_pos,
                   const long long* n_rec);
/* One shot over y-slab contexts (the explicit-context form of
 * propElasticFwdGpudomDec_3D / propElasticAdjGpudomDec_3D): slabs[s] are
 * contexts of the same parameters created with ny_domDec[s] planes and their
 * slab of the medium (planes shifted by the planes of the slabs before it less
 * 2*FAT each); ny_global is the whole grid's ny.  Positions are global and the
 * signals are as e3d_nl_forward (adjoint = 0) or e3d_nl_adjoint (adjoint = 1).
 * The contexts may share a device. */
int e3d_nl_propagate_slabs(e3d_context* const* slabs, int n_slabs, int ny_global, int adjoint, float* const* model9,
                           float* const* data9, const long long* const* src_pos, const long long* n_src,
                           const long long* const* rec_pos, const long long* n_rec);
int e3d_born_forward(e3d_context* ctx, const float* const* src9, float* const* data9,
                     const long long* const* src_pos, const long long* n_src, const long long* const* rec_pos,
                     const long long* n_rec, const float* const* pert8);
int e3d_born_adjoint(e3d_context* ctx, const float* const* src9, const float* const* data9,
                     const long long* const* src_pos, const long long* n_src, const long long* const* rec_pos,
                     const long long* n_rec, float* const* pert8);

/* Device-buffer propagations.  Signals are time-major [nts][ntot] with the
 * nine components concatenated; pos_dev is the matching int64 table and
 * off10[k]..off10[k+1] is component k's range.  Work is queued on the
 * context's stream; call e3d_synchronize before reading outputs.
 * Before anything is written, a read-only kernel checks the position tables
 * (e3d_nl_propagate_device, e3d_fwi_forward_device, e3d_fwi_gradient_device
 * and e3d_nl_propagate_device_noalloc): an entry inside the FAT ring or outside
 * the grid returns E3D_ERR_BOUNDS, as the host-buffer calls do for host
 * tables.  The check waits for the stream once per call. */
int e3d_nl_propagate_device(e3d_context* ctx, int adjoint, const long long* src_pos_dev, const int* src_off10,
                            const long long* rec_pos_dev, const int* rec_off10, float* src_sig_dev,
                            float* rec_sig_dev);
/* Batched nonlinear forward: `shots` shots in the context's medium advanced
 * together, one stepper launch per fine step for all of them (the reference
 * runs one propElasticFwdGpu_3D per shot from an OpenMP loop over GPUs,
 * nonlinearPropElasticShotsGpu_3D.cpp:177-216).  The position tables and
 * signals are the concatenation over shots, component-major: component k's
 * range off10[k]..off10[k+1] holds the entries of every shot, and an entry of
 * shot s carries s*nz*nx*ny added to its grid position.  Signals are
 * time-major over the combined tables.  The shots' wavefields take
 * 18*shots*nz*nx*ny floats; nz % 4 == 0; no free surface.  The tables are
 * checked on the device first, as above, against the stacked grids. */
int e3d_nl_forward_batch_device(e3d_context* ctx, int shots, const long long* src_pos_dev, const int* src_off10,
                                const long long* rec_pos_dev, const int* rec_off10, const float* src_sig_dev,
                                float* rec_sig_dev);
/* Irregular receivers as linear combinations of the regular receiver points
 * (spaceInterpGpu_3D::forward/adjoint, spaceInterpGpu_3D.cpp:140-175), all
 * arrays on the device.  Receiver row r = k*n_irreg + i for component k.
 *   regular -> irregular: irr[r] = sum_{f<n_taps} weight[r*n_taps+f] * reg[slot[r*n_taps+f]]
 *   irregular -> regular: reg[j] = sum_{row_ptr[j] <= e < row_ptr[j+1]} w[e] * irr[idx[e]]
 * slot and j index the concatenated regular receiver list (rec_pos_dev);
 * entries outside the lists contribute nothing. */
typedef struct e3d_trace_map {
  int n_irreg;
  int n_taps;
  const int* slot;
  const float* weight;
  const int* row_ptr;
  const int* idx;
  const float* w;
} e3d_trace_map;

/* FWI: nonlinear forward that also saves on-device wavefield checkpoints.
 * map == NULL: rec_sig_dev is regular-grid, time-major [nts][rec_off10[9]].
 * map != NULL: rec_sig_dev is irregular, time-major [nts][9*n_irreg]; the
 * regular traces only exist as a two-slice ring on the device. */
int e3d_fwi_forward_device(e3d_context* ctx, const long long* src_pos_dev, const int* src_off10,
                           const long long* rec_pos_dev, const int* rec_off10, const float* src_sig_dev,
                           float* rec_sig_dev, const e3d_trace_map* map);
/* FWI: Born adjoint of the residual, accumulated into eight device planes;
 * consumes the checkpoints of the preceding e3d_fwi_forward_device.  The
 * residual has the layout of rec_sig_dev above for the same map.
 * src_adj_dev (optional, time-major [nts][src_off10[9]], overwritten): the
 * exact adjoint of the nonlinear propagation with respect to the scaled
 * source signals -- the residual propagated by the exact-transpose stepper
 * and sampled at the source points with the transposed injection weights and
 * taper.  It makes the exact nonlinear adjoint available (the reference's
 * propElasticAdjGpu_3D runs the time-reversed stepper instead) and gives the
 * misfit's derivative through the medium scaling of the sources. */
int e3d_fwi_gradient_device(e3d_context* ctx, const long long* src_pos_dev, const int* src_off10,
                            const long long* rec_pos_dev, const int* rec_off10, const float* src_sig_dev,
                            const float* residual_dev, float* const* grad8_dev, const e3d_trace_map* map,
                            float* src_adj_dev);

/* Allocation-free variant of e3d_nl_propagate_device.  It has no counterpart
 * in the reference (whose drivers allocate and free device buffers on every
 * call).  It serves callers that cannot allocate device memory while they
 * propagate: a host framework that already holds most of the device's memory
 * in its own pool, or a loop that must not make cudaMalloc/cudaFree calls,
 * which can synchronize the whole device.  Nothing is allocated: the two
 * wavefield levels and the sponge taper live in one fixed device array of
 * e3d_noalloc_work_bytes() = 64 MiB, which every GPU that loads this library
 * holds until the process exits.  That limits the grid to nz*nx*ny of about
 * 0.93 M cells (18 float fields, the taper and one status word); larger grids
 * return E3D_ERR_ARG with the sizes in e3d_last_error().  No context is needed: the propagation runs on
 * the calling thread's current device, on `stream` (NULL = legacy default
 * stream), with the stepper of the "plain" variant; desc->device is ignored
 * and desc->free_surface must be 0.
 * planes8_dev: the eight medium planes on that device; positions, offsets and
 * time-major signals as for e3d_nl_propagate_device (the output signals are
 * overwritten).  The first call on a device looks up the device address of
 * the array (cudaGetSymbolAddress, with the device current) and caches it;
 * make that first call before any stream capture.  The cached address
 * belongs to the device's primary context; a call that finds another primary
 * context current (after cudaDeviceReset) looks the address up again.  Every call on a device
 * uses the same array and clears it at the start, so calls that overlap on
 * the GPU (on different streams, or from different threads) race and give
 * wrong results; order them on one stream. */
int e3d_nl_propagate_device_noalloc(const e3d_desc* desc, const float* const* planes8_dev, int adjoint,
                                    const long long* src_pos_dev, const int* src_off10,
                                    const long long* rec_pos_dev, const int* rec_off10, float* src_sig_dev,
                                    float* rec_sig_dev, void* stream);
/* Size in bytes of the fixed device array used by e3d_nl_propagate_device_noalloc. */
size_t e3d_noalloc_work_bytes(void);

/* Sampled kernel timing for roofline reporting: every n-th launch of each
 * timed kind is bracketed by CUDA events on the launching stream (n = 0
 * switches it off). */
int e3d_kernel_timing(e3d_context* ctx, int every);
/* Mean duration in ms and number of the sampled launches of one kind since
 * the previous read (waits for them to finish).  mode 0..2: bare steps of that
 * stepper mode; 3..5: the same modes with a fused decimation into coarse
 * accumulators or a fused Born secondary source; 6: the block imaging of the
 * decimation ring; 7: its source-velocity decimation.  The exact adjoint on the
 * premultiplied-only state runs as mode 1 (see e3d_set_premultiplied_adjoint). */
int e3d_kernel_timing_read(e3d_context* ctx, int mode, double* avg_ms, long long* count);
/* Number of kernel launches this context has issued. */
long long e3d_launch_count(const e3d_context* ctx);

/* Bare stepper (mode 0 forward, 1 time-reversed, 2 exact transpose on the dual
 * state) applied n_steps times to the context's working wavefields; for
 * benchmarking.  Modes 3..5 run modes 0..2 with the new level decimated into
 * two coarse accumulators (3 velocity fields for modes 3 and 4, all 9 fields for
 * 5), as the fused-accumulator passes do. */
int e3d_step_only(e3d_context* ctx, int mode, int n_steps);

/* ------------------------------------------------------------------------
 * Host preparation (native counterparts of the reference's C++ host code)
 * ---------------------------------------------------------------------- */
/* fdParamElastic_3D medium preparation (fdParamElastic_3D.cpp:130-193):
 * elastic = [rho; lambda; mu] (3*nz*nx*ny, z fastest) -> eight scaled planes. */
int e3d_medium_planes(int nz, int nx, int ny, float dtw, const float* elastic, float* const* out8);

/* staggerX/Y/Z forward (adjoint=0) or adjoint (adjoint=1), axis 0=z 1=x 2=y,
 * out = (add ? out : 0) + op(in)   (stagger_3D.cpp:23-208). */
int e3d_stagger(int nz, int nx, int ny, int axis, int adjoint, int add, const float* in, float* out);

/* spaceInterpGpu_3D linear weights and unique regular-grid points
 * (spaceInterpGpu_3D.cpp:113-138, 178-348) for one grid.
 * grid: nz,nx,ny; origins/samplings as float; pads[6] = fat, zPadMinus,
 * zPadPlus, xPadMinus, xPadPlus, yPad.  Outputs (caller-sized):
 *   index[nDev*nFilter], weight[nDev*nFilter], unique[<= nDev*nFilter], slot[nDev*nFilter];
 *   *n_unique receives the unique count.  nFilter = 8, or 16 with dipole. */
int e3d_space_interp_linear(const float* z, const float* x, const float* y, long long n_dev, int nz, int nx, int ny,
                            float oz, float ox, float oy, float dz, float dx, float dy, const int* pads6,
                            float error_tolerance, int dipole, float zshift, float xshift, float yshift,
                            long long* index, float* weight, long long* unique, long long* slot,
                            long long* n_unique);

/* spaceInterpGpu_3D with a choice of method (spaceInterpGpu_3D.cpp:13-79,
 * 178-480): E3D_INTERP_LINEAR (h_filter must be 1) or E3D_INTERP_SINC with
 * h_filter points on each side per axis.  nFilter = (2*h_filter)^3 points per
 * pole, z fastest then x then y, doubled with dipole.  Sinc weights are
 * sinc(wz) sinc(wx) sinc(wy), sinc(w) = sin(pi w)/(pi w), in double stored as
 * float; the stencil must lie inside the array.  The reference's sinc path
 * rejects every in-bounds stencil (its bounds test is inverted), so no output
 * of it exists to match: this is that path with the test written the right
 * way round.  compat = 1 keeps the reference's dipole arithmetic (shifts
 * truncated to int; the linear second pole's y offset divided by dz; the sinc
 * second pole with positive weights); compat = 0 corrects it (float shifts,
 * dy, negative second-pole weights for both methods).  With compat = 1 and
 * the linear method this is e3d_space_interp_linear. */
#define E3D_INTERP_LINEAR 0
#define E3D_INTERP_SINC 1
int e3d_space_interp(int method, int h_filter, const float* z, const float* x, const float* y, long long n_dev,
                     int nz, int nx, int ny, float oz, float ox, float oy, float dz, float dx, float dy,
                     const int* pads6, float error_tolerance, int dipole, float zshift, float xshift, float yshift,
                     int compat, long long* index, float* weight, long long* unique, long long* slot,
                     long long* n_unique);

#ifdef __cplusplus
}
#endif
#endif /* ELASTIC3D_B200_H */
