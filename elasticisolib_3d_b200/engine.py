"""Python handle on one propagation context of the native engine.

A ``Propagator`` owns an ``e3d_context`` (device buffers, stream) for one grid
and time axis.  Host-array methods mirror the reference drivers
(propElasticFwdGpu_3D, propElasticAdjGpu_3D, BornElasticFwdGpu_3D,
BornElasticAdjGpu_3D) with signal blocks in the reference layout: a list of
nine float32 arrays, component k shaped (nDevice_k, nts).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N
from .hostprep import FAT

# grid of each wavefield component: vx->x, vy->y, vz->z, sxx/syy/szz->center, sxz->xz, sxy->xy, syz->yz
COMP_GRID = (1, 2, 3, 0, 0, 0, 4, 5, 6)
CKPT_TYPES = {"auto": -1, "fp32": 0, "fp16": 1, "bf16": 2}


def _geom(pos7):
    pos = [N.as_i64(p) for p in pos7]
    P = N.ptr_array(pos)
    C = (ctypes.c_longlong * 7)(*[int(p.shape[0]) for p in pos])
    return P, C, pos


def domain_decomposition(ny, n_gpu, fat=None, min_pad=0):
    """y-slab sizes (ny_domDec) of a grid of ny planes over n_gpu GPUs, by the reference's rule
    (nonlinearPropElasticShotsGpu_3D.cpp:48-76): slab 0 takes ny//n_gpu + fat planes, middle slabs
    ny//n_gpu + 2*fat, the last the rest + fat; neighbours overlap by 2*fat planes.  Raises
    ValueError where the reference refuses the split (one GPU, or too few planes per slab)."""
    fat = FAT if fat is None else fat
    if n_gpu < 2:
        raise ValueError("domain decomposition needs at least two GPUs")
    chunk = ny // n_gpu
    if (chunk <= 3 * fat and n_gpu > 2) or (chunk <= 2 * fat and n_gpu == 2) or chunk - 2 * fat <= min_pad:
        raise ValueError("decomposition not feasible with this ny; use fewer GPUs")
    sizes = [chunk + fat] + [chunk + 2 * fat] * (n_gpu - 2) + [ny - chunk * (n_gpu - 1) + fat]
    return sizes


def forward_batch_plan(n_shots, n_cells, nts, src_points, rec_points, free_bytes, margin=0.9):
    """Shots per batched forward launch admitted by device memory: each shot of a batch holds both
    leapfrog levels of the nine fields (18 * n_cells floats), its time-major source and receiver
    signals (nts * (src_points + rec_points) floats) and its position tables (8 B per point);
    at most `margin` of `free_bytes` is used.  Returns the batches as lists of shot indices, as
    even in size as the budget allows.  ValueError when not even one shot fits."""
    if n_shots < 1:
        return []
    per_shot = 18 * int(n_cells) * 4 + int(nts) * (int(src_points) + int(rec_points)) * 4 + \
        8 * (int(src_points) + int(rec_points))
    k = int(margin * float(free_bytes)) // per_shot
    if k < 1:
        raise ValueError(f"one shot needs {per_shot / 1e9:.2f} GB of device memory, "
                         f"{margin * float(free_bytes) / 1e9:.2f} GB are available")
    n_batches = -(-n_shots // min(k, n_shots))
    base, extra = divmod(n_shots, n_batches)
    out, start = [], 0
    for b in range(n_batches):
        size = base + (1 if b < extra else 0)
        out.append(list(range(start, start + size)))
        start += size
    return out


def checkpoint_schedule(blocks, segment_len):
    """Checkpoint schedule of a record of `blocks` coarse blocks (nts - 1) with segments of
    `segment_len` blocks, as the engine runs it: (first block of each segment followed by
    `blocks`, source blocks the adjoint pass recomputes).  Host arithmetic only."""
    nmax = -(-int(blocks) // max(1, min(int(segment_len), int(blocks))))
    starts = (ctypes.c_int * (nmax + 1))()
    rec = ctypes.c_int(0)
    n = int(N.lib().e3d_checkpoint_schedule(int(blocks), int(segment_len), starts, nmax, ctypes.byref(rec)))
    if n < 0:
        raise ValueError(f"bad checkpoint schedule arguments: blocks={blocks}, segment_len={segment_len}")
    return list(starts[:n + 1]), rec.value


def checkpoint_plan(n_cells, ny, nts, budget_bytes, ckpt="auto", velocity="auto", segment=0):
    """The checkpoint plan the engine chooses for a padded grid of n_cells cells in ny y slices,
    nts coarse samples and budget_bytes for checkpoints and velocity slots: (state storage,
    velocity-slot storage, segment length, plan bytes), or None when nothing fits.  Host
    arithmetic only."""
    ck, vt, L, b = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0)
    st = int(N.lib().e3d_checkpoint_plan(int(n_cells), int(ny), int(nts), float(budget_bytes), CKPT_TYPES[ckpt],
                                         {"auto": -1, "fp32": 0, "fp16": 1}[velocity], int(segment),
                                         ctypes.byref(ck), ctypes.byref(vt), ctypes.byref(L), ctypes.byref(b)))
    if st == N.E3D_ERR_OOM:
        return None
    if st != N.E3D_OK:
        raise ValueError(f"bad checkpoint plan arguments (status {st})")
    return ("fp32", "fp16", "bf16")[ck.value], ("fp32", "fp16")[vt.value], L.value, b.value


class SlabPropagator:
    """One grid decomposed into y-slabs (the reference's domain decomposition): a Propagator per
    slab, each over ny_domdec[s] planes of the medium, slab s starting at global plane
    sum(ny_domdec[:s]) - 2*FAT*s; nl_forward / nl_adjoint take and return what Propagator's do on
    the whole grid (global positions) and give the same traces (e3d_nl_propagate_slabs).  The
    slabs may share a device."""

    def __init__(self, nz, nx, ny, nts, sub, minPad, dz, dx, dy, dts, alphaCos=0.99, devices=(0, 1),
                 ny_domdec=None, **kw):
        self.ny, self.nts = int(ny), int(nts)
        self.sizes = list(ny_domdec) if ny_domdec is not None else domain_decomposition(ny, len(devices), FAT,
                                                                                           minPad)
        if len(self.sizes) != len(devices):
            raise ValueError("one slab size per device")
        self.y0 = [0]
        for sz in self.sizes[:-1]:
            self.y0.append(self.y0[-1] + sz - 2 * FAT)  # neighbours overlap by 2*FAT planes
        self.slabs = [Propagator(nz, nx, sz, nts, sub, minPad, dz, dx, dy, dts, alphaCos, device=d, **kw)
                      for sz, d in zip(self.sizes, devices)]

    def set_medium(self, planes8):
        """Eight scaled medium planes of the whole grid, numpy (8, ny, nx, nz)."""
        for pr, y0, sz in zip(self.slabs, self.y0, self.sizes):
            pr.set_medium(np.ascontiguousarray(np.asarray(planes8)[:, y0:y0 + sz]))

    def _run(self, adjoint, model, data, src_pos7, rec_pos7):
        SP, SN, k1 = _geom(src_pos7)
        RP, RN, k2 = _geom(rec_pos7)
        hs = (ctypes.c_void_p * len(self.slabs))(*[pr.handle.value for pr in self.slabs])
        N.call("e3d_nl_propagate_slabs", hs, len(self.slabs), self.ny, int(adjoint), N.ptr_array(model),
               N.ptr_array(data), SP, SN, RP, RN)

    def nl_forward(self, model9, src_pos7, rec_pos7):
        model = [N.as_f32(m) for m in model9]
        data = [np.zeros((len(rec_pos7[COMP_GRID[k]]), self.nts), dtype=np.float32) for k in range(9)]
        self._run(False, model, data, src_pos7, rec_pos7)
        return data

    def nl_adjoint(self, data9, src_pos7, rec_pos7):
        data = [N.as_f32(d) for d in data9]
        model = [np.zeros((len(src_pos7[COMP_GRID[k]]), self.nts), dtype=np.float32) for k in range(9)]
        self._run(True, model, data, src_pos7, rec_pos7)
        return model

    def close(self):
        for pr in self.slabs:
            pr.close()


class BatchTables:
    """Stacked device tables of a batched forward (see Propagator.batch_tables)."""

    def __init__(self, shots, src_pos, src_off, rec_pos, rec_off, src_sig, rec_sig, lengths=None):
        self.shots, self.src_pos, self.src_off = shots, src_pos, list(src_off)
        self.rec_pos, self.rec_off, self.src_sig, self.rec_sig = rec_pos, list(rec_off), src_sig, rec_sig
        self.lengths = list(lengths) if lengths is not None else [src_sig.shape[0]] * shots

    def split(self, out):
        """Per-shot nine receiver blocks (n_k, nts_s) of a receiver-major array out (total, nts),
        each shot's traces cut to its own record length."""
        data = [[None] * 9 for _ in range(self.shots)]
        for k in range(9):
            nk = (self.rec_off[k + 1] - self.rec_off[k]) // self.shots
            for s in range(self.shots):
                a = self.rec_off[k] + s * nk
                data[s][k] = np.ascontiguousarray(out[a:a + nk, :self.lengths[s]])
        return data


class Propagator:
    def __init__(self, nz, nx, ny, nts, sub, minPad, dz, dx, dy, dts, alphaCos=0.99, device=0, fix_q1=0,
                 q2compat=1, q3compat=1, free_surface=0):
        self.nz, self.nx, self.ny, self.nts, self.sub = int(nz), int(nx), int(ny), int(nts), int(sub)
        self.shape = (self.ny, self.nx, self.nz)
        d = N.E3DDesc(int(device), self.nz, self.nx, self.ny, self.nts, self.sub, int(minPad), float(dz), float(dx),
                      float(dy), float(dts), float(alphaCos), int(fix_q1), int(q2compat), int(q3compat),
                      int(free_surface))
        self._h = ctypes.c_void_p()
        N.call("e3d_context_create", ctypes.byref(d), ctypes.byref(self._h))
        self.device = int(device)
        self.q2compat = int(q2compat)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            N.lib().e3d_context_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_medium(self, planes8):
        """Eight scaled medium planes: numpy (8, ny, nx, nz) float32, or a device tensor of that shape."""
        if hasattr(planes8, "data_ptr"):
            assert planes8.is_cuda and planes8.dtype.is_floating_point and planes8.is_contiguous()
            ptrs = N.ptr_array([planes8[k] for k in range(8)])
            N.call("e3d_set_medium", self._h, ptrs, 1)
        else:
            planes = [N.as_f32(planes8[k]) for k in range(8)]
            N.call("e3d_set_medium", self._h, N.ptr_array(planes), 0)

    LOADERS = {"plain": 0, "cpasync": 1, "tma": 2, "tma-ring": 3, "tma-ring-ldg": 4, "tma-ring-ldg2": 5, "split": 6,
               "split-fwd": 7, "split-pair": 8}

    def set_stepper_variant(self, tx=8, stages=3, loader="split-pair"):
        """Stepper variant: x tile width (8/16), shared-memory stages (2/3) and plane loader."""
        N.call("e3d_set_stepper_variant", self._h, int(tx), int(stages), self.LOADERS[loader])

    def set_graph_loop(self, on=True):
        """Replay coarse blocks of the nonlinear loop as CUDA graphs (default on)."""
        N.call("e3d_set_graph_loop", self._h, int(bool(on)))

    def set_stepper_chunks(self, chunks=0):
        """y chunks per (z, x) tile column of the stepper grid (0 = automatic)."""
        N.call("e3d_set_stepper_chunks", self._h, int(chunks))

    def set_checkpoint_policy(self, ckpt="auto", segment=0, budget_bytes=0.0):
        N.call("e3d_set_checkpoint_policy", self._h, CKPT_TYPES[ckpt], int(segment), float(budget_bytes))

    def set_stream(self, stream):
        """Queue work on an existing CUDA stream (a torch.cuda.Stream or a raw handle; handle 0 is
        the legacy default stream); None returns to the context's own stream."""
        if stream is None:
            N.call("e3d_set_stream", self._h, None, 1)
        else:
            N.call("e3d_set_stream", self._h, int(getattr(stream, "cuda_stream", stream)) or None, 0)

    def synchronize(self):
        N.call("e3d_synchronize", self._h)

    @property
    def checkpoint_type(self):
        """State storage of the current checkpoints: "fp32", "fp16" or "bf16"."""
        return ("fp32", "fp16", "bf16")[int(N.lib().e3d_checkpoint_type(self._h))]

    @property
    def checkpoint_segment(self):
        return int(N.lib().e3d_checkpoint_segment(self._h))

    @property
    def cells_per_step(self):
        return int(N.lib().e3d_cells_per_step(self._h))

    def _alloc_signals(self, pos7):
        return [np.zeros((len(pos7[COMP_GRID[k]]), self.nts), dtype=np.float32) for k in range(9)]

    def nl_forward(self, model9, src_pos7, rec_pos7):
        model = [N.as_f32(m) for m in model9]
        data = self._alloc_signals(rec_pos7)
        SP, SN, k1 = _geom(src_pos7)
        RP, RN, k2 = _geom(rec_pos7)
        N.call("e3d_nl_forward", self._h, N.ptr_array(model), N.ptr_array(data), SP, SN, RP, RN)
        return data

    def batch_tables(self, models, src_pos7s, rec_pos7):
        """Device tables of a batched forward: models[s] = nine regular source blocks (n_k, nts) of
        shot s on its tables src_pos7s[s]; the receivers rec_pos7 are shared.  Shot s owns cells
        [s n, (s+1) n) of each stacked field, so its positions carry the offset s n; component k's
        entries are the shots' tables in shot order.  Returns a BatchTables on this device."""
        import torch
        S = len(models)
        n = self.nz * self.nx * self.ny
        dev = torch.device("cuda", self.device)
        rtab = [np.asarray(rec_pos7[g], dtype=np.int64) for g in range(7)]
        src_pos, src_off, rec_pos, rec_off, sig = [], [0], [], [0], []
        for k in range(9):
            for s in range(S):
                tab = np.asarray(src_pos7s[s][COMP_GRID[k]], dtype=np.int64)
                src_pos.append(tab + s * n)
                blk = np.asarray(models[s][k], dtype=np.float32).reshape(len(tab), -1)
                # a shorter record is the same shot propagated to the longest one and cut
                sig.append(np.pad(blk, ((0, 0), (0, self.nts - blk.shape[1]))) if blk.shape[1] < self.nts else blk)
            src_off.append(src_off[-1] + sum(len(src_pos7s[s][COMP_GRID[k]]) for s in range(S)))
            # the reference's sxz receivers read the first n_xz entries of the z-grid table (quirk Q2)
            rk = rtab[3][:len(rtab[4])] if (self.q2compat and k == 6) else rtab[COMP_GRID[k]]
            for s in range(S):
                rec_pos.append(rk + s * n)
            rec_off.append(rec_off[-1] + S * len(rk))
        lengths = []
        for s in range(S):
            ks = [k for k in range(9) if len(src_pos7s[s][COMP_GRID[k]])]
            lengths.append(int(np.asarray(models[s][ks[0]]).reshape(len(src_pos7s[s][COMP_GRID[ks[0]]]), -1).shape[1])
                           if ks else self.nts)
            if lengths[-1] > self.nts:
                raise ValueError("a shot's record is longer than the propagator's nts")
        return BatchTables(S, torch.from_numpy(np.concatenate(src_pos)).to(dev), src_off,
                           torch.from_numpy(np.concatenate(rec_pos)).to(dev), rec_off,
                           torch.from_numpy(np.ascontiguousarray(np.concatenate(sig, axis=0).T)).to(dev),
                           torch.empty((self.nts, rec_off[-1]), dtype=torch.float32, device=dev), lengths)

    def nl_forward_batch_device(self, bt):
        """Launch the batched forward of BatchTables bt on the context's stream (asynchronous); the
        traces land in bt.rec_sig (nts, total receivers), time-major."""
        N.call("e3d_nl_forward_batch_device", self._h, bt.shots, bt.src_pos.data_ptr(),
               (ctypes.c_int * 10)(*bt.src_off), bt.rec_pos.data_ptr(), (ctypes.c_int * 10)(*bt.rec_off),
               bt.src_sig.data_ptr(), bt.rec_sig.data_ptr())

    def nl_forward_batch(self, models, src_pos7s, rec_pos7):
        """Batched nonlinear forward of several shots in one medium: one list of nine receiver
        blocks per shot, as nl_forward returns for each shot alone.  Shots may have different
        record lengths (the widths of their source blocks, at most nts): a shorter shot is
        propagated to nts with zero sources and its traces cut to its own length."""
        bt = self.batch_tables(models, src_pos7s, rec_pos7)
        self.nl_forward_batch_device(bt)
        N.call("e3d_synchronize", self._h)
        return bt.split(bt.rec_sig.cpu().numpy().T)

    def nl_forward_shots(self, models, src_pos7s, rec_pos7, free_bytes=None, margin=0.9):
        """Forward modelling of any number of shots: the shots are admitted into batched launches
        (nl_forward_batch) by the device memory free now (or `free_bytes`), as forward_batch_plan
        deals them.  Returns one list of nine receiver blocks per shot, in shot order."""
        import torch
        if free_bytes is None:
            free_bytes, _ = torch.cuda.mem_get_info(torch.device("cuda", self.device))
        src_points = max(sum(len(sp[COMP_GRID[k]]) for k in range(9)) for sp in src_pos7s) if src_pos7s else 0
        rec_points = sum(len(rec_pos7[COMP_GRID[k]]) for k in range(9))
        plan = forward_batch_plan(len(models), self.nz * self.nx * self.ny, self.nts, src_points, rec_points,
                                  free_bytes, margin)
        out = []
        for batch in plan:
            out.extend(self.nl_forward_batch([models[i] for i in batch], [src_pos7s[i] for i in batch], rec_pos7))
        return out

    def nl_adjoint(self, data9, src_pos7, rec_pos7):
        data = [N.as_f32(d) for d in data9]
        model = self._alloc_signals(src_pos7)
        SP, SN, k1 = _geom(src_pos7)
        RP, RN, k2 = _geom(rec_pos7)
        N.call("e3d_nl_adjoint", self._h, N.ptr_array(model), N.ptr_array(data), SP, SN, RP, RN)
        return model

    def born_forward(self, src9, pert8, src_pos7, rec_pos7):
        src = [N.as_f32(s) for s in src9]
        pert = [N.as_f32(p) for p in pert8]
        data = self._alloc_signals(rec_pos7)
        SP, SN, k1 = _geom(src_pos7)
        RP, RN, k2 = _geom(rec_pos7)
        N.call("e3d_born_forward", self._h, N.ptr_array(src), N.ptr_array(data), SP, SN, RP, RN, N.ptr_array(pert))
        return data

    def born_adjoint(self, src9, data9, src_pos7, rec_pos7, pert8_init=None):
        src = [N.as_f32(s) for s in src9]
        data = [N.as_f32(d) for d in data9]
        pert = [np.zeros(self.shape, dtype=np.float32) if pert8_init is None else np.array(pert8_init[k],
                                                                                             dtype=np.float32)
                for k in range(8)]
        SP, SN, k1 = _geom(src_pos7)
        RP, RN, k2 = _geom(rec_pos7)
        N.call("e3d_born_adjoint", self._h, N.ptr_array(src), N.ptr_array(data), SP, SN, RP, RN, N.ptr_array(pert))
        return pert

    def kernel_timing(self, every):
        """Sample every n-th launch of each timed kind with CUDA events (0 = off)."""
        N.call("e3d_kernel_timing", self._h, int(every))

    def kernel_timing_read(self, mode):
        """(mean ms, count) of the sampled launches of one kind since the last read: stepper modes 0..2,
        the same with a fused decimation or secondary source 3..5, block imaging 6, velocity decimation 7."""
        avg = ctypes.c_double(0)
        cnt = ctypes.c_longlong(0)
        N.call("e3d_kernel_timing_read", self._h, int(mode), ctypes.byref(avg), ctypes.byref(cnt))
        return avg.value, cnt.value

    @property
    def launch_count(self):
        return int(N.lib().e3d_launch_count(self._h))

    def step_only(self, mode, n_steps):
        N.call("e3d_step_only", self._h, int(mode), int(n_steps))

    # ---- device API (torch tensors) -------------------------------------------------
    def nl_propagate_device(self, adjoint, src_pos, src_off, rec_pos, rec_off, src_sig, rec_sig):
        so = (ctypes.c_int * 10)(*[int(v) for v in src_off])
        ro = (ctypes.c_int * 10)(*[int(v) for v in rec_off])
        N.call("e3d_nl_propagate_device", self._h, int(adjoint), src_pos.data_ptr(), so, rec_pos.data_ptr(), ro,
               src_sig.data_ptr(), rec_sig.data_ptr())

    @staticmethod
    def _trace_map(tmap):
        """ctypes reference to an E3DTraceMap built from a TraceTables-like object (or None)."""
        if tmap is None:
            return None
        m = N.E3DTraceMap(int(tmap.n_irreg), int(tmap.n_taps), tmap.slot.data_ptr(), tmap.weight.data_ptr(),
                          tmap.row_ptr.data_ptr(), tmap.idx.data_ptr(), tmap.w.data_ptr())
        return ctypes.byref(m), m

    def fwi_forward_device(self, src_pos, src_off, rec_pos, rec_off, src_sig, rec_sig, tmap=None):
        """Checkpointed nonlinear forward.  rec_sig: regular time-major (nts, rec_off[9]) without a
        trace map, irregular time-major (nts, 9*n_irreg) with one."""
        so = (ctypes.c_int * 10)(*[int(v) for v in src_off])
        ro = (ctypes.c_int * 10)(*[int(v) for v in rec_off])
        ref = self._trace_map(tmap)
        N.call("e3d_fwi_forward_device", self._h, src_pos.data_ptr(), so, rec_pos.data_ptr(), ro,
               src_sig.data_ptr(), rec_sig.data_ptr(), ref[0] if ref else None)

    def fwi_gradient_device(self, src_pos, src_off, rec_pos, rec_off, src_sig, residual, grad8, tmap=None,
                            src_adj=None):
        """Born-adjoint gradient planes into grad8; optionally the exact adjoint with respect to the
        scaled source signals into src_adj (time-major (nts, src_off[9]))."""
        so = (ctypes.c_int * 10)(*[int(v) for v in src_off])
        ro = (ctypes.c_int * 10)(*[int(v) for v in rec_off])
        ref = self._trace_map(tmap)
        N.call("e3d_fwi_gradient_device", self._h, src_pos.data_ptr(), so, rec_pos.data_ptr(), ro,
               src_sig.data_ptr(), residual.data_ptr(), N.ptr_array([grad8[k] for k in range(8)]),
               ref[0] if ref else None, src_adj.data_ptr() if src_adj is not None else None)

    def set_velocity_storage(self, kind="auto"):
        """Source velocity slots of the checkpoint plan: "auto", "fp32" or "fp16"."""
        N.call("e3d_set_velocity_storage", self._h, {"auto": -1, "fp32": 0, "fp16": 1}[kind])

    @property
    def velocity_storage(self):
        return ("fp32", "fp16")[int(N.lib().e3d_velocity_storage(self._h))]

    def set_decimation_ring(self, on=True):
        """Gradient passes: decimate fine levels from a ring once per coarse block (True, default) or
        through accumulators at every fine step (False)."""
        N.call("e3d_set_decimation_ring", self._h, 1 if on else 0)

    def set_premultiplied_adjoint(self, on=True):
        """Exact adjoint of the gradient passes on the premultiplied-only state where the medium
        allows it (True, default), or always on the dual raw + premultiplied state (False)."""
        N.call("e3d_set_premultiplied_adjoint", self._h, 1 if on else 0)

    def set_imaging_chunks(self, chunks=0):
        """y chunks of the block imaging launch (0 = automatic)."""
        N.call("e3d_set_imaging_chunks", self._h, int(chunks))

    IMAGING = {"auto": 0, "cells": 1, "tma": 2, "tma-levels": 3, "tma-levels-4": 4}

    def set_imaging_variant(self, variant="auto"):
        """Block imaging kernel: auto, cells (one thread per cell, global loads), tma (velocity tiles
        staged by TMA) or tma-levels (velocity tiles, adjoint levels and medium staged by TMA)."""
        N.call("e3d_set_imaging_variant", self._h, self.IMAGING[variant])
