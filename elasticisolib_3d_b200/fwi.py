"""FWI misfit and gradient over (rho, lambda, mu) as a torch.autograd.Function.

Per shot the device runs, through the engine's C ABI:
  1. the nonlinear forward of the scaled sources (propElasticFwdGpu_3D
     semantics), saving on-device wavefield checkpoints;
  2. the L2 residual at the irregular receivers (spaceInterpGpu_3D forward);
  3. the Born adjoint of the residual (BornElasticAdjGpu_3D semantics: exact
     transpose stepper, decimated adjoint field, imaging condition), with the
     source-side velocity of the last checkpoint segment kept from the
     forward pass and that of the earlier segments recomputed from the
     checkpoints, instead of the reference's pinned-host snapshot storage;
  4. the post-processing of BornElasticShotsGpu_3D::adjoint
     (BornElasticShotsGpu_3D.cpp:528-605): scaling by the density planes and
     2*dtw, unstaggering, giving (d rho, d lambda, d mu).
The gradient is therefore the reference's Born-adjoint gradient (the one its
EFWI driver uses, efwiMain_3D.py:195-196) of 0.5*||d_pred - d_obs||^2.

Medium preparation (fdParamElastic_3D.cpp:130-193), source scaling
(nonlinearPropElasticGpu_3D.cpp:200-277) and receiver interpolation run as
torch operations on the device.  Fields are (ny, nx, nz) tensors.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import hostprep as H
from .engine import COMP_GRID, Propagator

# ----------------------------------------------------------------------------
# staggering (stagger_3D.cpp) on (ny, nx, nz) tensors; axis 'z' -> dim 2, 'x' -> 1, 'y' -> 0
# ----------------------------------------------------------------------------
_DIM = {"z": 2, "x": 1, "y": 0}


def stagger_adjoint(d, axis):
    """m[i] = 0.5(d[i]+d[i-1]); m[0] = 0.5 d[0]; m[n-1] = d[n-1] + 0.5 d[n-2]."""
    d = d.movedim(_DIM[axis], -1)
    m = torch.empty_like(d)
    m[..., 1:-1] = 0.5 * (d[..., 1:-1] + d[..., :-2])
    m[..., 0] = 0.5 * d[..., 0]
    m[..., -1] = d[..., -1] + 0.5 * d[..., -2]
    return m.movedim(-1, _DIM[axis]).contiguous()


def stagger_forward(m, axis):
    """d[i] = 0.5(m[i]+m[i+1]) (i < n-1); d[n-1] = m[n-1]."""
    m = m.movedim(_DIM[axis], -1)
    d = torch.empty_like(m)
    d[..., :-1] = 0.5 * (m[..., :-1] + m[..., 1:])
    d[..., -1] = m[..., -1]
    return d.movedim(-1, _DIM[axis]).contiguous()


def medium_planes(rho, lam, mu, dtw):
    """Eight scaled planes (rhoxDtw ... muyzDtw) from float32 (rho, lambda, mu) tensors."""
    two = 2.0 * float(dtw)
    rhox = stagger_adjoint(rho, "x")
    rhoy = stagger_adjoint(rho, "y")
    rhoz = stagger_adjoint(rho, "z")
    t1 = stagger_adjoint(mu, "x")
    muxz = stagger_adjoint(t1, "z")
    muxy = stagger_adjoint(t1, "y")
    muyz = stagger_adjoint(stagger_adjoint(mu, "y"), "z")
    out = torch.empty((8,) + tuple(rho.shape), dtype=torch.float32, device=rho.device)
    out[0] = (two / rhox.double()).float()
    out[1] = (two / rhoy.double()).float()
    out[2] = (two / rhoz.double()).float()
    out[3] = (two * (lam.double() + 2.0 * mu.double())).float()
    out[4] = (two * lam.double()).float()
    out[5] = (two * muxz.double()).float()
    out[6] = (two * muxy.double()).float()
    out[7] = (two * muyz.double()).float()
    return out


def planes_to_model(grad8, planes, dtw):
    """Adjoint of the Born model preparation: 8 staggered planes -> (d rho, d lambda, d mu)
    (BornElasticShotsGpu_3D.cpp:542-605)."""
    two = 2.0 * float(dtw)
    g = [grad8[k] * planes[k] for k in range(3)] + [(grad8[k].double() * two).float() for k in range(3, 8)]
    drho = stagger_forward(g[0], "x") + stagger_forward(g[1], "y")
    drho = drho + stagger_forward(g[2], "z")
    t2 = stagger_forward(stagger_forward(g[5], "z"), "x")
    t2 = t2 + stagger_forward(stagger_forward(g[6], "y"), "x")
    t2 = t2 + stagger_forward(stagger_forward(g[7], "z"), "y")
    return drho, g[3].clone(), g[4] + t2


# ----------------------------------------------------------------------------
# acquisition on the device
# ----------------------------------------------------------------------------
@dataclass
class DeviceSet:
    """Nine-component concatenated regular-grid points of one device set."""
    pos: torch.Tensor        # (ntot,) int64
    off: list                # 10 offsets
    slot: list               # per grid: (nIrreg, nTaps) int64 into that grid's unique list
    weight: list             # per grid: (nIrreg, nTaps) float32 (8 trilinear, (2h)^3 sinc, doubled by a dipole)
    n_irreg: int

    @staticmethod
    def from_devices(devices7, device, q2_receivers=False):
        pos, off = [], [0]
        for k in range(9):
            g = COMP_GRID[k]
            if q2_receivers and k == 6:  # sxz receivers read the z-grid table (reference quirk Q2)
                u = devices7[3].getRegPosUnique()[:devices7[4].getNDeviceReg()]
            else:
                u = devices7[g].getRegPosUnique()
            pos.append(np.asarray(u, dtype=np.int64))
            off.append(off[-1] + len(u))
        return DeviceSet(pos=torch.from_numpy(np.concatenate(pos)).to(device), off=off,
                         slot=[torch.from_numpy(d.slot).to(device) for d in devices7],
                         weight=[torch.from_numpy(d.weight).to(device) for d in devices7],
                         n_irreg=devices7[0].getNDeviceIrreg())

    def comp(self, k):
        return slice(self.off[k], self.off[k + 1])

    def to_irregular(self, reg):
        """(nts, ntot) regular-grid traces -> (9, nIrreg, nts) (spaceInterpGpu_3D::forward)."""
        out = []
        for k in range(9):
            g = COMP_GRID[k]
            rk = reg[:, self.comp(k)]
            acc = torch.zeros((reg.shape[0], self.n_irreg), dtype=reg.dtype, device=reg.device)
            for f in range(self.slot[g].shape[1]):
                acc = acc + self.weight[g][:, f] * rk[:, self.slot[g][:, f]]
            out.append(acc.t())
        return torch.stack(out)

    def to_regular(self, irreg):
        """(9, nIrreg, nts) -> (nts, ntot) (spaceInterpGpu_3D::adjoint)."""
        nts = irreg.shape[2]
        reg = torch.zeros((nts, self.off[9]), dtype=irreg.dtype, device=irreg.device)
        for k in range(9):
            g = COMP_GRID[k]
            d = irreg[k].t()  # (nts, nIrreg)
            blk = torch.zeros((nts, self.off[k + 1] - self.off[k]), dtype=irreg.dtype, device=irreg.device)
            for f in range(self.slot[g].shape[1]):
                blk.index_add_(1, self.slot[g][:, f], d * self.weight[g][:, f])
            reg[:, self.comp(k)] = blk
        return reg


def scale_sources(sig_reg, src: DeviceSet, planes, dx, dy, dz):
    """Medium scaling of regular-grid source signals (nonlinearPropElasticGpu_3D.cpp:200-277).
    sig_reg: (nts, ntot) time-major; returns a new tensor."""
    flat = planes.reshape(8, -1)
    out = sig_reg.clone()
    for k, m in ((0, 0), (1, 1), (2, 2), (6, 5), (7, 6), (8, 7)):
        sl = src.comp(k)
        out[:, sl] = sig_reg[:, sl] * flat[m][src.pos[sl]]
    c = src.comp(3)
    pc = src.pos[c]
    l2m, lam = flat[3][pc], flat[4][pc]
    sxx, syy, szz = sig_reg[:, src.comp(3)], sig_reg[:, src.comp(4)], sig_reg[:, src.comp(5)]
    out[:, src.comp(3)] = sxx * l2m + (syy + szz) * lam
    out[:, src.comp(4)] = syy * l2m + (sxx + szz) * lam
    out[:, src.comp(5)] = szz * l2m + (sxx + syy) * lam
    area = np.float32(1.0 / float(np.float32(np.float32(dx) * np.float32(dy)) * np.float32(dz)))
    return out * float(area)


@dataclass
class TraceTables:
    """Device tables of the engine's trace map (e3d_trace_map): the nine components'
    irregular receivers as linear combinations of the regular receiver points.
    Receiver row r = k*n_irreg + i; irregular traces are time-major (nts, 9*n_irreg)."""
    n_irreg: int
    n_taps: int
    slot: torch.Tensor       # (9*n_irreg*n_taps,) int32, index into the concatenated regular list
    weight: torch.Tensor     # (9*n_irreg*n_taps,) float32
    row_ptr: torch.Tensor    # (n_reg+1,) int32, spread rows
    idx: torch.Tensor        # (nnz,) int32, receiver row of each spread entry
    w: torch.Tensor          # (nnz,) float32

    @staticmethod
    def from_set(rec: DeviceSet, device):
        """Gather rows follow spaceInterpGpu_3D::forward (device, then tap); each spread row lists
        its entries in the order spaceInterpGpu_3D::adjoint accumulates them (device, then tap),
        spaceInterpGpu_3D.cpp:140-175."""
        n_irreg = rec.n_irreg
        slots, wts = [], []
        for k in range(9):
            g = COMP_GRID[k]
            slots.append(rec.slot[g].cpu().numpy().astype(np.int64) + rec.off[k])
            wts.append(rec.weight[g].cpu().numpy().astype(np.float32))
        slot = np.concatenate(slots).reshape(-1) if n_irreg else np.zeros(0, np.int64)
        weight = np.concatenate(wts).reshape(-1) if n_irreg else np.zeros(0, np.float32)
        n_taps = slot.size // (9 * n_irreg) if n_irreg else 8
        n_reg = rec.off[9]
        assert slot.size == 0 or (slot.min() >= 0 and slot.max() < n_reg)
        rows = np.repeat(np.arange(9 * n_irreg, dtype=np.int64), n_taps)
        order = np.argsort(slot, kind="stable")
        row_ptr = np.zeros(n_reg + 1, dtype=np.int64)
        np.cumsum(np.bincount(slot, minlength=n_reg), out=row_ptr[1:])
        assert row_ptr[-1] < 2 ** 31

        def dev(a, dt):
            return torch.from_numpy(np.ascontiguousarray(a).astype(dt)).to(device)

        return TraceTables(n_irreg, n_taps, dev(slot, np.int32), dev(weight, np.float32), dev(row_ptr, np.int32),
                           dev(rows[order], np.int32), dev(weight[order], np.float32))


def time_major(d9):
    """(9, nIrreg, nts) irregular traces -> time-major (nts, 9*nIrreg)."""
    d9 = torch.as_tensor(d9)
    return d9.permute(2, 0, 1).reshape(d9.shape[2], -1).contiguous()


def component_major(dt, n_irreg):
    """Time-major (nts, 9*nIrreg) -> (9, nIrreg, nts)."""
    return dt.reshape(dt.shape[0], 9, n_irreg).permute(1, 2, 0).contiguous()


@dataclass
class Shot:
    src: DeviceSet
    rec: DeviceSet
    sig_reg: torch.Tensor      # (nts, ntot_src) unscaled regular-grid source signals
    d_obs: torch.Tensor        # (nts, 9*nRec) observed data at the irregular receivers, time-major
    tables: TraceTables = None


def make_shot(src_devices7, rec_devices7, model_irreg9, d_obs, device, q2compat=True):
    """Spread the irregular source signals to the regular grid (spaceInterpGpu_3D::adjoint) and
    move everything to the device.  model_irreg9: list of 9 (nIrregSrc, nts) arrays; d_obs:
    (9, nRec, nts) observed traces or None."""
    src = DeviceSet.from_devices(src_devices7, device)
    rec = DeviceSet.from_devices(rec_devices7, device, q2_receivers=q2compat)
    nts = model_irreg9[0].shape[1]
    blocks = []
    for k in range(9):
        g = COMP_GRID[k]
        blocks.append(src_devices7[g].adjoint(False, None, np.asarray(model_irreg9[k], dtype=np.float32)))
    sig = torch.from_numpy(np.ascontiguousarray(np.concatenate(blocks, axis=0).T)).to(device)
    assert sig.shape == (nts, src.off[9])
    if d_obs is not None:
        d_obs = time_major(torch.as_tensor(np.asarray(d_obs, dtype=np.float32)).to(device))
    return Shot(src, rec, sig, d_obs, TraceTables.from_set(rec, device))


def _half_sum_sq(x, rows_per_chunk=64):
    """0.5*sum(x^2) accumulated in float64 over chunks of time samples (bounded temporaries)."""
    tot = torch.zeros((), dtype=torch.float64, device=x.device)
    for i in range(0, x.shape[0], rows_per_chunk):
        c = x[i:i + rows_per_chunk]
        tot += torch.sum(c * c, dtype=torch.float64)
    return 0.5 * tot


class FwiProblem:
    """One propagation grid, its context and shots; shared by forward modelling and gradients."""

    def __init__(self, fd: H.FdParam, device="cuda", ckpt="auto", segment=0, variant=(8, 3, "split-pair"),
                 velocity="auto", q3compat=1, source_term=False, decimation_ring=True, premultiplied=True):
        """q3compat=1 keeps the reference's Born yz shear term (the xz derivative pair, quirk Q3);
        0 uses the yz pair, the linearisation of the propagator's own yz stress update.
        source_term=True adds the misfit's derivative through the medium scaling of the source
        signals (the exact adjoint sampled at the source points, chained through medium_planes and
        scale_sources by autograd), which the reference's Born-adjoint gradient leaves out.
        decimation_ring=True decimates the fine levels of each coarse block from a ring of levels in
        one launch per block; False fuses two coarse accumulators into every fine step.
        premultiplied=True runs the ring passes' exact adjoint on the premultiplied-only state where
        the medium allows it; False keeps the dual raw + premultiplied state."""
        if getattr(fd, "freeSurface", 0):
            raise ValueError("FWI gradients with a free surface are not supported (no exact adjoint of it)")
        self.fd = fd
        self.device = torch.device(device)
        self.prop = Propagator(fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx),
                               float(fd.dy), float(fd.dts), float(fd.alphaCos),
                               device=self.device.index or 0, q3compat=q3compat)
        # variant "auto": timed on the grid by the autotuner at the first set_model
        self.autotune = variant == "auto"
        self.tuned = None
        if not self.autotune:
            self.prop.set_stepper_variant(*variant)
        self.prop.set_checkpoint_policy(ckpt, segment)
        self.prop.set_velocity_storage(velocity)
        self.prop.set_decimation_ring(decimation_ring)
        self.prop.set_premultiplied_adjoint(premultiplied)
        self.ckpt, self.segment = ckpt, segment
        self.source_term = source_term
        self.auto_budget = segment == 0
        self.shots = []
        # multi-GPU: every rank holds all shots, takes its share and all-reduces the result
        self.distributed = False
        self.group = None
        # optional masks (efwiMain_3D.py:158-233): data mask on the residual, time-major
        # (nts, 9*nRec) or broadcastable to it; gradient mask (3, ny, nx, nz) on (rho, lambda, mu)
        self.data_mask = None
        self.grad_mask = None

    def distribute(self, group=None, dealing="static", store=None, tag="fwi", broadcast=True):
        """Share the shots among the ranks of `group` (torch.distributed, one rank per GPU).
        dealing "static": rank r takes shots r, r+world, ...; "dynamic": every rank takes the next
        undealt shot from a counter in `store` (a torch.distributed Store; by default a client of
        the rendezvous store at MASTER_ADDR:MASTER_PORT), so that ranks with cheaper shots take
        more of them.  `tag` names the counters; problems evaluated in the same job need distinct
        tags.  broadcast: every evaluation first broadcasts (rho, lambda, mu) from the group's
        first rank, so that all ranks propagate in the same medium even if their copies drifted."""
        if dealing not in ("static", "dynamic"):
            raise ValueError(f"unknown shot dealing {dealing!r}")
        self.distributed = True
        self.group = group
        self.dealing = dealing
        self.store = store
        self.tag = tag
        self.evaluations = 0
        self.broadcast = broadcast
        return self

    def _bind_stream(self):
        self.prop.set_stream(torch.cuda.current_stream(self.device))

    def set_model(self, rho, lam, mu):
        planes = medium_planes(rho, lam, mu, self.fd.dtw)
        self._bind_stream()
        self.prop.set_medium(planes)
        if self.autotune and self.tuned is None:
            from .autotune import autotune_gradient
            self.tuned = autotune_gradient(self.prop)
            self._bind_stream()
        return planes

    def forward_data(self, shot: Shot, planes):
        """Checkpointed nonlinear forward of one shot: predicted irregular traces, time-major
        (nts, 9*nRec), and the scaled regular-grid source signals."""
        fd = self.fd
        sig = scale_sources(shot.sig_reg, shot.src, planes, fd.dx, fd.dy, fd.dz).contiguous()
        d_pred = torch.empty((fd.nts, 9 * shot.rec.n_irreg), dtype=torch.float32, device=self.device)
        self._bind_stream()
        if self.auto_budget:
            # leave room for what the gradient step allocates after the forward: gradient planes
            # and the model post-processing temporaries
            n = planes[0].numel()
            torch.cuda.empty_cache()
            self.prop.set_checkpoint_policy(self.ckpt, self.segment, -float(24 * n * 4 + (2 << 30)))
        self.prop.fwi_forward_device(shot.src.pos, shot.src.off, shot.rec.pos, shot.rec.off, sig, d_pred,
                                     shot.tables)
        return d_pred, sig

    def predict(self, shot: Shot, planes):
        """Predicted data (9, nRec, nts) of one shot."""
        d_pred, _ = self.forward_data(shot, planes)
        return component_major(d_pred, shot.rec.n_irreg)

    def shot_misfit_and_gradient(self, shot: Shot, planes, src_adj=None):
        """0.5*||d_pred - d_obs||^2 of one shot and its Born-adjoint gradient planes (8, ny, nx, nz);
        with src_adj (nts, src.off[9]) the exact adjoint at the source points is written there."""
        res, sig = self.forward_data(shot, planes)
        res.sub_(shot.d_obs)  # the residual overwrites the prediction
        if self.data_mask is not None:
            # objective 0.5*||M (d_pred - d_obs)||^2: residual M r, adjoint source M (M r)
            res.mul_(self.data_mask)
        loss = _half_sum_sq(res)
        if self.data_mask is not None:
            res.mul_(self.data_mask)
        grad8 = torch.zeros_like(planes)
        self._bind_stream()
        self.prop.fwi_gradient_device(shot.src.pos, shot.src.off, shot.rec.pos, shot.rec.off, sig, res, grad8,
                                      shot.tables, src_adj)
        return loss, grad8


def shard_shots(n_shots, rank, world):
    """Shots of one rank: rank, rank+world, ...  Shots are independent propagations, so they
    shard with no exchange (the reference deals them to GPUs from one OpenMP loop,
    nonlinearPropElasticShotsGpu_3D.cpp:178-204)."""
    return list(range(rank, n_shots, world))


def rendezvous_store(timeout_s=300.0):
    """A client of the store torch.distributed's env:// initialisation (and torchrun) serve at
    MASTER_ADDR:MASTER_PORT."""
    import datetime
    import os
    return torch.distributed.TCPStore(os.environ["MASTER_ADDR"], int(os.environ["MASTER_PORT"]), is_master=False,
                                      timeout=datetime.timedelta(seconds=timeout_s))


class ShotQueue:
    """Dynamic dealing of n_shots shots over the ranks that iterate queues with the same key:
    each step takes the next undealt shot from an atomic counter in a torch.distributed Store,
    as the reference deals shots to GPUs from an OpenMP loop with a dynamic schedule
    (nonlinearPropElasticShotsGpu_3D.cpp:178-204).  Every shot is dealt exactly once."""

    def __init__(self, n_shots, key, store):
        self.n_shots = int(n_shots)
        self.key = key
        self.store = store

    def __iter__(self):
        while True:
            i = int(self.store.add(self.key, 1)) - 1
            if i >= self.n_shots:
                return
            yield i


def broadcast_model(tensors, group=None):
    """Overwrite (rho, lambda, mu) on every rank of `group` with the first rank's copy (one
    broadcast of a flat buffer); a no-op without an initialised process group."""
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return tensors
    flat = torch.cat([t.detach().reshape(-1).float() for t in tensors])
    src = torch.distributed.get_global_rank(group, 0) if group is not None else 0
    torch.distributed.broadcast(flat, src=src, group=group)
    out, off = [], 0
    for t in tensors:
        out.append(flat[off:off + t.numel()].view_as(t).to(t.dtype))
        off += t.numel()
    return out


def reduce_misfit(total, grads, group=None):
    """Sum the misfit and the (rho, lambda, mu) gradient over the ranks of `group`: one
    all-reduce of the flat gradient (NCCL over NVLink between GPUs; the reference sums shot
    gradients on the host, BornElasticShotsGpu_3D.cpp:528-540) and one of the misfit in its own
    precision (FP64), so that the distributed misfit keeps the digits the single-rank one has."""
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return total, grads
    flat = torch.cat([g.reshape(-1) for g in grads])
    tot = total.reshape(1).clone()
    torch.distributed.all_reduce(flat, group=group)
    torch.distributed.all_reduce(tot, group=group)
    out, off = [], 0
    for g in grads:
        out.append(flat[off:off + g.numel()].view_as(g))
        off += g.numel()
    return tot[0], out


def _source_scaling_gradient(rho, lam, mu, problem, src_terms):
    """d/d(rho, lambda, mu) of sum_shots <src_adj, scale_sources(sig, medium_planes(rho, lambda, mu))>:
    the misfit's dependence through the medium scaling of the source signals."""
    fd = problem.fd
    with torch.enable_grad():
        m = [x.detach().float().requires_grad_(True) for x in (rho, lam, mu)]
        planes = medium_planes(m[0], m[1], m[2], fd.dtw)
        acc = torch.zeros((), dtype=torch.float64, device=rho.device)
        for shot, adj in src_terms:
            s = scale_sources(shot.sig_reg, shot.src, planes, fd.dx, fd.dy, fd.dz)
            acc = acc + torch.sum(s.double() * adj.double())
        return torch.autograd.grad(acc, m)


class ElasticFwiMisfit(torch.autograd.Function):
    """L(rho, lambda, mu) = sum over shots of 0.5*||d_pred - d_obs||^2.

    The forward pass computes the misfit and, shot by shot, the Born-adjoint
    gradient (so at most one shot's checkpoints are alive at a time); the
    backward pass scales the stored gradient by the incoming gradient.
    """

    @staticmethod
    def forward(ctx, rho, lam, mu, problem: FwiProblem, shot_ids=None):
        model = [rho.float().contiguous(), lam.float().contiguous(), mu.float().contiguous()]
        if problem.distributed and getattr(problem, "broadcast", False):
            model = [m.contiguous() for m in broadcast_model(model, problem.group)]
        planes = problem.set_model(*model)
        if shot_ids is not None:
            ids = shot_ids
        elif problem.distributed and getattr(problem, "dealing", "static") == "dynamic":
            if problem.store is None:
                problem.store = rendezvous_store()
            ids = ShotQueue(len(problem.shots), f"e3d/shots/{problem.tag}/{problem.evaluations}", problem.store)
            problem.evaluations += 1
        elif problem.distributed:
            ids = shard_shots(len(problem.shots), torch.distributed.get_rank(problem.group),
                              torch.distributed.get_world_size(problem.group))
        else:
            ids = range(len(problem.shots))
        total = torch.zeros((), dtype=torch.float64, device=rho.device)
        g8 = torch.zeros_like(planes)
        src_terms = []
        for i in ids:
            shot = problem.shots[i]
            src_adj = None
            if problem.source_term:
                src_adj = torch.empty((problem.fd.nts, shot.src.off[9]), dtype=torch.float32, device=rho.device)
            loss, grad8 = problem.shot_misfit_and_gradient(shot, planes, src_adj)
            total = total + loss
            g8 += grad8
            if src_adj is not None:
                src_terms.append((shot, src_adj))
        g = planes_to_model(g8, planes, problem.fd.dtw)
        if src_terms:
            g = tuple(a + b for a, b in zip(g, _source_scaling_gradient(*model, problem, src_terms)))
        if problem.grad_mask is not None:
            g = tuple(gk * problem.grad_mask[k] for k, gk in enumerate(g))
        if problem.distributed:
            total, g = reduce_misfit(total, list(g), problem.group)
        ctx.save_for_backward(*g)
        return total

    @staticmethod
    def backward(ctx, grad_out):
        grho, glam, gmu = ctx.saved_tensors
        s = grad_out.to(grho.dtype)
        return grho * s, glam * s, gmu * s, None, None
