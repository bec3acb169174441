"""FWI gradient serving over grids of uneven size.

A `GradientServer` takes gradient requests -- (finite-difference parameters of a grid, an elastic
model, a shot) -- and answers each with the misfit and the (rho, lambda, mu) gradient.  Requests
may use different grids and record lengths.  Per GPU, the server keeps one `FwiProblem` per
(grid, record length):
  * its stepper variant is autotuned once per grid shape (`autotune.autotune_gradient`) and reused;
  * checkpoints are stored as FP16 with per-slice scales unless told otherwise;
  * before a problem for a new grid is opened, problems that are not needed are closed, least
    recently used first, until the device's free memory admits the new one (its working fields
    plus the smallest checkpoint plan, estimated from the cell count and record length).
Requests are dealt to GPUs by grid, so that a GPU keeps serving the grid it holds; each GPU's
requests run in submission order on one host thread.
"""
from __future__ import annotations

import threading
from collections import OrderedDict
from dataclasses import dataclass, field

import numpy as np
import torch

from . import fwi as F
from . import hostprep as H


@dataclass
class GradientRequest:
    fd: H.FdParam                 # grid, time axis and medium QC of the request
    model: np.ndarray             # (3, ny, nx, nz) rho, lambda, mu
    src7: list                    # spaceInterpGpu_3D x7 of the shot's sources
    rec7: list                    # spaceInterpGpu_3D x7 of the receivers
    wavelet9: list                # 9 (nSrc, nts) irregular source signals
    d_obs: np.ndarray             # (9, nRec, nts) observed data
    result: tuple = field(default=None, repr=False)   # (misfit, (g_rho, g_lambda, g_mu)) once served


def _key(fd):
    """Everything of a request's fdParamElastic_3D that its FwiProblem is built from: the grid, the
    time axes, the sponge (width and taper constant) and the free-surface flag (a free-surface
    request must reach FwiProblem, which refuses it, rather than reuse a problem without one)."""
    return (fd.nz, fd.nx, fd.ny, fd.nts, fd.sub, fd.minPad, float(fd.dz), float(fd.dx), float(fd.dy),
            float(fd.dts), float(getattr(fd, "alphaCos", 0.99)), int(getattr(fd, "freeSurface", 0)))


def _estimate_bytes(fd):
    """Working fields of a gradient (about 100 fields of n cells) plus a 16-bit checkpoint plan near
    the square-root schedule: an admission estimate, not an allocation."""
    n = fd.nz * fd.nx * fd.ny
    blocks = max(fd.nts - 1, 1)
    ck, vs = 18 * n * 2, 3 * n * 4
    best = min(((blocks + l - 1) // l - 1) * ck + (l + 3) * vs for l in range(1, blocks + 1))
    return 100 * n * 4 + best


class GradientServer:
    def __init__(self, devices=(0,), ckpt="fp16", autotune=True, reserve_bytes=2 << 30):
        self.devices = list(devices)
        self.ckpt = ckpt
        self.autotune = autotune
        self.reserve = reserve_bytes
        self.variants = {}                      # grid shape -> tuned variant
        self.open = {d: OrderedDict() for d in self.devices}   # device -> key -> FwiProblem
        self._lock = threading.Lock()

    def _problem(self, dev, fd):
        key = _key(fd)
        probs = self.open[dev]
        if key in probs:
            probs.move_to_end(key)
            return probs[key]
        need = _estimate_bytes(fd) + self.reserve
        torch.cuda.synchronize(dev)
        while probs and torch.cuda.mem_get_info(dev)[0] < need:
            _, old = probs.popitem(last=False)   # least recently used
            old.prop.close()
            del old
            torch.cuda.empty_cache()
        shape = (fd.nz, fd.nx, fd.ny)
        with self._lock:
            tuned = self.variants.get(shape)
        variant = tuned if tuned is not None else ("auto" if self.autotune else (8, 3, "split-pair"))
        prob = F.FwiProblem(fd, device=f"cuda:{dev}", ckpt=self.ckpt, variant=variant)
        probs[key] = prob
        return prob

    def _serve_one(self, dev, req: GradientRequest):
        torch.cuda.set_device(dev)
        prob = self._problem(dev, req.fd)
        prob.shots = [F.make_shot(req.src7, req.rec7, req.wavelet9, req.d_obs, f"cuda:{dev}")]
        m = [torch.tensor(np.asarray(req.model[k], np.float32), device=f"cuda:{dev}", requires_grad=True)
             for k in range(3)]
        loss = F.ElasticFwiMisfit.apply(m[0], m[1], m[2], prob)
        loss.backward()
        if prob.autotune and prob.tuned is not None:
            with self._lock:
                self.variants.setdefault((req.fd.nz, req.fd.nx, req.fd.ny), prob.tuned[0])
        req.result = (float(loss.item()), tuple(x.grad.cpu().numpy() for x in m))
        prob.shots = []
        return req.result

    def serve(self, requests):
        """Serve the requests; returns their (misfit, gradient) results in submission order."""
        requests = list(requests)
        # deal grids to GPUs (a GPU keeps the grids it was given), keeping submission order per GPU
        grids = []
        for r in requests:
            k = _key(r.fd)
            if k not in grids:
                grids.append(k)
        owner = {k: self.devices[i % len(self.devices)] for i, k in enumerate(grids)}
        queues = {d: [r for r in requests if owner[_key(r.fd)] == d] for d in self.devices}
        errors = []

        def worker(dev):
            try:
                for r in queues[dev]:
                    self._serve_one(dev, r)
            except Exception as e:  # reported after the other GPUs finish
                errors.append(e)

        threads = [threading.Thread(target=worker, args=(d,)) for d in self.devices if queues[d]]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]
        return [r.result for r in requests]

    def close(self):
        for probs in self.open.values():
            for p in probs.values():
                p.prop.close()
            probs.clear()
