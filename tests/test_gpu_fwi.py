"""GPU: the autograd FWI misfit/gradient against the FP64 oracle (
gradient relative error <= 1e-3 against FP64)."""
import numpy as np
import pytest
import torch

from fwi_case import OracleFwi, explosive, survey
from elasticisolib_3d_b200 import fwi as F
from elasticisolib_3d_b200 import hostprep as H

pytestmark = pytest.mark.gpu


def _problem(sv, ckpt="fp32", segment=0, variant=(8, 2, "tma")):
    fd = H.FdParam(sv.elastic, sv.axes, sv.par)
    prob = F.FwiProblem(fd, ckpt=ckpt, segment=segment, variant=variant)
    ax7 = H.grid_axes(*(a.n for a in sv.axes), *(a.o for a in sv.axes), *(a.d for a in sv.axes))
    src = H.build_devices(*sv.src_xyz[0], ax7, fd.nts, sv.par)
    rec = H.build_devices(*sv.rec_xyz, ax7, fd.nts, sv.par)
    return prob, src, rec


@pytest.mark.parametrize("ckpt,segment,variant", [("fp32", 0, (8, 2, "tma")), ("fp32", 3, (8, 2, "plain")),
                                                   ("fp16", 4, (8, 2, "tma"))])
def test_fwi_gradient_matches_fp64_oracle(ckpt, segment, variant):
    sv, true = survey()
    orc = OracleFwi(sv)
    d_obs, _ = orc.data(true)
    loss_ref, g_ref = orc.misfit_and_gradient(sv.elastic, d_obs)
    prob, src, rec = _problem(sv, ckpt, segment, variant)
    prob.shots.append(F.make_shot(src, rec, explosive(sv.par.getInt("nts"), sv.wavelet), d_obs.astype(np.float32),
                                  "cuda"))
    m = [torch.tensor(sv.elastic[k], device="cuda", requires_grad=True) for k in range(3)]
    loss = F.ElasticFwiMisfit.apply(m[0], m[1], m[2], prob)
    loss.backward()
    g = np.stack([x.grad.double().cpu().numpy() for x in m])
    assert abs(loss.item() - loss_ref) / loss_ref < 1e-4
    for k in range(3):
        err = np.linalg.norm(g[k] - g_ref[k]) / np.linalg.norm(g_ref[k])
        assert err < 1e-3, (k, err)
