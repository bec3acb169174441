"""GPU: the gradient server over three grids of different size and record length, against the
same gradients computed one problem at a time."""
import numpy as np
import pytest
import torch

from fwi_case import explosive
from elasticisolib_3d_b200 import fwi as F
from elasticisolib_3d_b200 import hostprep as H
from elasticisolib_3d_b200 import synthetic as S
from elasticisolib_3d_b200.serving import GradientRequest, GradientServer

pytestmark = pytest.mark.gpu


def _request(seed, nzi, nxi, nyi, nts):
    sv = S.small_survey(seed=seed, nzi=nzi, nxi=nxi, nyi=nyi, pad=4, nts=nts, nrec=8)
    rng = np.random.default_rng(seed + 7)
    true = sv.elastic.astype(np.float64)
    true[:, 4:-4, 4:-4, 4:-4] *= 1 + 0.02 * rng.standard_normal(true[:, 4:-4, 4:-4, 4:-4].shape)
    fd = H.FdParam(sv.elastic, sv.axes, sv.par)
    ax7 = H.grid_axes(*(a.n for a in sv.axes), *(a.o for a in sv.axes), *(a.d for a in sv.axes))
    src = H.build_devices(*sv.src_xyz[0], ax7, fd.nts, sv.par)
    rec = H.build_devices(*sv.rec_xyz, ax7, fd.nts, sv.par)
    # observed data from the perturbed model, modelled with the library itself
    prob = F.FwiProblem(H.FdParam(true.astype(np.float32), sv.axes, sv.par), ckpt="fp32")
    shot = F.make_shot(src, rec, explosive(fd.nts, sv.wavelet), None, "cuda")
    planes = prob.set_model(*[torch.tensor(true[k], dtype=torch.float32, device="cuda") for k in range(3)])
    d_obs = prob.predict(shot, planes).cpu().numpy()
    prob.prop.close()
    return GradientRequest(fd, sv.elastic, src, rec, explosive(fd.nts, sv.wavelet), d_obs)


def _standalone(req):
    prob = F.FwiProblem(req.fd, ckpt="fp16")
    prob.shots.append(F.make_shot(req.src7, req.rec7, req.wavelet9, req.d_obs, "cuda"))
    m = [torch.tensor(req.model[k], device="cuda", requires_grad=True) for k in range(3)]
    loss = F.ElasticFwiMisfit.apply(m[0], m[1], m[2], prob)
    loss.backward()
    out = (float(loss.item()), tuple(x.grad.cpu().numpy() for x in m))
    prob.prop.close()
    return out


def test_server_over_uneven_grids_matches_standalone_gradients():
    reqs = [_request(1, 16, 16, 16, 24), _request(2, 16, 32, 16, 32), _request(3, 16, 16, 16, 24),
            _request(4, 32, 16, 24, 20), _request(5, 16, 32, 16, 32)]
    server = GradientServer(devices=(0,), ckpt="fp16", autotune=True)
    results = server.serve(reqs)
    assert len(server.variants) == 3  # tuned once per grid shape
    for req, (loss, grads) in zip(reqs, results):
        ref_loss, ref_grads = _standalone(req)
        assert abs(loss - ref_loss) / ref_loss < 1e-5
        for g, r in zip(grads, ref_grads):
            assert np.linalg.norm(g - r) / np.linalg.norm(r) < 1e-5
    server.close()
