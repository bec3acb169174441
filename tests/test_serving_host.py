"""CPU: the gradient server's host logic -- requests dealt to devices by grid (a device keeps the
grids it was given), submission order kept per device and in the results, errors reported after
the other devices finish.  The per-request GPU work is replaced by a recorder."""
import threading
from types import SimpleNamespace

import pytest

from elasticisolib_3d_b200.serving import GradientRequest, GradientServer


def _fd(n, nts):
    return SimpleNamespace(nz=n, nx=n, ny=n, nts=nts, sub=4, minPad=40, dz=10.0, dx=10.0, dy=10.0, dts=0.002)


def _requests():
    grids = [_fd(200, 1000), _fd(300, 2000), _fd(200, 1000), _fd(330, 3000), _fd(300, 2000), _fd(200, 1500)]
    return [GradientRequest(fd, None, None, None, None, None) for fd in grids]


def test_requests_are_dealt_by_grid_in_submission_order(monkeypatch):
    server = GradientServer(devices=(0, 1), autotune=False)
    seen, lock = [], threading.Lock()

    def fake(dev, req):
        with lock:
            seen.append((dev, id(req)))
        req.result = (float(dev), id(req))
        return req.result

    monkeypatch.setattr(server, "_serve_one", fake)
    reqs = _requests()
    out = server.serve(reqs)
    assert [o[1] for o in out] == [id(r) for r in reqs]          # results in submission order
    dev_of = dict((i, d) for d, i in seen)
    # same grid (shape and record) -> same device; four distinct grids over two devices
    assert dev_of[id(reqs[0])] == dev_of[id(reqs[2])]
    assert dev_of[id(reqs[1])] == dev_of[id(reqs[4])]
    assert {dev_of[id(r)] for r in reqs} == {0, 1}
    for d in (0, 1):                                              # per-device order kept
        ids = [i for dd, i in seen if dd == d]
        assert ids == [id(r) for r in reqs if dev_of[id(r)] == d]


def test_a_failing_device_is_reported_after_the_others(monkeypatch):
    server = GradientServer(devices=(0, 1), autotune=False)
    done = []

    def fake(dev, req):
        if dev == 1:
            raise RuntimeError("device 1 failed")
        done.append(id(req))
        req.result = (0.0, None)
        return req.result

    monkeypatch.setattr(server, "_serve_one", fake)
    reqs = _requests()
    with pytest.raises(RuntimeError, match="device 1 failed"):
        server.serve(reqs)
    assert done  # device 0 finished its requests


def test_least_recently_used_problems_close_to_admit_a_new_grid(monkeypatch):
    import torch
    from elasticisolib_3d_b200 import serving as SV

    opened, closed = [], []

    class FakeProblem:
        def __init__(self, fd, device=None, ckpt=None, variant=None):
            self.fd = fd
            self.prop = SimpleNamespace(close=lambda: closed.append(fd.nz))
            opened.append(fd.nz)

    total = 3 * SV._estimate_bytes(_fd(200, 1000)) + 3 * (2 << 30)   # room for about three 200^3 grids
    open_problems = lambda: sum(len(p) for p in server.open.values())   # noqa: E731
    monkeypatch.setattr(SV.F, "FwiProblem", FakeProblem)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda dev=None: None)
    monkeypatch.setattr(torch.cuda, "empty_cache", lambda: None)
    monkeypatch.setattr(torch.cuda, "mem_get_info",
                        lambda dev=None: (total - open_problems() * (SV._estimate_bytes(_fd(200, 1000)) + (2 << 30)),
                                          total))
    server = SV.GradientServer(devices=(0,), autotune=False)
    a, b, c, d = _fd(200, 1000), _fd(201, 1000), _fd(202, 1000), _fd(203, 1000)
    server._problem(0, a)
    server._problem(0, b)
    server._problem(0, a)          # a is now the most recently used
    server._problem(0, c)          # fits: three open
    server._problem(0, d)          # does not fit: b (least recently used) closes first
    assert closed and closed[0] == 201
    assert opened == [200, 201, 202, 203]


def test_requests_differing_only_in_the_sponge_or_free_surface_get_their_own_problem(monkeypatch):
    """The problem cache is keyed by everything FwiProblem takes from the request's parameters: a
    request whose taper constant (alphaCos) differs gets its own problem, and a free-surface request
    reaches FwiProblem (which refuses it) instead of reusing a problem built without one."""
    import torch
    from elasticisolib_3d_b200 import serving as SV

    built = []

    class FakeProblem:
        def __init__(self, fd, device=None, ckpt=None, variant=None):
            if getattr(fd, "freeSurface", 0):
                raise ValueError("free surface")
            built.append(fd)
            self.fd = fd
            self.prop = SimpleNamespace(close=lambda: None)

    monkeypatch.setattr(SV.F, "FwiProblem", FakeProblem)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda dev=None: None)
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda dev=None: (1 << 50, 1 << 50))
    server = SV.GradientServer(devices=(0,), autotune=False)
    a = _fd(200, 1000)
    a.alphaCos, a.freeSurface = 0.99, 0
    b = SimpleNamespace(**vars(a))
    b.alphaCos = 0.95
    pa = server._problem(0, a)
    pb = server._problem(0, b)
    assert pa is not pb and pb.fd.alphaCos == 0.95
    assert server._problem(0, SimpleNamespace(**vars(a))) is pa      # identical parameters: reused
    fs = SimpleNamespace(**vars(a))
    fs.freeSurface = 1
    with pytest.raises(ValueError, match="free surface"):
        server._problem(0, fs)
    assert len(built) == 2
