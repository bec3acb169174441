"""CPU: host parts of the drop-in operators against the oracle (bit-exact where the arithmetic is)."""
import numpy as np

from operator_case import OperatorCase
from elasticisolib_3d_b200 import operators as OP
from oracle import oracle as O


def test_medium_scaling_matches_oracle_bitwise():
    c = OperatorCase()
    rng = np.random.default_rng(0)
    med = c.med(c.sv.elastic)
    src = c.src_dev[0]
    reg = [rng.standard_normal((src[O.COMP_GRID[k]].getNDeviceReg(), c.nts)).astype(np.float32) for k in range(9)]
    ref = [r.copy() for r in reg]
    O.scale_signals(ref, c.o_src[0], med, c.d[1], c.d[2], c.d[0])
    OP.scale_signals(reg, src, med, c.d[1], c.d[2], c.d[0])
    for a, b in zip(reg, ref):
        np.testing.assert_array_equal(a, b)


def test_born_model_preparation_matches_oracle_bitwise():
    c = OperatorCase()
    rng = np.random.default_rng(1)
    med = c.med(c.sv.elastic)
    model = (rng.standard_normal((3,) + med.shape[1:]) * 1e-2).astype(np.float32)
    np.testing.assert_array_equal(OP.born_model_to_planes(model, med[0:3], c.dtw),
                                  O.born_model_to_planes(model, med[0:3], c.dtw, np.float32))
    planes = rng.standard_normal((8,) + med.shape[1:]).astype(np.float32)
    np.testing.assert_array_equal(OP.born_planes_to_model(planes, med[0:3], c.dtw),
                                  O.born_planes_to_model(planes, med[0:3], c.dtw, None, np.float32))


def test_born_model_preparation_adjoint_pair():
    c = OperatorCase()
    rng = np.random.default_rng(2)
    med = c.med(c.sv.elastic)
    m = rng.standard_normal((3,) + med.shape[1:]).astype(np.float32)
    g = rng.standard_normal((8,) + med.shape[1:]).astype(np.float32)
    lhs = np.vdot(OP.born_model_to_planes(m, med[0:3], c.dtw).astype(np.float64), g)
    rhs = np.vdot(m.astype(np.float64), OP.born_planes_to_model(g, med[0:3], c.dtw))
    assert abs(lhs - rhs) / abs(rhs) < 1e-5


def test_data_component_sampling():
    rng = np.random.default_rng(3)
    dom = rng.standard_normal((2, 9, 5, 7)).astype(np.float32)
    op = OP.ElasticDatComp_3D("p,vx,vz,syz", dom)
    out = np.zeros(op.range_shape, np.float32)
    op.forward(False, dom, out)
    np.testing.assert_allclose(out[:, 0], (dom[:, 3] + dom[:, 4] + dom[:, 5]) / 3.0, rtol=1e-6)
    np.testing.assert_array_equal(out[:, 1], dom[:, 0])
    np.testing.assert_array_equal(out[:, 2], dom[:, 2])
    np.testing.assert_array_equal(out[:, 3], dom[:, 8])
    d = rng.standard_normal(op.range_shape).astype(np.float32)
    m = np.zeros_like(dom)
    op.adjoint(False, m, d)
    assert abs(np.vdot(out.astype(np.float64), d) - np.vdot(dom.astype(np.float64), m)) < 1e-3
