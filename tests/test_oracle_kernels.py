"""Kernel-level oracle functions against test_curved_beam.hpp (Mathematica data)
and the reference's math unit tests."""
import ctypes

import numpy as np
import pytest

from oracle.oracle_py import lib
from tests.workloads_ref import load_golden

D = ctypes.POINTER(ctypes.c_double)


def p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(D)


@pytest.fixture(scope="module")
def cb():
    return {k: (np.array(v) if isinstance(v, list) else v)
            for k, v in load_golden("curved_beam.json").items()}


def test_lagrange_weights(cb):
    L = lib()
    gll = np.array(cb["kGLLNodes"])
    for qp, x in enumerate(cb["kGaussQuadraturePoints"]):
        w = np.zeros(3)
        L.orc_lagrange_interp_weights(ctypes.c_double(x), p(gll), 3, p(w) if False else w.ctypes.data_as(D))
        np.testing.assert_allclose(w, cb["kExpectedInterpWeights"].reshape(7, 3)[qp], atol=1e-12)
        L.orc_lagrange_deriv_weights(ctypes.c_double(x), p(gll), 3, w.ctypes.data_as(D))
        np.testing.assert_allclose(w, cb["kExpectedDerivWeights"].reshape(7, 3)[qp], atol=1e-12)


def test_jacobian(cb):
    L = lib()
    nodes = cb["kCurvedBeamNodes_data"].reshape(3, 7)
    dphi = cb["kDerivWeightsFlat"].reshape(3, 7)
    x0p = np.zeros((7, 3))
    jac = np.zeros(7)
    L.orc_calc_jacobian(3, 7, p(dphi), p(nodes), x0p.ctypes.data_as(D), jac.ctypes.data_as(D))
    np.testing.assert_allclose(jac, cb["kExpectedJacobians"], atol=1e-12)
    np.testing.assert_allclose(np.linalg.norm(x0p, axis=1), 1.0, atol=1e-12)


def test_forces_and_matrices(cb):
    L = lib()
    fc = np.zeros(6)
    L.orc_calc_fc(p(cb["kCurvedBeamCuu_data"]), p(cb["kCurvedBeamStrain_data"]), fc.ctypes.data_as(D))
    np.testing.assert_allclose(fc, cb["kExpectedFc_data"], atol=1e-6)
    fd = np.zeros(6)
    L.orc_calc_fd(p(cb["kX0pupSS_data"]), p(cb["kExpectedFc_data"]), fd.ctypes.data_as(D))
    np.testing.assert_allclose(fd, cb["kExpectedFd_data"], atol=1e-6)
    cuu = np.zeros(36)
    L.orc_rotate_section(p(cb["xr_data"]), p(cb["Cstar_data"]), cuu.ctypes.data_as(D))
    np.testing.assert_allclose(cuu, cb["kExpectedCuu_data"], atol=1e-6)
    out = np.zeros(36)
    L.orc_calc_ouu(p(cb["kCurvedBeamCuu_data"]), p(cb["kX0pupSS_data"]),
                   p(cb["kCurvedBeamM_tilde_data"]), p(cb["kCurvedBeamN_tilde_data"]),
                   out.ctypes.data_as(D))
    np.testing.assert_allclose(out, cb["kExpectedOuu_data"], atol=1e-6)
    L.orc_calc_puu(p(cb["kCurvedBeamCuu_data"]), p(cb["kX0pupSS_data"]),
                   p(cb["kCurvedBeamN_tilde_data"]), out.ctypes.data_as(D))
    np.testing.assert_allclose(out, cb["kExpectedPuu_data"], atol=1e-6)
    L.orc_calc_quu(p(cb["kCurvedBeamCuu_data"]), p(cb["kX0pupSS_data"]),
                   p(cb["kCurvedBeamN_tilde_data"]), out.ctypes.data_as(D))
    np.testing.assert_allclose(out, cb["kExpectedQuu_data"], atol=1e-6)


def test_integrate_residual(cb):
    L = lib()
    out = np.zeros((3, 6))
    z6 = np.zeros((7, 6))
    L.orc_integrate_residual(3, 7, p(cb["kGaussQuadratureWeights"]), p(cb["kExpectedJacobians"]),
                             p(cb["kInterpWeightsFlat"].reshape(3, 7)),
                             p(cb["kDerivWeightsFlat"].reshape(3, 7)), p(np.zeros((3, 6))),
                             p(cb["kFc"]), p(cb["kFd"]), p(cb["kFi"]), p(z6), p(z6),
                             out.ctypes.data_as(D))
    np.testing.assert_allclose(out.ravel(), cb["kExpectedResidualVector"], atol=1e-8)


def test_integrate_stiffness(cb):
    L = lib()
    out = np.zeros((3, 3, 36))
    L.orc_integrate_stiffness(3, 7, p(cb["kGaussQuadratureWeights"]), p(cb["kExpectedJacobians"]),
                              p(cb["kInterpWeightsFlat"].reshape(3, 7)),
                              p(cb["kDerivWeightsFlat"].reshape(3, 7)), p(cb["kKuu"]),
                              p(cb["kPuu"]), p(cb["kCuu"]), p(cb["kOuu"]), p(cb["kQuu"]),
                              out.ctypes.data_as(D))
    np.testing.assert_allclose(out.ravel(), cb["kExpectedStiffnessMatrix_data"], atol=1e-7)


def test_gll_points_match_rotor_nodes():
    """GenerateGLLPoints(10) reproduces the IEA-15 node_xi literals."""
    L = lib()
    pts = np.zeros(11)
    L.orc_gll_points(10, pts.ctypes.data_as(D))
    np.testing.assert_allclose(pts, load_golden("iea15_rotor.json")["node_xi"], atol=1e-15)


def test_tangent_operator_small_angle():
    """calculate_tangent_operator.hpp: identity below phi = 1e-16."""
    L = lib()
    T = np.zeros(36)
    L.orc_tangent_operator(ctypes.c_double(0.01), p(np.zeros(6)), T.ctypes.data_as(D))
    np.testing.assert_array_equal(T.reshape(6, 6), np.eye(6))


def test_revolute_joint_kernels():
    """The oracle's revolute joint (residual and gradients, generator torque,
    output) against the reference's unit tests
    test_calculate_revolute_joint_{constraint,force,output}.cpp at their 1e-15
    (unnormalised quaternions: the formulas, not rotations, are checked)."""
    L = lib()
    g = load_golden("revolute_unit.json")
    c = g["constraint"]
    res, bg, tg, sr = np.zeros(6), np.zeros(36), np.zeros(36), np.zeros(6)
    L.orc_revolute_joint(p(c["X0"]), p(c["axes"]), p(c["base_node_u"]), p(c["target_node_u"]),
                         ctypes.c_double(0.), res.ctypes.data_as(D), bg.ctypes.data_as(D),
                         tg.ctypes.data_as(D), sr.ctypes.data_as(D))
    np.testing.assert_allclose(res, c["residual_terms_exact_data"], rtol=0, atol=g["tolerance"])
    np.testing.assert_allclose(bg, c["base_gradient_terms_exact_data"], rtol=0, atol=g["tolerance"])
    np.testing.assert_allclose(tg, -np.array(c["base_gradient_terms_exact_data"]), rtol=0,
                               atol=g["tolerance"])
    f = g["force"]
    L.orc_revolute_joint(p([0., 0., 0.]), p(f["axes"]), p([0., 0., 0., 1., 0., 0., 0.]), p(f["node_u"]),
                         ctypes.c_double(f["constraint_inputs"][0]), res.ctypes.data_as(D),
                         bg.ctypes.data_as(D), tg.ctypes.data_as(D), sr.ctypes.data_as(D))
    np.testing.assert_allclose(sr, f["residual_terms_exact_data"], rtol=0, atol=g["tolerance"])
    o = g["output"]
    out = np.zeros(3)
    L.orc_revolute_output(p(o["axes"]), p(o["node_u"][7:]), p(o["node_udot"][6:]), p(o["node_uddot"][6:]),
                          out.ctypes.data_as(D))
    np.testing.assert_allclose(out, o["outputs_exact_data"], rtol=0, atol=g["tolerance"])


@pytest.mark.parametrize("key,ctype", [("fixed_bc", 1), ("prescribed_bc", 2), ("rigid_joint", 3),
                                       ("rotation_control", 5)])
def test_six_row_constraint_kernels(key, ctype):
    """The oracle's FixedBC, PrescribedBC, RigidJoint and RotationControl
    residuals and gradients against the reference's unit tests
    test_calculate_*_constraint.cpp (unnormalised quaternions).  The tests'
    own bounds (1e-15 / 1e-12 absolute on entries up to ~6e3) hold the
    reference's operation order; the oracle's order is held to 1e-15 of the
    largest entry, a few units in the last place (measured: exact for the
    FixedBC, <= 3.3e-16 relative for the others)."""
    L = lib()
    c = load_golden("constraint_unit.json")[key]
    ident = [0., 0., 0., 1., 0., 0., 0.]
    inp = c.get("constraint_inputs", ident)
    axis = c["axes"][:3] if "axes" in c else [0., 0., 0.]
    base = c.get("base_node_u", ident)
    target = c.get("target_node_u", c.get("node_u"))
    res, bg, tg = np.zeros(6), np.zeros(36), np.zeros(36)
    L.orc_constraint_kernel(ctype, p(c["X0"]), p(axis), p(inp), p(base), p(target), res.ctypes.data_as(D),
                            bg.ctypes.data_as(D), tg.ctypes.data_as(D))
    def close(a, b):
        b = np.asarray(b)
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-15 * max(1.0, np.abs(b).max()))
    close(res, c["residual_terms_exact_data"])
    close(tg, c["target_gradient_terms_exact_data"])
    if "base_gradient_terms_exact_data" in c:
        close(bg, c["base_gradient_terms_exact_data"])
