"""The oracle against the reference's own regression-test golden values.

Fixtures come from tests/golden/make_golden.py (reference test sources read as
text).  Tolerances are the reference tests' own.
"""
import math

import numpy as np
import pytest

from oracle.oracle_py import OracleModel
from openturbine_b200.model import StepParameters
from tests.workloads_ref import (cantilever_test_loads, cantilever_test_model,
                                 iea15_hub_displacement, iea15_rotor_model, load_golden,
                                 rotating_beam_root_displacement, rotating_beam_test_model,
                                 solver_test_model, solver_test_root_displacement)


def test_iea15_rotor_q_1e13():
    """test_rotor.cpp:87-189: 3 blades, 11 GLL nodes, 51-pt trapezoid, 11 steps."""
    d = load_golden("iea15_rotor.json")
    m, p, bc = iea15_rotor_model(d)
    o = OracleModel(m.pack())
    assert (o.info.num_dofs, o.info.num_system_dofs) == (216, 198)
    for i in range(d["num_steps"]):
        u = iea15_hub_displacement(i, d)
        for c in bc:
            o.set_prescribed(c, u)
        st, _ = o.step(p)
        assert st == 0
    q = o.state("q")
    for node, comp, val in d["expected_q"]:
        ev = q[val[0], val[1]] if isinstance(val, list) else val
        assert abs(q[node, comp] - ev) <= d["tolerance"], (node, comp, q[node, comp], ev)


def test_cantilever_tip():
    """test_cantilever_beam.cpp:31-138."""
    g = load_golden("cantilever.json")
    m, p = cantilever_test_model()
    o = OracleModel(m.pack())
    for k in range(3):
        o.set_node_fx(cantilever_test_loads(k))
        st, _ = o.step(p)
        assert st == 0
        np.testing.assert_allclose(o.state("q")[4, :3], g["tip_q"][k], rtol=0, atol=g["tolerance"])


def test_solver_predict_assembly():
    """test_solver.cpp:18-243: state and b after predict + assemble."""
    g = load_golden("solver.json")["predict"]
    m = solver_test_model(2.0)
    o = OracleModel(m.pack())
    o.set_prescribed(0, solver_test_root_displacement(2.0))
    o.predict_and_assemble(StepParameters(True, 10, 0.01, 0.9))
    b, _ = o.system_vectors()
    np.testing.assert_allclose(b, g["b"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(o.state("q").ravel(), g["q"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(o.state("q_delta").ravel(), g["q_delta"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(o.state("v").ravel(), g["v"], rtol=0, atol=1e-6)


def test_solver_one_iteration():
    """test_solver.cpp:247-440: x, convergence_err[0] and state after one iteration."""
    g = load_golden("solver.json")["one_iteration"]
    m = solver_test_model(2.0)
    o = OracleModel(m.pack())
    o.set_prescribed(0, solver_test_root_displacement(2.0))
    st, it = o.step(StepParameters(True, 1, 0.01, 0.9))
    assert (st, it) == (1, 1)  # max_iter 1 -> Step() returns false after one iteration
    _, x = o.system_vectors()
    np.testing.assert_allclose(x, g["x"], rtol=0, atol=1e-6)
    assert abs(o.convergence()[0] - g["convergence_err"]) <= 1e-6 * g["convergence_err"]
    for f in ("q_delta", "v", "vd", "q"):
        np.testing.assert_allclose(o.state(f).ravel(), g[f], rtol=0, atol=1e-6)
    np.testing.assert_allclose(o.state("lambda").ravel(), g["lambda"], rtol=0, atol=1e-6)


def test_solver_two_iterations():
    """test_solver.cpp:444-605: b and x of the second iteration."""
    g = load_golden("solver.json")["two_iterations"]
    m = solver_test_model(0.0)
    o = OracleModel(m.pack())
    q = StepParameters(True, 2, 0.01, 0.9)
    from openturbine_b200.model import RotationVectorToQuaternion
    u = RotationVectorToQuaternion([0., 0., 0.1 * 0.01])
    o.set_prescribed(0, [0., 0., 0., *u])
    o.step(q)
    b, x = o.system_vectors()
    np.testing.assert_allclose(b, g["b"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(x, g["x"], rtol=0, atol=1e-6)


def test_rotating_beam_ten_steps():
    """test_rotating_beam.cpp:93-150."""
    g = load_golden("rotating_beam.json")
    m, p = rotating_beam_test_model()
    o = OracleModel(m.pack())
    for i in range(10):
        o.set_prescribed(0, rotating_beam_root_displacement(i))
        st, _ = o.step(p)
        assert st == 0
    np.testing.assert_allclose(o.state("q").ravel(), g["q"], rtol=0, atol=g["tolerance"])


def test_iea15_hub_rotor_converges_and_holds_the_joints():
    """test_rotor.cpp:191-243 (IEA15RotorHub): every step converges within
    max_iter = 6, the hub follows its prescribed rotation, and every blade root
    stays rigidly attached: u_root = R_hub X0 - X0 and R_root = R_hub R0."""
    from openturbine_b200.model import QuaternionCompose, RotateVectorByQuaternion
    from tests.workloads_ref import iea15_hub_rotor_model
    d = load_golden("iea15_rotor.json")
    m, p, hub_bc, hub_id = iea15_hub_rotor_model(d)
    o = OracleModel(m.pack())
    assert o.info.num_dofs == 3 * 66 + 6 + 4 * 6
    for i in range(d["num_steps"]):
        o.set_prescribed(hub_bc, iea15_hub_displacement(i, d))
        st, it = o.step(p)
        assert st == 0 and it <= 6
    q, x0 = o.state("q"), o.state("x0")
    qh = q[hub_id, 3:]
    np.testing.assert_allclose(q[hub_id], iea15_hub_displacement(d["num_steps"] - 1, d), atol=1e-12)
    for be in m.GetBeamElements():
        r = be.node_ids[0]
        X0 = x0[r, :3] - x0[hub_id, :3]
        np.testing.assert_allclose(q[r, :3], np.array(RotateVectorByQuaternion(qh, X0)) - X0, atol=1e-6)
        np.testing.assert_allclose(np.abs(np.dot(q[r, 3:], qh)), 1.0, atol=1e-9)


def test_rotation_control_fixed_hub_ten_steps():
    """test_rotating_beam.cpp:390-456 (RotationControlConstraint): the blade
    root pitched about x by pitch = t pi/2 from a fixed hub, 10 steps, q of all
    7 nodes (the hub last) at the test's 1e-6."""
    from tests.workloads_ref import rotation_control_inputs, rotation_control_test_model
    g = load_golden("rotation_control.json")["fixed_hub"]
    m, p, rc, _ = rotation_control_test_model(prescribed_hub=False)
    o = OracleModel(m.pack())
    for i in range(g["steps"]):
        pitch, _ = rotation_control_inputs(i)
        o.set_prescribed(rc, [pitch, 0., 0., 1., 0., 0., 0.])
        st, _ = o.step(p)
        assert st == 0
    np.testing.assert_allclose(o.state("q").ravel(), g["q"], rtol=0, atol=g["tolerance"])


def test_rotation_control_prescribed_hub_hundred_steps():
    """test_rotating_beam.cpp:458-512 (CompoundRotationControlConstraint): hub
    turned about z by azimuth = 0.5 t pi/2 while the root pitches by t pi/2;
    after 100 steps the root's rotation vector matches at the test's 1e-8."""
    from tests.workloads_ref import (quaternion_to_rotation_vector, rotation_control_inputs,
                                     rotation_control_test_model)
    g = load_golden("rotation_control.json")["prescribed_hub"]
    m, p, rc, bc = rotation_control_test_model(prescribed_hub=True)
    o = OracleModel(m.pack())
    for i in range(g["steps"]):
        pitch, u_hub = rotation_control_inputs(i)
        o.set_prescribed(rc, [pitch, 0., 0., 1., 0., 0., 0.])
        o.set_prescribed(bc, u_hub)
        st, _ = o.step(p)
        assert st == 0
    rv = quaternion_to_rotation_vector(o.state("q")[0, 3:])
    np.testing.assert_allclose(rv, g["rv_root"], rtol=0, atol=g["tolerance"])


def test_revolute_joint_five_steps():
    """test_rotating_beam.cpp:516-579 (RevoluteJointConstraint): q of the 6
    blade nodes, the hub and the ground after 5 steps at the test's 1e-6."""
    from tests.workloads_ref import revolute_joint_test_model
    g = load_golden("revolute_joint.json")["revolute"]
    m, p, rj = revolute_joint_test_model()
    o = OracleModel(m.pack())
    assert o.info.num_dofs == 8 * 6 + 6 + 5 + 6
    for _ in range(g["steps"]):
        o.set_prescribed(rj, [0., 0., 0., 1., 0., 0., 0.])
        st, _ = o.step(p)
        assert st == 0
    np.testing.assert_allclose(o.state("q").ravel(), g["q"], rtol=0, atol=g["tolerance"])


@pytest.mark.parametrize("key", ["tilt0", "tilt90"])
def test_generator_torque(key):
    """test_rotating_beam.cpp:581-680 (GeneratorTorque_Tilt0 / _Tilt90): after
    10 steps under a 100 N m generator torque, the azimuth node's q and v and
    the revolute joint's output (rotation, rate, acceleration about the shaft)
    at the test's 1e-6."""
    from tests.workloads_ref import generator_torque_model
    g = load_golden("revolute_joint.json")["generator_torque"]
    tilt = 0.0 if key == "tilt0" else math.pi / 2.
    m, p, rj, az = generator_torque_model(tilt)
    o = OracleModel(m.pack())
    for _ in range(g["steps"]):
        o.set_prescribed(rj, [g["torque"], 0., 0., 1., 0., 0., 0.])
        st, _ = o.step(p)
        assert st == 0
    np.testing.assert_allclose(o.state("q")[az], g[key]["azimuth_q"], rtol=0, atol=g["tolerance"])
    np.testing.assert_allclose(o.state("v")[az], g[key]["azimuth_v"], rtol=0, atol=g["tolerance"])
    np.testing.assert_allclose(o.state("output")[rj], g[key]["output"], rtol=0, atol=g["tolerance"])


def test_heavy_top_final_rotation():
    """test_heavy_top.cpp:9-75: the top's q after 400 steps (0.8 s) at the
    test's 1e-10; the ground node carries three DOFs (15 DOFs in all)."""
    from tests.workloads_ref import heavy_top_model
    g = load_golden("heavy_top.json")
    m, p, _ = heavy_top_model()
    o = OracleModel(m.pack())
    assert o.info.num_dofs == 6 + 3 + 3 + 3
    for _ in range(g["steps"]):
        st, _ = o.step(p)
        assert st == 0
    np.testing.assert_allclose(o.state("q")[0], g["q_mass_node"], rtol=0, atol=g["tolerance"])


def test_cfd_platform_precession():
    """test_cfd_interface.cpp:12-124 (PrecessionTest): the platform node's q
    after 500 and 600 steps at the test's 1e-12."""
    from tests.workloads_ref import cfd_platform_model
    g = load_golden("cfd_platform.json")["precession"]
    m, p, plat = cfd_platform_model(False)
    o = OracleModel(m.pack())
    for i in range(600):
        st, _ = o.step(p)
        assert st == 0
        if i + 1 == 500:
            np.testing.assert_allclose(o.state("q")[plat], g["q_500"], rtol=0, atol=g["tolerance"])
    np.testing.assert_allclose(o.state("q")[plat], g["q_600"], rtol=0, atol=g["tolerance"])


def test_cfd_floating_platform():
    """test_cfd_interface.cpp:126-222 (FloatingPlatform): three mooring lines
    (position-only fairleads and anchors, 42 DOFs); the platform's q after
    step 100 at the test's 1e-12."""
    from tests.workloads_ref import cfd_platform_loads, cfd_platform_model
    g = load_golden("cfd_platform.json")["floating_platform"]
    m, p, plat = cfd_platform_model(True)
    o = OracleModel(m.pack())
    assert o.info.num_dofs == 6 + 6 * 3 + 6 * 3
    f = np.zeros((o.info.num_nodes, 6))
    for i in range(g["step"] + 1):
        f[plat] = cfd_platform_loads(i)
        o.set_state_f(f)
        st, _ = o.step(p)
        assert st == 0
    np.testing.assert_allclose(o.state("q")[plat], g["q"], rtol=0, atol=g["tolerance"])


def test_mass_external_force_velocity():
    """test_masses.cpp:79-144: v after 1000 steps at the test's 1e-12."""
    from tests.workloads_ref import mass_external_force_model
    g = load_golden("masses_springs.json")["mass_external_force"]
    m, p, f = mass_external_force_model()
    o = OracleModel(m.pack())
    o.set_state_f(f)
    for _ in range(g["steps"]):
        st, _ = o.step(p)
        assert st == 0
    np.testing.assert_allclose(o.state("v")[0], g["v"], rtol=0, atol=g["tolerance"])


def test_precession_final_rotation():
    """test_precession.cpp:29-53: q after 500 steps at the test's 1e-12."""
    from tests.workloads_ref import precession_model
    g = load_golden("masses_springs.json")["precession"]
    m, p = precession_model()
    o = OracleModel(m.pack())
    for _ in range(g["steps"]):
        st, _ = o.step(p)
        assert st == 0
    np.testing.assert_allclose(o.state("q")[0], g["q"], rtol=0, atol=g["tolerance"])


def test_spring_mass_oscillation():
    """test_spring_mass_system.cpp:62-96: x displacement of the mass at T/2 and T."""
    from tests.workloads_ref import spring_mass_model
    g = load_golden("masses_springs.json")["spring_mass"]
    m, p = spring_mass_model()
    o = OracleModel(m.pack())
    for step in range(1, g["steps"] + 1):
        st, _ = o.step(p)
        assert st == 0
        q = o.state("q")
        if step == g["steps"] // 2:
            assert abs(q[0, 0]) <= 1e-14
            assert abs(q[1, 0] - g["q1x_half"]) <= g["tolerance"]
    assert abs(q[1, 0] - g["q1x_end"]) <= g["tolerance"]


def test_spring_mass_chain_stays_in_equilibrium():
    """test_spring_mass_system.cpp:113-185: every x displacement stays 0 (1e-14)."""
    from tests.workloads_ref import spring_mass_chain_model
    g = load_golden("masses_springs.json")["spring_mass_chain"]
    m, p = spring_mass_chain_model()
    o = OracleModel(m.pack())
    for _ in range(g["steps"]):
        st, _ = o.step(p)
        assert st == 0
        assert np.abs(o.state("q")[:, 0]).max() <= g["tolerance"]
