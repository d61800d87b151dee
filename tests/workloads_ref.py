"""Model builders that restate the reference's regression-test setups.

Each builder follows the cited reference test so that the oracle (and the GPU
path) can be checked against the reference's golden values.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from openturbine_b200.model import (BeamSection, CreateTrapezoidalQuadrature, GenerateGLLPoints,
                                    Model, RotateVectorByQuaternion, RotationVectorToQuaternion,
                                    StepParameters)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name: str) -> dict:
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


# Uniform composite section of test_cantilever_beam.cpp / test_solver.cpp.
COMPOSITE_MASS = np.diag([8.538e-2, 8.538e-2, 8.538e-2, 1.4433e-2, 0.40972e-2, 1.0336e-2])
COMPOSITE_STIFF = np.array([
    [1368.17e3, 0., 0., 0., 0., 0.],
    [0., 88.56e3, 0., 0., 0., 0.],
    [0., 0., 38.78e3, 0., 0., 0.],
    [0., 0., 0., 16.9600e3, 17.6100e3, -0.3510e3],
    [0., 0., 0., 17.6100e3, 59.1200e3, -0.3700e3],
    [0., 0., 0., -0.3510e3, -0.3700e3, 141.470e3],
])
GAUSS7 = [
    [-0.9491079123427585, 0.1294849661688697], [-0.7415311855993943, 0.27970539148927664],
    [-0.40584515137739696, 0.3818300505051189], [6.123233995736766e-17, 0.4179591836734694],
    [0.4058451513773971, 0.3818300505051189], [0.7415311855993945, 0.27970539148927664],
    [0.9491079123427585, 0.1294849661688697],
]
GLL6_S = [0., 0.11747233803526763, 0.35738424175967748, 0.64261575824032247,
          0.88252766196473242, 1.]


def cantilever_test_model():
    """tests/regression_tests/regression/test_cantilever_beam.cpp:31-100."""
    node_s = [0., 0.17267316464601146, 0.5, 0.8273268353539885, 1.]
    m = Model()
    m.SetGravity(0., 0., 0.)
    ids = [m.AddNode().SetElemLocation(s).SetPosition(10 * s, 0., 0., 1., 0., 0., 0.).Build()
           for s in node_s]
    m.AddBeamElement(ids, [BeamSection(0., COMPOSITE_MASS, COMPOSITE_STIFF),
                           BeamSection(1., COMPOSITE_MASS, COMPOSITE_STIFF)], GAUSS7)
    m.AddFixedBC(ids[0])
    return m, StepParameters(True, 5, 0.005, 0.0)


def cantilever_test_loads(step: int) -> np.ndarray:
    fx = np.zeros((5, 6))
    fx[4, 2] = 100. * math.sin(10.0 * 0.005 * (step + 1))
    return fx


def solver_test_model(x_root: float = 2.0, with_velocity: bool = True):
    """tests/regression_tests/regression/test_solver.cpp:18-110 (6-node rotating beam)."""
    omega = 0.1
    m = Model()
    m.SetGravity(0., 0., 0.)
    ids = []
    for s in GLL6_S:
        x = 10 * s + x_root
        b = m.AddNode().SetElemLocation(s).SetPosition(x, 0., 0., 1., 0., 0., 0.)
        if with_velocity:
            b.SetVelocity(0., x * omega, 0., 0., 0., omega)
        ids.append(b.Build())
    m.AddBeamElement(ids, [BeamSection(0., COMPOSITE_MASS, COMPOSITE_STIFF),
                           BeamSection(1., COMPOSITE_MASS, COMPOSITE_STIFF)], GAUSS7)
    m.AddPrescribedBC(ids[0])
    return m


def solver_test_root_displacement(x_root: float = 2.0, omega: float = 0.1, h: float = 0.01):
    u_rot = RotationVectorToQuaternion([0., 0., omega * h])
    xr = RotateVectorByQuaternion(u_rot, [x_root, 0., 0.])
    return [xr[0] - x_root, xr[1] - 0., xr[2] - 0., *u_rot]


def rotating_beam_test_model():
    """tests/regression_tests/regression/test_rotating_beam.cpp:93-125."""
    m = Model()
    m.SetGravity(0., 0., 0.)
    ids = [m.AddNode().SetElemLocation(s).SetPosition(10 * s, 0., 0., 1., 0., 0., 0.).Build()
           for s in GLL6_S]
    m.AddBeamElement(ids, [BeamSection(0., COMPOSITE_MASS, COMPOSITE_STIFF),
                           BeamSection(1., COMPOSITE_MASS, COMPOSITE_STIFF)], GAUSS7)
    m.TranslateBeam(0, [2.0, 0., 0.])
    m.SetBeamVelocityAboutPoint(0, [0., 0., 0., 0., 0., 0.1], [0., 0., 0.])
    m.AddPrescribedBC(ids[0])
    return m, StepParameters(True, 5, 0.01, 0.9)


def rotating_beam_root_displacement(i: int, omega: float = 0.1, h: float = 0.01):
    x0_root = [2., 0., 0.]
    q = RotationVectorToQuaternion([0., 0., omega * h * (i + 1)])
    xr = RotateVectorByQuaternion(q, x0_root)
    return [xr[0] - x0_root[0], xr[1] - x0_root[1], xr[2] - x0_root[2], *q]


def rotation_control_test_model(prescribed_hub: bool = False):
    """tests/regression_tests/regression/test_rotating_beam.cpp:390-430
    (RotationControlConstraint: hub held by a FixedBC) and :458-500
    (CompoundRotationControlConstraint: hub turned by a PrescribedBC).  The
    blade root is pitched about x by a RotationControl from the hub.  Returns
    (model, params, rotation-control constraint id, hub BC constraint id)."""
    m = Model()
    m.SetGravity(0., 0., 0.)
    ids = [m.AddNode().SetElemLocation(s).SetPosition(10 * s, 0., 0., 1., 0., 0., 0.).Build()
           for s in GLL6_S]
    m.AddBeamElement(ids, [BeamSection(0., COMPOSITE_MASS, COMPOSITE_STIFF),
                           BeamSection(1., COMPOSITE_MASS, COMPOSITE_STIFF)], GAUSS7)
    m.TranslateBeam(0, [2.0, 0., 0.])
    hub = m.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build()
    rc = m.AddRotationControl([hub, ids[0]], [1., 0., 0.])
    bc = m.AddPrescribedBC(hub) if prescribed_hub else m.AddFixedBC(hub)
    return m, StepParameters(True, 5, 0.01, 0.9), rc, bc


def revolute_joint_test_model():
    """tests/regression_tests/regression/test_rotating_beam.cpp:516-560
    (RevoluteJointConstraint): a blade on a hub node that turns about z on a
    revolute joint from a fixed ground node one unit below it, zero torque,
    blade spinning at 0.1 rad/s about z.  Returns (model, params, revolute
    constraint id); node order: blade (6), hub, ground."""
    m = Model()
    m.SetGravity(0., 0., 0.)
    ids = [m.AddNode().SetElemLocation(s).SetPosition(10 * s, 0., 0., 1., 0., 0., 0.).Build()
           for s in GLL6_S]
    m.AddBeamElement(ids, [BeamSection(0., COMPOSITE_MASS, COMPOSITE_STIFF),
                           BeamSection(1., COMPOSITE_MASS, COMPOSITE_STIFF)], GAUSS7)
    m.TranslateBeam(0, [2.0, 0., 0.])
    m.SetBeamVelocityAboutPoint(0, [0., 0., 0., 0., 0., 0.1], [0., 0., 0.])
    hub = m.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build()
    ground = m.AddNode().SetPosition(0., 0., -1., 1., 0., 0., 0.).Build()
    m.AddFixedBC(ground)
    rj = m.AddRevoluteJointConstraint([ground, hub], [0., 0., 0.], np.zeros(1))
    m.AddRigidJointConstraint([hub, ids[0]])
    return m, StepParameters(True, 5, 0.01, 0.9), rj


def generator_torque_model(tilt: float):
    """tests/regression_tests/regression/test_rotating_beam.cpp:581-650
    (GeneratorTorqueWithAxisTilt): the blade, tilted by `tilt` about x, on a
    hub rigidly held by an azimuth node that turns on a revolute joint about
    (0, sin tilt, cos tilt) from a fixed shaft base, with a generator torque of
    100.  Returns (model, params, revolute constraint id, azimuth node id)."""
    m = Model()
    m.SetGravity(0., 0., 0.)
    q_tilt = RotationVectorToQuaternion([tilt, 0., 0.])
    ids = [m.AddNode().SetElemLocation(s).SetPosition(10 * s, 0., 0., 1., 0., 0., 0.).Build()
           for s in GLL6_S]
    m.AddBeamElement(ids, [BeamSection(0., COMPOSITE_MASS, COMPOSITE_STIFF),
                           BeamSection(1., COMPOSITE_MASS, COMPOSITE_STIFF)], GAUSS7)
    m.TranslateBeam(0, [2.0, 0., 0.])
    m.RotateBeamAboutPoint(0, q_tilt, [0., 0., 0.])
    shaft = m.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build()
    azimuth = m.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build()
    hub = m.AddNode().SetPosition(0., math.sin(tilt), math.cos(tilt), 1., 0., 0., 0.).Build()
    m.AddFixedBC(shaft)
    rj = m.AddRevoluteJointConstraint([shaft, azimuth], [0., math.sin(tilt), math.cos(tilt)],
                                      np.array([100.0]))
    m.AddRigidJointConstraint([azimuth, hub])
    m.AddRigidJointConstraint([hub, ids[0]])
    return m, StepParameters(True, 5, 0.01, 0.0), rj, azimuth


def heavy_top_model():
    """tests/regression_tests/regression/test_heavy_top.cpp:9-75: a 15 kg top
    (inertia diag(0.234375, 0.46875, 0.234375)) at (0, 1, 0) spinning at
    (0, 150, -4.61538) rad/s, held at the origin by a rigid joint to a
    position-only ground node with a prescribed (zero) position; gravity
    -9.81 z; h = 0.002, rho_inf 0.9, tolerances 1e-5 / 1e-3.  Returns (model,
    params, ground BC id)."""
    m = Model()
    m.SetGravity(0., 0., -9.81)
    mass, inertia = 15., (0.234375, 0.46875, 0.234375)
    x, omega = (0., 1., 0.), (0., 150., -4.61538)
    x_dot = (omega[1] * x[2] - omega[2] * x[1], omega[2] * x[0] - omega[0] * x[2],
             omega[0] * x[1] - omega[1] * x[0])
    omega_dot = (661.3461692307691919, 0., 0.)
    x_ddot = (0., -21.3017325444000001, -30.9608307692308244)
    top = (m.AddNode().SetPosition(x[0], x[1], x[2], 1., 0., 0., 0.)
           .SetVelocity(*x_dot, *omega).SetAcceleration(*x_ddot, *omega_dot).Build())
    m.AddMassElement(top, np.diag([mass, mass, mass, *inertia]))
    ground = m.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build()
    m.AddRigidJoint6DOFsTo3DOFs([top, ground])
    bc = m.AddPrescribedBC3DOFs(ground)
    return m, StepParameters(True, 10, 0.002, 0.9, a_tol=1e-5, r_tol=1e-3), bc


PLATFORM_MASS = 1.419625e7
PLATFORM_MOI = (1.2898e10, 1.2851e10, 1.4189e10)
MOORING = [((-40.87, 0.0, -14.), (-105.47, 0.0, -58.4)), ((20.43, -35.39, -14.), (52.73, -91.34, -58.4)),
           ((20.43, 35.39, -14.), (52.73, 91.34, -58.4))]


def cfd_platform_model(mooring: bool):
    """src/interfaces/cfd/interface.cpp:47-115 (CreateFloatingPlatform) with the
    inputs of tests/regression_tests/interfaces/test_cfd_interface.cpp: the
    platform node with its mass, then per mooring line a position-only fairlead
    (RigidJoint6DOFsTo3DOFs from the platform) and anchor (FixedBC3DOFs) joined
    by a spring.  mooring=False: PrecessionTest (unit mass, inertia diag(1, 1,
    0.5), spin (0.5, 0.5, 1), no gravity, rho_inf 1); True: FloatingPlatform
    (14,196 t platform at z = -7.53, three lines of k = 48.9 kN, l0 = 55.432 m,
    gravity -9.8124, rho_inf 0).  Returns (model, params, platform node id)."""
    m = Model()
    if mooring:
        m.SetGravity(0., 0., -9.8124)
        pos, vel = (0., 0., -7.53), (0., 0., 0., 0., 0., 0.)
        mass = np.diag([PLATFORM_MASS] * 3 + list(PLATFORM_MOI))
    else:
        pos, vel = (0., 0., 0.), (0., 0., 0., 0.5, 0.5, 1.)
        mass = np.diag([1., 1., 1., 1., 1., .5])
    plat = m.AddNode().SetPosition(*pos, 1., 0., 0., 0.).SetVelocity(*vel).Build()
    m.AddMassElement(plat, mass)
    for fair, anch in (MOORING if mooring else []):
        f = m.AddNode().SetPosition(*fair, 1., 0., 0., 0.).Build()
        a = m.AddNode().SetPosition(*anch, 1., 0., 0., 0.).Build()
        m.AddFixedBC3DOFs(a)
        m.AddRigidJoint6DOFsTo3DOFs([plat, f])
        m.AddSpringElement(f, a, 48.9e3, 55.432)
    return m, StepParameters(True, 5, 0.01, 0.0 if mooring else 1.0), plat


def cfd_platform_loads(i: int, h: float = 0.01) -> np.ndarray:
    """Platform loads before step i of the FloatingPlatform test (t = i h):
    buoyancy balancing gravity and the initial spring forces plus a sway force
    and three moments, all sinusoidal."""
    t = i * h
    spring0 = 1907514.4912628897
    buoy = spring0 + 9.8124 * PLATFORM_MASS
    w = 2. * math.pi
    return np.array([0., 1e6 * math.sin(w / 20. * t), buoy + 0.5 * spring0 * math.sin(w / 20. * t),
                     5.0e5 * math.sin(w / 15. * t), 1.0e6 * math.sin(w / 30. * t), 2.0e7 * math.sin(w / 60. * t)])


def rotation_control_inputs(i: int, h: float = 0.01):
    """Pitch angle and hub displacement before step i (0-based) of the two
    rotation-control tests: pitch = t pi/2, azimuth = 0.5 t pi/2 about z."""
    t = h * (i + 1)
    q = RotationVectorToQuaternion([0., 0., 0.5 * t * math.pi / 2.])
    return t * math.pi / 2., [0., 0., 0., *q]


def quaternion_to_rotation_vector(q):
    """src/math/quaternion_operations.hpp:267-281 QuaternionToRotationVector."""
    theta = 2. * math.acos(q[0])
    s = math.sqrt(1. - q[0] * q[0])
    if s > 1e-12:
        return [theta * q[1] / s, theta * q[2] / s, theta * q[3] / s]
    return [0., 0., 0.]


def iea15_rotor_model(data: dict | None = None):
    """tests/regression_tests/regression/test_rotor.cpp:25-65 (CreateIEA15Blades)."""
    d = data or load_golden("iea15_rotor.json")
    m = Model()
    m.SetGravity(*d["gravity"])
    node_loc = [(xi + 1.) / 2. for xi in d["node_xi"]]
    sections = [BeamSection(s["position"], np.array(s["M_star"]).reshape(6, 6),
                            np.array(s["C_star"]).reshape(6, 6)) for s in d["sections"]]
    omega = d["omega"]
    velocity = [0., 0., 0., omega[0], omega[1], omega[2]]
    hub = [d["hub_radius"], 0., 0.]
    nb = 3
    for b in range(nb):
        rq = RotationVectorToQuaternion([0., 0., -2. * math.pi * b / nb])
        ids = [m.AddNode().SetElemLocation(node_loc[j]).SetPosition(d["node_coords"][j]).Build()
               for j in range(len(node_loc))]
        e = m.AddBeamElement(ids, sections, d["quadrature"])
        m.TranslateBeam(e, hub)
        m.RotateBeamAboutPoint(e, rq, [0., 0., 0.])
        m.SetBeamVelocityAboutPoint(e, velocity, [0., 0., 0.])
    bc = [m.AddPrescribedBC(be.node_ids[0]) for be in m.GetBeamElements()]
    params = StepParameters(True, d["max_iter"], d["h"], d["rho_inf"])
    return m, params, bc


def iea15_hub_displacement(i: int, data: dict | None = None):
    d = data or load_golden("iea15_rotor.json")
    w, h = d["omega"], d["h"]
    q = RotationVectorToQuaternion([w[0] * h * (i + 1), w[1] * h * (i + 1), w[2] * h * (i + 1)])
    return [0., 0., 0., *q]


def iea15_hub_rotor_model(data: dict | None = None):
    """test_rotor.cpp:191-243 (IEA15RotorHub): the IEA-15 blades of
    CreateIEA15Blades, a hub node at the origin, a rigid joint from the hub to
    every blade root and a prescribed hub motion."""
    d = data or load_golden("iea15_rotor.json")
    m = Model()
    m.SetGravity(*d["gravity"])
    node_loc = [(xi + 1.) / 2. for xi in d["node_xi"]]
    sections = [BeamSection(s["position"], np.array(s["M_star"]).reshape(6, 6),
                            np.array(s["C_star"]).reshape(6, 6)) for s in d["sections"]]
    omega = d["omega"]
    velocity = [0., 0., 0., omega[0], omega[1], omega[2]]
    hub = [d["hub_radius"], 0., 0.]
    for b in range(3):
        rq = RotationVectorToQuaternion([0., 0., -2. * math.pi * b / 3])
        ids = [m.AddNode().SetElemLocation(node_loc[j]).SetPosition(d["node_coords"][j]).Build()
               for j in range(len(node_loc))]
        e = m.AddBeamElement(ids, sections, d["quadrature"])
        m.TranslateBeam(e, hub)
        m.RotateBeamAboutPoint(e, rq, [0., 0., 0.])
        m.SetBeamVelocityAboutPoint(e, velocity, [0., 0., 0.])
    hub_id = m.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build()
    for be in m.GetBeamElements():
        m.AddRigidJointConstraint([hub_id, be.node_ids[0]])
    hub_bc = m.AddPrescribedBC(hub_id)
    params = StepParameters(True, 6, d["h"], 0.0)
    return m, params, hub_bc, hub_id


# ---- point masses and springs (tests/regression_tests/regression/) -----------------
def mass_external_force_model():
    """test_masses.cpp:79-144 (ExternalForce): a free unit mass, force_x = 5 and
    torque_y = 3 in state.f, h = 0.001, rho_inf = 0, 1000 steps."""
    m = Model()
    m.SetGravity(0., 0., 0.)
    n = m.AddNode().SetPosition(0, 0, 0, 1, 0, 0, 0).Build()
    m.AddMassElement(n, np.eye(6))
    f = np.zeros((1, 6))
    f[0, 0], f[0, 4] = 5., 3.
    return m, StepParameters(True, 5, 0.001, 0.0), f


def precession_model():
    """test_precession.cpp:9-40: a free mass spinning with v = (0,0,0,0.5,0.5,1)
    and inertia diag(1, 1, 0.5); h = 0.01, rho_inf = 1, 500 steps."""
    m = Model()
    n = m.AddNode().SetVelocity(0., 0., 0., 0.5, 0.5, 1.0).Build()
    m.AddMassElement(n, np.diag([1., 1., 1., 1., 1., 0.5]))
    return m, StepParameters(True, 6, 0.01, 1.0)


def spring_mass_model():
    """test_spring_mass_system.cpp:23-60: a unit mass at x = 2 on a spring
    (k = 10, l0 = 0) to a fixed node at the origin; h = T/1000 with
    T = 2 pi sqrt(m/k), rho_inf = 0, 1000 steps."""
    m = Model()
    fixed = m.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build()
    mass = m.AddNode().SetPosition(2., 0., 0., 1., 0., 0., 0.).Build()
    m.AddMassElement(mass, np.eye(6))
    m.AddFixedBC(fixed)
    m.AddSpringElement(fixed, mass, 10., 0.)
    period = 2. * math.pi * math.sqrt(1. / 10.)
    return m, StepParameters(True, 6, period / 1000., 0.0)


def spring_mass_chain_model(number_of_masses: int = 10):
    """test_spring_mass_system.cpp:113-185: equal unit masses between equal
    springs (k = 10, l0 = 0) anchored at both ends: static equilibrium."""
    m = Model()
    position = 0.
    m.AddNode().SetPosition(position, 0., 0., 1., 0., 0., 0.)
    for _ in range(number_of_masses):
        position += 0.5
        m.AddNode().SetPosition(position, 0., 0., 1., 0., 0., 0.)
    position += 0.5
    m.AddNode().SetPosition(position, 0., 0., 1., 0., 0., 0.)
    for k in range(number_of_masses):
        m.AddMassElement(k + 1, np.eye(6))
    for k in range(number_of_masses + 1):
        m.AddSpringElement(k, k + 1, 10., 0.)
    m.AddFixedBC(0)
    m.AddFixedBC(number_of_masses + 1)
    final_time = 2. * math.pi * math.sqrt(1. / 10.)
    return m, StepParameters(True, 6, final_time / 1000., 0.0)


def two_element_cantilever_model():
    """A 10 m cantilever of two quadratic elements sharing the middle node C:
    element 1 = (A, B, C) along +x, element 2 = (E, D, C) parametrised from the
    tip back to C (Node::s is one value per node, so the shared node sits at
    s = 1 of both elements).  Composite section of test_cantilever_beam.cpp,
    4 Gauss points per element, FixedBC at A; the tip load goes on E
    (element 2, local node 0)."""
    m = Model()
    m.SetGravity(0., 0., 0.)
    xs = [0., 2.5, 5., 7.5, 10.]
    ss = [0., 0.5, 1., 0.5, 0.]
    ids = [m.AddNode().SetElemLocation(s).SetPosition(x, 0., 0., 1., 0., 0., 0.).Build()
           for x, s in zip(xs, ss)]
    secs = [BeamSection(0., COMPOSITE_MASS, COMPOSITE_STIFF),
            BeamSection(1., COMPOSITE_MASS, COMPOSITE_STIFF)]
    g4 = [[x, w] for x, w in zip(*np.polynomial.legendre.leggauss(4))]
    m.AddBeamElement([ids[0], ids[1], ids[2]], secs, g4)
    m.AddBeamElement([ids[4], ids[3], ids[2]], secs, g4)
    m.AddFixedBC(ids[0])
    return m, StepParameters(True, 5, 0.005, 0.0)


def two_element_cantilever_loads(step: int) -> np.ndarray:
    """node_FX rows per element node (element 1: A, B, C; element 2: E, D, C)."""
    fx = np.zeros((6, 6))
    fx[3, 2] = 100. * math.sin(10.0 * 0.005 * (step + 1))
    return fx


# ---- beams in one dense bordered system --------------------------------------------
def two_beams_model():
    """BladeInterfaceTest.TwoBeams (tests/regression_tests/interfaces/
    test_blade_interface.cpp:312-372): two straight 10 m beams of order 3 along
    x, built like components::BeamBuilder builds them from a straight reference
    axis (GLL nodes, 21 sections at s = 0, 0.05, ..., 1 with the test's
    diagonal mass and coupled stiffness, trapezoidal quadrature at the
    sections), the second moved 10 m along x; a PrescribedBC at the first
    beam's root and a RigidJoint from its tip to the second beam's root;
    gravity -9.81 z; StepParameters(true, 6, 0.01, 0)."""
    section_s = [0.05 * k for k in range(21)]
    mass = np.diag([8.538e-2, 8.538e-2, 8.538e-2, 1.4433e-2, 0.40972e-2, 1.0336e-2])
    stiff = np.diag([1368.17e3, 88.56e3, 38.78e3, 16.96e3, 59.12e3, 141.47e3])
    stiff[3, 4] = stiff[4, 3] = 17.61e3
    stiff[3, 5] = stiff[5, 3] = -0.351e3
    stiff[4, 5] = stiff[5, 4] = -0.37e3
    secs = [BeamSection(s, mass, stiff) for s in section_s]
    quad = CreateTrapezoidalQuadrature(section_s)
    m = Model()
    m.SetGravity(0., 0., -9.81)
    beams = []
    for b in range(2):
        ids = [m.AddNode().SetElemLocation(s).SetPosition(10. * s + 10. * b, 0., 0., 1., 0., 0., 0.).Build()
               for s in [(x + 1.) / 2. for x in GenerateGLLPoints(3)]]
        m.AddBeamElement(ids, secs, quad)
        beams.append(ids)
    m.AddPrescribedBC(beams[0][0])
    m.AddRigidJointConstraint([beams[0][-1], beams[1][0]])
    return m, StepParameters(True, 6, 0.01, 0.)


def moored_cantilever_model():
    """The cantilever of test_cantilever_beam.cpp with a mooring line at its
    tip (the floating platform's line of test_cfd_interface.cpp on a beam): a
    position-only fairlead node carried by a RigidJoint6DOFsTo3DOFs from the tip,
    a spring to a position-only anchor held by a FixedBC3DOFs; the tip also
    carries a point mass.  Solved as one dense system."""
    m, p = cantilever_test_model()
    tip = 4
    fair = m.AddNode().SetPosition(10., 0., -1., 1., 0., 0., 0.).Build()
    anchor = m.AddNode().SetPosition(10., 0., -21., 1., 0., 0., 0.).Build()
    m.AddRigidJoint6DOFsTo3DOFs([tip, fair])
    m.AddSpringElement(fair, anchor, 5.0e3, 19.0)
    m.AddFixedBC3DOFs(anchor)
    m.AddMassElement(tip, np.diag([50., 50., 50., 5., 5., 5.]))
    return m, p


# ---- condensed dense models (beams longer than one FP64 beam system) ---------------
def chain_beam(m: Model, n_elem: int, order: int, length: float, q_axis, sections, quad, origin=(0., 0., 0.)):
    """Adds a straight beam of n_elem elements of the given order along the
    local x axis rotated by q_axis, the elements sharing their end nodes.
    Node::s is one value per node, so the elements alternate direction: odd
    elements are parametrised from their far end back to the shared node,
    which then sits at the same s in both elements.  Returns the node ids in
    order along the beam and the element node lists."""
    gll = [(x + 1.) / 2. for x in GenerateGLLPoints(order)]
    le = length / n_elem
    ends = []
    for e in range(n_elem + 1):
        s = 0. if e % 2 == 0 else 1.
        p = RotateVectorByQuaternion(q_axis, [le * e, 0., 0.])
        ends.append(m.AddNode().SetElemLocation(s).SetPosition(
            origin[0] + p[0], origin[1] + p[1], origin[2] + p[2], *q_axis).Build())
    along = [ends[0]]
    elems = []
    for e in range(n_elem):
        fwd = e % 2 == 0
        inner = []
        for s in gll[1:-1]:
            xl = le * e + le * (s if fwd else 1. - s)
            p = RotateVectorByQuaternion(q_axis, [xl, 0., 0.])
            inner.append(m.AddNode().SetElemLocation(s).SetPosition(
                origin[0] + p[0], origin[1] + p[1], origin[2] + p[2], *q_axis).Build())
        nodes = [ends[e]] + inner + [ends[e + 1]] if fwd else [ends[e + 1]] + inner + [ends[e]]
        m.AddBeamElement(nodes, sections, quad)
        elems.append(nodes)
        along += (inner if fwd else inner[::-1]) + [ends[e + 1]]
    return along, elems


def four_element_cantilever_model():
    """A 40 m cantilever of four order-10 elements (41 nodes) with the
    composite section of test_cantilever_beam.cpp and 12 Gauss points per
    element, FixedBC at the root, no gravity: larger than one FP64 beam
    system, so each element's interior nodes are condensed inside the
    element and the four shared end nodes form the bordered system."""
    m = Model()
    m.SetGravity(0., 0., 0.)
    secs = [BeamSection(0., COMPOSITE_MASS, COMPOSITE_STIFF), BeamSection(1., COMPOSITE_MASS, COMPOSITE_STIFF)]
    g12 = [[x, w] for x, w in zip(*np.polynomial.legendre.leggauss(12))]
    along, elems = chain_beam(m, 4, 10, 40., [1., 0., 0., 0.], secs, g12)
    m.AddFixedBC(along[0])
    return m, StepParameters(True, 6, 0.005, 0.0), along, elems


def chain_tip_loads(elems, tip: int, step: int, h: float = 0.005) -> np.ndarray:
    """node_FX rows per element node (elements in order) with a tip force
    100 sin(10 t) along z and a tip moment about x."""
    rows = sum(len(e) for e in elems)
    fx = np.zeros((rows, 6))
    at = 0
    for nodes in elems:
        if tip in nodes:
            r = at + nodes.index(tip)
            fx[r, 2] = 100. * math.sin(10.0 * h * (step + 1))
            fx[r, 3] = 20. * math.sin(7.0 * h * (step + 1))
            break
        at += len(nodes)
    return fx


def hollow_circle_section(s: float, E: float, G: float, rho: float, D: float, t: float, nu: float):
    """Mass and stiffness of a thin-walled circular tube in the beam's frame
    (axial direction first): the properties of hollow_circle_properties.hpp
    (area, I, J, Timoshenko shear factor 6(1 + nu)/(7 + 6 nu)), placed on
    the diagonal as [EA, kGA, kGA, GJ, EI, EI] and [m, m, m, Ip, I, I]."""
    ro, ri = D / 2., D / 2. - t
    A = math.pi * (ro ** 2 - ri ** 2)
    I = math.pi * (ro ** 4 - ri ** 4) / 4.
    J = 2. * I
    k = 6. * (1. + nu) / (7. + 6. * nu)
    mass = np.diag([rho * A, rho * A, rho * A, rho * 2. * I, rho * I, rho * I])
    stiff = np.diag([E * A, k * G * A, k * G * A, G * J, E * I, E * I])
    return BeamSection(s, mass, stiff)


def tower_model():
    """A 90 m steel tower along z of three order-10 elements (31 nodes; 6 m
    tube, 30 mm wall, 12 Gauss points per element) with a PrescribedBC at
    its base, a nacelle point mass at its top and gravity -9.81 z; the top
    node (a point mass) and the shared element ends form the bordered
    system of the condensed model."""
    m = Model()
    m.SetGravity(0., 0., -9.81)
    secs = [hollow_circle_section(s, 200e9, 79.3e9, 7850., 6., 0.03, 0.3) for s in (0., 1.)]
    g12 = [[x, w] for x, w in zip(*np.polynomial.legendre.leggauss(12))]
    qz = [math.sqrt(0.5), 0., -math.sqrt(0.5), 0.]   # local x -> global z
    along, elems = chain_beam(m, 3, 10, 90., qz, secs, g12)
    m.AddPrescribedBC(along[0])
    m.AddMassElement(along[-1], np.diag([2.0e5, 2.0e5, 2.0e5, 4.0e6, 3.0e6, 3.0e6]))
    return m, StepParameters(True, 6, 0.01, 0.0), along, elems


def two_long_beams_model():
    """BladeInterfaceTest.TwoBeams with two order-20 beams (21 nodes each):
    joined by a RigidJoint they need 264 unknowns as one dense system, so the
    model is condensed (each beam's 19 interior nodes eliminated inside the
    beam)."""
    section_s = [0.05 * k for k in range(21)]
    mass = np.diag([8.538e-2, 8.538e-2, 8.538e-2, 1.4433e-2, 0.40972e-2, 1.0336e-2])
    stiff = np.diag([1368.17e3, 88.56e3, 38.78e3, 16.96e3, 59.12e3, 141.47e3])
    stiff[3, 4] = stiff[4, 3] = 17.61e3
    stiff[3, 5] = stiff[5, 3] = -0.351e3
    stiff[4, 5] = stiff[5, 4] = -0.37e3
    secs = [BeamSection(s, mass, stiff) for s in section_s]
    quad = CreateTrapezoidalQuadrature(section_s)
    m = Model()
    m.SetGravity(0., 0., -9.81)
    beams = []
    for b in range(2):
        ids = [m.AddNode().SetElemLocation(s).SetPosition(10. * s + 10. * b, 0., 0., 1., 0., 0., 0.).Build()
               for s in [(x + 1.) / 2. for x in GenerateGLLPoints(20)]]
        m.AddBeamElement(ids, secs, quad)
        beams.append(ids)
    m.AddPrescribedBC(beams[0][0])
    m.AddRigidJointConstraint([beams[0][-1], beams[1][0]])
    return m, StepParameters(True, 6, 0.01, 0.), beams


def revolute_pendulum_model():
    """A beam-free dense model with a revolute joint: a shaft base held by a
    FixedBC, a revolute joint about x to a light hub node carrying a point
    mass, and a heavy point mass rigidly jointed to the hub 0.5 m off the
    axis; gravity -9.81 z swings it about the joint while the joint's torque
    drives it.  Solved as one dense bordered system (the revolute joint as
    five constraint rows, not a drive train)."""
    m = Model()
    m.SetGravity(0., 0., -9.81)
    base = m.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build()
    hub = m.AddNode().SetPosition(1., 0., 0., 1., 0., 0., 0.).Build()
    bob = m.AddNode().SetPosition(1., 0.5, 0., 1., 0., 0., 0.).Build()
    m.AddFixedBC(base)
    m.AddRevoluteJointConstraint([base, hub], [1., 0., 0.])
    m.AddRigidJointConstraint([hub, bob])
    m.AddMassElement(hub, np.diag([2., 2., 2., 0.5, 0.4, 0.4]))
    m.AddMassElement(bob, np.diag([20., 20., 20., 1., 1., 1.]))
    return m, StepParameters(True, 8, 0.005, 0.5)
