"""Host-side mirror of Kynema's model-building API.

This module re-exposes the reference's setup surface -- ``Model`` with
``AddNode()`` / ``NodeBuilder``, ``AddBeamElement``, ``AddFixedBC``,
``AddPrescribedBC``, ``TranslateBeam``, ``RotateBeamAboutPoint``,
``SetBeamVelocityAboutPoint`` -- plus ``BeamSection``, ``StepParameters`` and
the quaternion / quadrature helpers the reference's tests use to build
models.  It only collects host data; ``Model.to_desc()`` packs it into the
``kyn_model_desc`` C struct consumed by the CUDA library (``kyn_model_create``).

Reference files (paths relative to the reference project root):
  src/model/model.hpp:74-693          Model builder
  src/model/node.hpp:35-538           Node / NodeBuilder kinematics
  src/elements/beams/beam_section.hpp BeamSection
  src/step/step_parameters.hpp:12-53  StepParameters
  src/math/quaternion_operations.hpp  quaternion helpers
  src/math/interpolation.hpp          GLL points
  src/elements/beams/beam_quadrature.hpp CreateTrapezoidalQuadrature
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

# ---- constraint types (src/constraints/constraint_type.hpp:9-24) ----------
FIXED_BC = 1
PRESCRIBED_BC = 2
RIGID_JOINT = 3
REVOLUTE_JOINT = 4
ROTATION_CONTROL = 5
FIXED_BC_3DOF = 6
PRESCRIBED_BC_3DOF = 7
RIGID_JOINT_6DOF_TO_3DOF = 8
INVALID_NODE_ID = 0  # Model::InvalidNodeID


# ---- quaternion helpers (src/math/quaternion_operations.hpp) --------------
def RotationVectorToQuaternion(phi: Sequence[float]) -> list[float]:
    """Host form (quaternion_operations.hpp:299-311): identity below 1e-12."""
    angle = math.sqrt(phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2])
    if abs(angle) < 1e-12:
        return [1.0, 0.0, 0.0, 0.0]
    s = math.sin(angle / 2.0)
    c = math.cos(angle / 2.0)
    f = s / angle
    return [c, phi[0] * f, phi[1] * f, phi[2] * f]


def QuaternionCompose(q1: Sequence[float], q2: Sequence[float]) -> list[float]:
    """quaternion_operations.hpp:216-224."""
    return [
        q1[0] * q2[0] - q1[1] * q2[1] - q1[2] * q2[2] - q1[3] * q2[3],
        q1[0] * q2[1] + q1[1] * q2[0] + q1[2] * q2[3] - q1[3] * q2[2],
        q1[0] * q2[2] - q1[1] * q2[3] + q1[2] * q2[0] + q1[3] * q2[1],
        q1[0] * q2[3] + q1[1] * q2[2] - q1[2] * q2[1] + q1[3] * q2[0],
    ]


def RotateVectorByQuaternion(q: Sequence[float], v: Sequence[float]) -> list[float]:
    """quaternion_operations.hpp:133-146."""
    return [
        (q[0] * q[0] + q[1] * q[1] - q[2] * q[2] - q[3] * q[3]) * v[0]
        + 2.0 * (q[1] * q[2] - q[0] * q[3]) * v[1]
        + 2.0 * (q[1] * q[3] + q[0] * q[2]) * v[2],
        2.0 * (q[1] * q[2] + q[0] * q[3]) * v[0]
        + (q[0] * q[0] - q[1] * q[1] + q[2] * q[2] - q[3] * q[3]) * v[1]
        + 2.0 * (q[2] * q[3] - q[0] * q[1]) * v[2],
        2.0 * (q[1] * q[3] - q[0] * q[2]) * v[0]
        + 2.0 * (q[2] * q[3] + q[0] * q[1]) * v[1]
        + (q[0] * q[0] - q[1] * q[1] - q[2] * q[2] + q[3] * q[3]) * v[2],
    ]


def CrossProduct(a: Sequence[float], b: Sequence[float]) -> list[float]:
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


# ---- quadrature helpers ----------------------------------------------------
def _legendre(n: int, x: float) -> float:
    if n == 0:
        return 1.0
    if n == 1:
        return x
    p2, p1, p = 1.0, x, 0.0
    for i in range(2, n + 1):
        p = ((2.0 * i - 1.0) * x * p1 - (i - 1.0) * p2) / i
        p2, p1 = p1, p
    return p


def GenerateGLLPoints(order: int) -> list[float]:
    """Gauss-Lobatto-Legendre points by Newton iteration (interpolation.hpp)."""
    if order < 1:
        raise ValueError("Polynomial order must be >= 1")
    n = order + 1
    pts = [0.0] * n
    pts[0], pts[-1] = -1.0, 1.0
    for i in range(1, order):
        x = -math.cos(i * math.pi / order)
        for _ in range(1000):
            xo = x
            pn, pm = _legendre(n - 1, x), _legendre(n - 2, x)
            x -= (x * pn - pm) / (n * pn)
            if abs(x - xo) <= np.finfo(float).eps:
                break
        pts[i] = x
    return pts


def CreateTrapezoidalQuadrature(grid: Sequence[float]) -> list[list[float]]:
    """src/elements/beams/beam_quadrature.hpp:11-28."""
    n = len(grid)
    gmin, gmax = min(grid), max(grid)
    rng = gmax - gmin
    quad = [[-1.0, (grid[1] - grid[0]) / rng]]
    for i in range(1, n - 1):
        quad.append([2.0 * (grid[i] - gmin) / rng - 1.0, (grid[i + 1] - grid[i - 1]) / rng])
    quad.append([1.0, (grid[n - 1] - grid[n - 2]) / rng])
    return quad


def GaussLegendreQuadrature(n: int) -> list[list[float]]:
    x, w = np.polynomial.legendre.leggauss(n)
    return [[float(a), float(b)] for a, b in zip(x, w)]


# ---- data classes ----------------------------------------------------------
@dataclass
class BeamSection:
    """src/elements/beams/beam_section.hpp: position in [0,1], M_star, C_star."""

    position: float
    M_star: np.ndarray
    C_star: np.ndarray

    def __post_init__(self) -> None:
        self.M_star = np.asarray(self.M_star, dtype=np.float64).reshape(6, 6)
        self.C_star = np.asarray(self.C_star, dtype=np.float64).reshape(6, 6)


@dataclass
class Node:
    """src/model/node.hpp:35-60."""

    id: int
    x0: list = field(default_factory=lambda: [0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0])
    u: list = field(default_factory=lambda: [0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0])
    v: list = field(default_factory=lambda: [0.0] * 6)
    vd: list = field(default_factory=lambda: [0.0] * 6)
    s: float = 0.0

    def DisplacedPosition(self) -> list[float]:
        q = QuaternionCompose(self.x0[3:7], self.u[3:7])
        return [self.x0[0] + self.u[0], self.x0[1] + self.u[1], self.x0[2] + self.u[2], *q]

    def Translate(self, d: Sequence[float]) -> "Node":
        self.x0[0] += d[0]
        self.x0[1] += d[1]
        self.x0[2] += d[2]
        return self

    def RotateAboutPoint(self, q: Sequence[float], point: Sequence[float]) -> "Node":
        """node.hpp:87-118 (quaternion overload)."""
        r = [self.x0[0] - point[0], self.x0[1] - point[1], self.x0[2] - point[2]]
        rr = RotateVectorByQuaternion(q, r)
        self.x0[0] = rr[0] + point[0]
        self.x0[1] = rr[1] + point[1]
        self.x0[2] = rr[2] + point[2]
        self.x0[3:7] = QuaternionCompose(q, self.x0[3:7])
        return self

    def SetVelocityAboutPoint(self, velocity: Sequence[float], point: Sequence[float]) -> None:
        """node.hpp:196-219."""
        dp = self.DisplacedPosition()
        r = [dp[0] - point[0], dp[1] - point[1], dp[2] - point[2]]
        w = [velocity[3], velocity[4], velocity[5]]
        wxr = CrossProduct(w, r)
        self.v = [velocity[0] + wxr[0], velocity[1] + wxr[1], velocity[2] + wxr[2], *w]


class NodeBuilder:
    """src/model/node.hpp:284-538."""

    def __init__(self, node: Node):
        self.node = node

    def SetPosition(self, *p) -> "NodeBuilder":
        vals = list(p[0]) if len(p) == 1 else list(p)
        if len(vals) == 7:
            self.node.x0 = [float(x) for x in vals]
        elif len(vals) == 3:
            self.node.x0[0:3] = [float(x) for x in vals]
        else:
            raise ValueError("SetPosition takes 3 or 7 values")
        return self

    def SetOrientation(self, *p) -> "NodeBuilder":
        vals = list(p[0]) if len(p) == 1 else list(p)
        self.node.x0[3:7] = [float(x) for x in vals]
        return self

    def SetDisplacement(self, *p) -> "NodeBuilder":
        vals = list(p[0]) if len(p) == 1 else list(p)
        if len(vals) == 7:
            self.node.u = [float(x) for x in vals]
        else:
            self.node.u[0:3] = [float(x) for x in vals]
        return self

    def SetVelocity(self, *p) -> "NodeBuilder":
        vals = list(p[0]) if len(p) == 1 else list(p)
        if len(vals) == 6:
            self.node.v = [float(x) for x in vals]
        else:
            self.node.v[0:3] = [float(x) for x in vals]
        return self

    def SetAcceleration(self, *p) -> "NodeBuilder":
        vals = list(p[0]) if len(p) == 1 else list(p)
        if len(vals) == 6:
            self.node.vd = [float(x) for x in vals]
        else:
            self.node.vd[0:3] = [float(x) for x in vals]
        return self

    def SetElemLocation(self, s: float) -> "NodeBuilder":
        self.node.s = float(s)
        return self

    def Build(self) -> int:
        return self.node.id


@dataclass
class BeamElement:
    id: int
    node_ids: list
    sections: list
    quadrature: list


@dataclass
class MassElement:
    """src/elements/masses/mass_element.hpp."""

    id: int
    node_id: int
    mass: np.ndarray


@dataclass
class SpringElement:
    """src/elements/springs/spring_element.hpp."""

    id: int
    node_ids: tuple
    stiffness: float
    undeformed_length: float


@dataclass
class Constraint:
    """src/constraints/constraint.hpp."""

    id: int
    type: int
    node_ids: tuple
    axis_vector: tuple = (0.0, 0.0, 0.0)
    initial_displacement: tuple = (0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0)


class StepParameters:
    """src/step/step_parameters.hpp:12-53 (derived coefficients kept for tests)."""

    def __init__(self, is_dynamic_solve: bool, max_iter: int, h: float, rho_inf: float,
                 a_tol: float = 1e-5, r_tol: float = 1e-3, precision: int = 0,
                 refine_iters: int = 0):
        self.is_dynamic_solve = bool(is_dynamic_solve)
        self.max_iter = int(max_iter)
        self.h = float(h)
        self.rho_inf = float(rho_inf)
        self.alpha_m = (2.0 * rho_inf - 1.0) / (rho_inf + 1.0)
        self.alpha_f = rho_inf / (rho_inf + 1.0)
        self.gamma = 0.5 + self.alpha_f - self.alpha_m
        self.beta = 0.25 * (self.gamma + 0.5) * (self.gamma + 0.5)
        self.gamma_prime = self.gamma / (h * self.beta) if is_dynamic_solve else 0.0
        self.beta_prime = ((1.0 - self.alpha_m) / (h * h * self.beta * (1.0 - self.alpha_f))
                           if is_dynamic_solve else 0.0)
        self.conditioner = self.beta * h * h
        self.absolute_convergence_tol = float(a_tol)
        self.relative_convergence_tol = float(r_tol)
        self.precision = int(precision)
        self.refine_iters = int(refine_iters)

    def to_c(self) -> "KynStepParams":
        return KynStepParams(int(self.is_dynamic_solve), self.max_iter, self.h, self.rho_inf,
                             self.absolute_convergence_tol, self.relative_convergence_tol,
                             self.precision, self.refine_iters)


# ---- C structs (include/kynema_b200.h) -------------------------------------
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


class KynModelDesc(ctypes.Structure):
    _fields_ = [
        ("num_nodes", ctypes.c_int32),
        ("node_x0", _dp), ("node_u", _dp), ("node_v", _dp), ("node_vd", _dp), ("node_s", _dp),
        ("num_beams", ctypes.c_int32),
        ("beam_node_offsets", _ip), ("beam_node_ids", _ip), ("beam_section_offsets", _ip),
        ("section_position", _dp), ("section_mass", _dp), ("section_stiffness", _dp),
        ("beam_qp_offsets", _ip), ("qp_xi", _dp), ("qp_weight", _dp),
        ("num_constraints", ctypes.c_int32),
        ("constraint_type", _ip), ("constraint_base_node", _ip), ("constraint_target_node", _ip),
        ("constraint_axis", _dp), ("constraint_initial_displacement", _dp),
        ("gravity", ctypes.c_double * 3),
        ("num_masses", ctypes.c_int32), ("mass_node", _ip), ("mass_matrix", _dp),
        ("num_springs", ctypes.c_int32), ("spring_nodes", _ip), ("spring_stiffness", _dp),
        ("spring_length", _dp),
    ]


class KynStepParams(ctypes.Structure):
    _fields_ = [
        ("is_dynamic_solve", ctypes.c_int32), ("max_iter", ctypes.c_int32),
        ("h", ctypes.c_double), ("rho_inf", ctypes.c_double),
        ("absolute_convergence_tol", ctypes.c_double),
        ("relative_convergence_tol", ctypes.c_double),
        ("precision", ctypes.c_int32), ("refine_iters", ctypes.c_int32),
    ]


class KynModelInfo(ctypes.Structure):
    _fields_ = [
        ("num_nodes", ctypes.c_int32), ("num_beams", ctypes.c_int32),
        ("num_constraints", ctypes.c_int32), ("num_system_dofs", ctypes.c_int32),
        ("num_dofs", ctypes.c_int32), ("nnz", ctypes.c_int32),
        ("max_beam_nodes", ctypes.c_int32), ("max_beam_qps", ctypes.c_int32),
        ("device_bytes", ctypes.c_int64), ("condensed_dofs", ctypes.c_int32),
    ]


class PackedModel:
    """Numpy arrays behind a KynModelDesc; keeps them alive while in use."""

    def __init__(self, arrays: dict, gravity):
        self.arrays = arrays
        self.gravity = [float(g) for g in gravity]
        d = KynModelDesc()
        a = arrays
        d.num_nodes = a["node_x0"].shape[0]
        for k in ("node_x0", "node_u", "node_v", "node_vd", "node_s", "section_position",
                  "section_mass", "section_stiffness", "qp_xi", "qp_weight",
                  "constraint_axis", "constraint_initial_displacement", "mass_matrix",
                  "spring_stiffness", "spring_length"):
            setattr(d, k, a[k].ctypes.data_as(_dp) if a[k].size else None)
        d.num_beams = a["beam_node_offsets"].shape[0] - 1
        d.num_constraints = a["constraint_type"].shape[0]
        d.num_masses = a["mass_node"].shape[0]
        d.num_springs = a["spring_nodes"].shape[0]
        for k in ("beam_node_offsets", "beam_node_ids", "beam_section_offsets", "beam_qp_offsets",
                  "constraint_type", "constraint_base_node", "constraint_target_node",
                  "mass_node", "spring_nodes"):
            setattr(d, k, a[k].ctypes.data_as(_ip) if a[k].size else None)
        for i in range(3):
            d.gravity[i] = self.gravity[i]
        self.desc = d

    @property
    def num_nodes(self) -> int:
        return int(self.arrays["node_x0"].shape[0])

    @property
    def num_element_nodes(self) -> int:
        return int(self.arrays["beam_node_ids"].shape[0])


class Model:
    """src/model/model.hpp:74-693 (beams, FixedBC, PrescribedBC, RigidJoint,
    RotationControl, gravity)."""

    InvalidNodeID = INVALID_NODE_ID

    def __init__(self, gravity: Sequence[float] = (0.0, 0.0, 0.0)):
        self.gravity_ = [float(g) for g in gravity]
        self.nodes_: list[Node] = []
        self.beam_elements_: list[BeamElement] = []
        self.constraints_: list[Constraint] = []
        self.controls_: dict = {}
        self.mass_elements_: list[MassElement] = []
        self.spring_elements_: list[SpringElement] = []

    def SetGravity(self, x: float, y: float, z: float) -> None:
        self.gravity_ = [float(x), float(y), float(z)]

    # nodes
    def AddNode(self) -> NodeBuilder:
        self.nodes_.append(Node(len(self.nodes_)))
        return NodeBuilder(self.nodes_[-1])

    def GetNode(self, i: int) -> Node:
        return self.nodes_[i]

    def NumNodes(self) -> int:
        return len(self.nodes_)

    # beams
    def AddBeamElement(self, node_ids, sections, quadrature) -> int:
        eid = len(self.beam_elements_)
        self.beam_elements_.append(
            BeamElement(eid, [int(i) for i in node_ids], list(sections),
                        [[float(q[0]), float(q[1])] for q in quadrature]))
        return eid

    def GetBeamElements(self) -> list[BeamElement]:
        return self.beam_elements_

    def NumBeamElements(self) -> int:
        return len(self.beam_elements_)

    def TranslateBeam(self, eid: int, d: Sequence[float]) -> None:
        for n in self.beam_elements_[eid].node_ids:
            self.nodes_[n].Translate(d)

    def RotateBeamAboutPoint(self, eid: int, q: Sequence[float], point: Sequence[float]) -> None:
        for n in self.beam_elements_[eid].node_ids:
            self.nodes_[n].RotateAboutPoint(q, point)

    def SetBeamVelocityAboutPoint(self, eid: int, velocity, point) -> None:
        for n in self.beam_elements_[eid].node_ids:
            self.nodes_[n].SetVelocityAboutPoint(velocity, point)

    # point masses and springs
    def AddMassElement(self, node_id: int, mass) -> int:
        """src/model/model.hpp:305-311: a 6x6 mass matrix (material frame) at a node."""
        eid = len(self.mass_elements_)
        self.mass_elements_.append(MassElement(eid, int(node_id), np.asarray(mass, dtype=np.float64)
                                               .reshape(6, 6)))
        return eid

    def GetMassElements(self) -> list["MassElement"]:
        return self.mass_elements_

    def NumMassElements(self) -> int:
        return len(self.mass_elements_)

    def AddSpringElement(self, node1_id: int, node2_id: int, stiffness: float,
                         undeformed_length: float) -> int:
        """src/model/model.hpp:376-389: a translational spring between two nodes."""
        eid = len(self.spring_elements_)
        self.spring_elements_.append(SpringElement(eid, (int(node1_id), int(node2_id)),
                                                   float(stiffness), float(undeformed_length)))
        return eid

    def GetSpringElements(self) -> list["SpringElement"]:
        return self.spring_elements_

    def NumSpringElements(self) -> int:
        return len(self.spring_elements_)

    # constraints
    def AddFixedBC(self, node_id: int) -> int:
        cid = len(self.constraints_)
        self.constraints_.append(Constraint(cid, FIXED_BC, (INVALID_NODE_ID, int(node_id))))
        return cid

    def AddPrescribedBC(self, node_id: int,
                        initial_displacement=(0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0)) -> int:
        cid = len(self.constraints_)
        self.constraints_.append(Constraint(cid, PRESCRIBED_BC, (INVALID_NODE_ID, int(node_id)),
                                            (0.0, 0.0, 0.0),
                                            tuple(float(x) for x in initial_displacement)))
        return cid

    def AddFixedBC3DOFs(self, node_id: int) -> int:
        """src/model/model.hpp:570-583: fixes the position of a position-only node."""
        cid = len(self.constraints_)
        self.constraints_.append(Constraint(cid, FIXED_BC_3DOF, (INVALID_NODE_ID, int(node_id))))
        return cid

    def AddPrescribedBC3DOFs(self, node_id: int,
                             initial_displacement=(0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0)) -> int:
        """src/model/model.hpp:585-597: prescribes the position of a position-only node."""
        cid = len(self.constraints_)
        self.constraints_.append(Constraint(cid, PRESCRIBED_BC_3DOF, (INVALID_NODE_ID, int(node_id)),
                                            (0.0, 0.0, 0.0),
                                            tuple(float(x) for x in initial_displacement)))
        return cid

    def AddRigidJoint6DOFsTo3DOFs(self, node_ids) -> int:
        """src/model/model.hpp:599-611 AddRigidJoint6DOFsTo3DOFs({base, target}):
        a position-only target carried rigidly by a six-DOF base."""
        cid = len(self.constraints_)
        self.constraints_.append(Constraint(cid, RIGID_JOINT_6DOF_TO_3DOF, (int(node_ids[0]), int(node_ids[1]))))
        return cid

    def AddRigidJointConstraint(self, node_ids) -> int:
        """src/model/model.hpp AddRigidJointConstraint({base, target})."""
        cid = len(self.constraints_)
        self.constraints_.append(Constraint(cid, RIGID_JOINT, (int(node_ids[0]), int(node_ids[1]))))
        return cid

    def AddRotationControl(self, node_ids, axis, control=None) -> int:
        """src/model/model.hpp:550-562 AddRotationControl({base, target}, axis,
        control).  `control` stands for the reference's double*: any object
        that float() reads (a one-element array, for instance); its value at
        each step is the commanded angle.  Context.set_control(model_id,
        constraint_id, angle) passes it to a created model."""
        cid = len(self.constraints_)
        self.constraints_.append(Constraint(cid, ROTATION_CONTROL, (int(node_ids[0]), int(node_ids[1])),
                                            tuple(float(x) for x in axis)))
        self.controls_[cid] = control
        return cid

    def AddRevoluteJointConstraint(self, node_ids, axis, torque=None) -> int:
        """src/model/model.hpp:529-541 AddRevoluteJointConstraint({base, target},
        axis, torque): the target turns freely about `axis` (a zero axis takes
        the base-to-target direction).  `torque` stands for the reference's
        double*, read like a RotationControl's control before each step;
        Context.set_control(model_id, constraint_id, torque) passes it to a
        created model."""
        cid = len(self.constraints_)
        self.constraints_.append(Constraint(cid, REVOLUTE_JOINT, (int(node_ids[0]), int(node_ids[1])),
                                            tuple(float(x) for x in axis)))
        self.controls_[cid] = torque
        return cid

    def Controls(self) -> dict:
        """Constraint id -> control object of the RotationControl and
        RevoluteJoint constraints."""
        return dict(self.controls_)

    def NumConstraints(self) -> int:
        return len(self.constraints_)

    # packing
    def to_arrays(self) -> dict:
        nn = len(self.nodes_)
        f64 = np.float64
        a = {
            "node_x0": np.array([n.x0 for n in self.nodes_], dtype=f64).reshape(nn, 7),
            "node_u": np.array([n.u for n in self.nodes_], dtype=f64).reshape(nn, 7),
            "node_v": np.array([n.v for n in self.nodes_], dtype=f64).reshape(nn, 6),
            "node_vd": np.array([n.vd for n in self.nodes_], dtype=f64).reshape(nn, 6),
            "node_s": np.array([n.s for n in self.nodes_], dtype=f64),
        }
        bno, bni, bso, sp, sm, ss, bqo, qx, qw = [0], [], [0], [], [], [], [0], [], []
        for b in self.beam_elements_:
            bni.extend(b.node_ids)
            bno.append(len(bni))
            for s in b.sections:
                sp.append(s.position)
                sm.append(s.M_star.reshape(36))
                ss.append(s.C_star.reshape(36))
            bso.append(len(sp))
            for q in b.quadrature:
                qx.append(q[0])
                qw.append(q[1])
            bqo.append(len(qx))
        i32 = np.int32
        a.update({
            "beam_node_offsets": np.array(bno, dtype=i32),
            "beam_node_ids": np.array(bni, dtype=i32),
            "beam_section_offsets": np.array(bso, dtype=i32),
            "section_position": np.array(sp, dtype=f64),
            "section_mass": np.array(sm, dtype=f64).reshape(-1, 36),
            "section_stiffness": np.array(ss, dtype=f64).reshape(-1, 36),
            "beam_qp_offsets": np.array(bqo, dtype=i32),
            "qp_xi": np.array(qx, dtype=f64),
            "qp_weight": np.array(qw, dtype=f64),
        })
        nc = len(self.constraints_)
        a.update({
            "constraint_type": np.array([c.type for c in self.constraints_], dtype=i32),
            "constraint_base_node": np.array([c.node_ids[0] for c in self.constraints_], dtype=i32),
            "constraint_target_node": np.array([c.node_ids[1] for c in self.constraints_],
                                               dtype=i32),
            "constraint_axis": np.array([c.axis_vector for c in self.constraints_],
                                        dtype=f64).reshape(nc, 3),
            "constraint_initial_displacement": np.array(
                [c.initial_displacement for c in self.constraints_], dtype=f64).reshape(nc, 7),
        })
        a.update({
            "mass_node": np.array([m.node_id for m in self.mass_elements_], dtype=i32),
            "mass_matrix": np.array([m.mass for m in self.mass_elements_],
                                    dtype=f64).reshape(-1, 36),
            "spring_nodes": np.array([s.node_ids for s in self.spring_elements_],
                                     dtype=i32).reshape(-1, 2),
            "spring_stiffness": np.array([s.stiffness for s in self.spring_elements_], dtype=f64),
            "spring_length": np.array([s.undeformed_length for s in self.spring_elements_],
                                      dtype=f64),
        })
        for k in a:
            a[k] = np.ascontiguousarray(a[k])
        return a

    def pack(self) -> PackedModel:
        return PackedModel(self.to_arrays(), self.gravity_)
