"""Seeded synthetic workloads for the beam path.

No public dataset or benchmark suite is involved; these generators build the
named configurations from seeded numpy streams (global seed 20261203, one
stream per model id):

* ``cantilever_model`` -- single cantilever: straight beam along x, L = 10 m,
  one element of order 4 (5 GLL nodes), 7-point Gauss quadrature, uniform
  section C* = diag(1e9, 4e8, 4e8, 1e7, 2e7, 2e7), M* = diag(10,10,10,2,1,1),
  clamped root, tip force Fz = 1e4 sin(2 pi t).
* ``rotor_model`` -- three 60 m blades (11 GLL nodes, 21 stations, 21-point
  trapezoidal quadrature), sections tapered 10x root to tip with seeded
  perturbations and SPD couplings, hub prescribed rotation 0.8 rad/s, gravity.
* ``batch_cantilevers`` -- N cantilevers with nodes U{5..21}, Gauss points
  nodes+2, length U(5, 100) m, rotor-style sections, tip load amplitude
  U(1e3, 1e5) N and frequency U(0.1, 5) Hz.
* ``precision_cantilever_model`` -- the same batch with the bending and
  torsion stiffness of each beam scaled log-uniformly in [0.1, 100] (EA/EI
  swept), for the accuracy report of the FP32 form.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .model import (BeamSection, CreateTrapezoidalQuadrature, GaussLegendreQuadrature,
                    GenerateGLLPoints, Model, QuaternionCompose, RotateVectorByQuaternion,
                    RotationVectorToQuaternion, StepParameters)

GLOBAL_SEED = 20261203
BASE_STIFFNESS = np.diag([1e9, 4e8, 4e8, 1e7, 2e7, 2e7])
BASE_MASS = np.diag([10.0, 10.0, 10.0, 2.0, 1.0, 1.0])


def rng_for(model_id: int) -> np.random.Generator:
    return np.random.default_rng(np.random.SeedSequence([GLOBAL_SEED, int(model_id)]))


def gll_node_locations(num_nodes: int) -> list[float]:
    return [(x + 1.0) / 2.0 for x in GenerateGLLPoints(num_nodes - 1)]


def perturbed_section(base: np.ndarray, scale: float, rng: np.random.Generator) -> np.ndarray:
    """Diagonal x (1 + U(-0.05, 0.05)); symmetric couplings N(0, 0.05 sqrt(Kii Kjj)),
    redrawn until symmetric positive definite."""
    for _ in range(100):
        d = np.diag(base) * scale * (1.0 + rng.uniform(-0.05, 0.05, 6))
        K = np.diag(d)
        for i in range(6):
            for j in range(i + 1, 6):
                K[i, j] = K[j, i] = rng.normal(0.0, 0.05 * math.sqrt(d[i] * d[j]))
        if np.linalg.eigvalsh(K).min() > 0.0:
            return K
    raise RuntimeError("could not draw an SPD section")


def tapered_sections(rng: np.random.Generator, stations: int = 21,
                     stiffness_scale: float = 1.0) -> list[BeamSection]:
    out = []
    for k in range(stations):
        s = k / (stations - 1)
        taper = 1.0 - 0.9 * s  # linear, 10x smaller at the tip
        K = perturbed_section(BASE_STIFFNESS * np.diag([1, 1, 1, stiffness_scale,
                                                        stiffness_scale, stiffness_scale]),
                              taper, rng)
        M = perturbed_section(BASE_MASS, taper, rng)
        out.append(BeamSection(s, M, K))
    return out


# ---- config: single cantilever -------------------------------------------------
def cantilever_model(num_nodes: int = 5, length: float = 10.0, num_qps: int = 7):
    m = Model()
    ids = [m.AddNode().SetElemLocation(s).SetPosition(length * s, 0., 0., 1., 0., 0., 0.).Build()
           for s in gll_node_locations(num_nodes)]
    sec = [BeamSection(0.0, BASE_MASS, BASE_STIFFNESS), BeamSection(1.0, BASE_MASS, BASE_STIFFNESS)]
    m.AddBeamElement(ids, sec, GaussLegendreQuadrature(num_qps))
    m.AddFixedBC(ids[0])
    return m


def cantilever_params(max_iter: int = 10) -> StepParameters:
    return StepParameters(True, max_iter, 0.01, 0.9, a_tol=1e-7, r_tol=1e-3)


def cantilever_tip_load(step: int, h: float = 0.01, amp: float = 1e4, freq: float = 1.0) -> float:
    return amp * math.sin(2.0 * math.pi * freq * h * (step + 1))


# ---- config: three-blade rotor ---------------------------------------------------
@dataclass
class RotorSpec:
    blade_length: float = 60.0
    hub_radius: float = 2.0
    num_nodes: int = 11
    stations: int = 21
    omega: float = 0.8


def rotor_model(model_id: int = 0, spec: RotorSpec = RotorSpec()):
    rng = rng_for(model_id)
    m = Model()
    m.SetGravity(0.0, 0.0, -9.81)
    node_s = gll_node_locations(spec.num_nodes)
    grid = [k / (spec.stations - 1) for k in range(spec.stations)]
    quad = CreateTrapezoidalQuadrature(grid)
    sections = tapered_sections(rng, spec.stations)
    velocity = [0.0, 0.0, 0.0, 0.0, 0.0, spec.omega]
    roots = []
    for b in range(3):
        ids = [m.AddNode().SetElemLocation(s)
               .SetPosition(spec.hub_radius + spec.blade_length * s, 0., 0., 1., 0., 0., 0.).Build()
               for s in node_s]
        e = m.AddBeamElement(ids, sections, quad)
        q = RotationVectorToQuaternion([0.0, 0.0, 2.0 * math.pi * b / 3.0])
        m.RotateBeamAboutPoint(e, q, [0.0, 0.0, 0.0])
        m.SetBeamVelocityAboutPoint(e, velocity, [0.0, 0.0, 0.0])
        roots.append(ids[0])
    bcs = [m.AddPrescribedBC(r) for r in roots]
    return m, bcs


def rotor_root_inputs(model: Model, bcs, step: int, h: float = 0.01, omega: float = 0.8):
    """Prescribed root displacement: u = R_hub x0_root - x0_root, q = exp(omega t z)."""
    q = RotationVectorToQuaternion([0.0, 0.0, omega * h * (step + 1)])
    out = []
    for c in bcs:
        node = model.GetNode(model.constraints_[c].node_ids[1])
        x0 = node.x0[:3]
        xr = RotateVectorByQuaternion(q, x0)
        out.append([xr[0] - x0[0], xr[1] - x0[1], xr[2] - x0[2], *q])
    return out


def rotor_params() -> StepParameters:
    return StepParameters(True, 10, 0.01, 0.9)


# ---- config: batch of uneven cantilevers ---------------------------------------------
@dataclass
class BeamDraw:
    model_id: int
    num_nodes: int
    length: float
    amp: float
    freq: float


def draw_batch(n: int, first_id: int = 0) -> list[BeamDraw]:
    out = []
    for i in range(first_id, first_id + n):
        r = rng_for(i)
        out.append(BeamDraw(i, int(r.integers(5, 22)), float(r.uniform(5.0, 100.0)),
                            float(r.uniform(1e3, 1e5)), float(r.uniform(0.1, 5.0))))
    return out


def batch_cantilever_model(d: BeamDraw, stiffness_scale: float = 1.0) -> Model:
    rng = rng_for(d.model_id + 1_000_000)
    m = Model()
    ids = [m.AddNode().SetElemLocation(s).SetPosition(d.length * s, 0., 0., 1., 0., 0., 0.).Build()
           for s in gll_node_locations(d.num_nodes)]
    m.AddBeamElement(ids, tapered_sections(rng, 21, stiffness_scale),
                     GaussLegendreQuadrature(d.num_nodes + 2))
    m.AddFixedBC(ids[0])
    return m


def precision_scale(d: BeamDraw) -> float:
    """Stiffness scale of the rotational (torsion and bending) block of beam d in
    the precision batch: log-uniform in [0.1, 100], so that EA/EI sweeps three
    decades and the conditioned tangent of the first Newton iteration spans
    ~2e7..3e9 (tests/test_workloads.py measures it on the oracle)."""
    return float(10.0 ** rng_for(d.model_id + 2_000_000).uniform(-1.0, 2.0))


def precision_cantilever_model(d: BeamDraw) -> Model:
    """The batch cantilever of draw d with its EI scaled by precision_scale(d)."""
    return batch_cantilever_model(d, stiffness_scale=precision_scale(d))


def batch_params(max_iter: int = 10) -> StepParameters:
    return StepParameters(True, max_iter, 0.01, 0.9, a_tol=1e-7, r_tol=1e-3)


def tip_loads(draws: list[BeamDraw], step: int, h: float = 0.01) -> np.ndarray:
    t = h * (step + 1)
    return np.array([d.amp * math.sin(2.0 * math.pi * d.freq * t) for d in draws])


def node_fx_for(d: BeamDraw, fz: float) -> np.ndarray:
    fx = np.zeros((d.num_nodes, 6))
    fx[-1, 2] = fz
    return fx
