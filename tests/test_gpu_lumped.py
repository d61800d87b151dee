"""Point masses and springs on the GPU path: models without beam elements (one
dense system over all nodes) and beams carrying masses, against the oracle and
the reference's golden values (test_masses.cpp, test_precession.cpp,
test_spring_mass_system.cpp)."""
import numpy as np
import pytest

from oracle.oracle_py import OracleModel
from tests.test_gpu_parity import (ACCEL_REL, FIELDS, Twin, assert_convergence_close,
                                   assert_state_close)
from tests.workloads_ref import (cantilever_test_loads, cantilever_test_model,
                                 load_golden, mass_external_force_model, precession_model,
                                 spring_mass_chain_model, spring_mass_model)

pytestmark = pytest.mark.gpu


class LumpedTwin(Twin):
    """The oracle with the dense solve of the whole system, twice (no
    quadrature, so the second run is the same order: floor 0)."""

    def __init__(self, pm):
        self.o = OracleModel(pm)
        self.alt = OracleModel(pm, solver_mode=2)
        self.info = self.o.info

    def set_state_f(self, f):
        self.o.set_state_f(f)
        self.alt.set_state_f(f)


@pytest.fixture(scope="module")
def ctx():
    from openturbine_b200.runtime import Context
    c = Context(0)
    yield c
    c.close()


def _run(ctx, m, p, steps, f=None, check=None):
    pm = m.pack()
    mid = ctx.create_model(pm)
    rp, ci, _ = ctx.crs(mid, values=False)
    tw = LumpedTwin(pm)
    orp, oci, _ = tw.crs()
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    if f is not None:
        ctx.set_state_f(mid, f)
        tw.set_state_f(f)
    for k in range(steps):
        st, it = ctx.step([mid], p)
        ost, oit = tw.step(p)
        assert (st[0], it[0]) == (ost, oit) == (0, oit)
        assert_convergence_close(ctx.convergence(mid), tw.convergence())
        if check:
            check(k + 1, ctx.state(mid, "q"))
    assert_state_close(ctx, mid, tw, fields=FIELDS)
    return mid


def test_mass_external_force(ctx):
    g = load_golden("masses_springs.json")["mass_external_force"]
    m, p, f = mass_external_force_model()
    mid = _run(ctx, m, p, g["steps"], f=f)
    np.testing.assert_allclose(ctx.state(mid, "v")[0], g["v"], rtol=0, atol=g["tolerance"])
    ctx.destroy_model(mid)


def test_precession(ctx):
    g = load_golden("masses_springs.json")["precession"]
    m, p = precession_model()
    mid = _run(ctx, m, p, g["steps"])
    np.testing.assert_allclose(ctx.state(mid, "q")[0], g["q"], rtol=0, atol=g["tolerance"])
    ctx.destroy_model(mid)


def test_spring_mass_oscillation(ctx):
    g = load_golden("masses_springs.json")["spring_mass"]
    m, p = spring_mass_model()

    def check(step, q):
        if step == g["steps"] // 2:
            assert abs(q[1, 0] - g["q1x_half"]) <= g["tolerance"]
        if step == g["steps"]:
            assert abs(q[1, 0] - g["q1x_end"]) <= g["tolerance"]
    mid = _run(ctx, m, p, g["steps"], check=check)
    ctx.destroy_model(mid)


def test_spring_mass_chain_equilibrium(ctx):
    g = load_golden("masses_springs.json")["spring_mass_chain"]
    m, p = spring_mass_chain_model()

    def check(step, q):
        assert np.abs(q[:, 0]).max() <= g["tolerance"]
    mid = _run(ctx, m, p, 50, check=check)
    ctx.destroy_model(mid)


def test_cantilever_with_tip_mass_and_gravity(ctx):
    """A point mass (with an offset centre of mass) at the tip of the cantilever
    of test_cantilever_beam.cpp, gravity on: the beam kernel adds the mass's
    terms to the tip's block row; same Newton decisions and states as the oracle."""
    from tests.test_gpu_parity import Twin as BeamTwin
    m, p = cantilever_test_model()
    m.SetGravity(0., 0., -9.81)
    mm = np.diag([5., 5., 5., 0.2, 0.3, 0.4])
    mm[0, 4] = mm[4, 0] = 0.1   # m * eta coupling
    m.AddMassElement(4, mm)
    pm = m.pack()
    mid = ctx.create_model(pm)
    rp, ci, _ = ctx.crs(mid, values=False)
    tw = BeamTwin(pm)
    orp, oci, _ = tw.crs()
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    for k in range(20):
        fx = cantilever_test_loads(k)
        ctx.set_node_fx(mid, fx)
        tw.set_node_fx(fx)
        st, it = ctx.step([mid], p)
        ost, oit = tw.step(p)
        assert (st[0], it[0]) == (ost, oit)
        # Same Newton decisions, and equal norms while the correction is larger
        # than the tolerance.  A converged norm (here ~1e-2) measures a correction
        # from a residual in which the tip weight and the internal forces cancel;
        # the GPU's elimination and blocked LU round it differently from the
        # oracle's pivoted LU (2e-5 relative at 0.0128), while the states agree
        # to 1e-15.
        g, o = ctx.convergence(mid), tw.convergence()
        assert len(g) == len(o)
        for x, y in zip(g, o):
            assert (x <= 1.0) == (y <= 1.0)
            if y > 1.0:
                assert abs(x - y) <= 1e-6 * y, (x, y)
    assert_state_close(ctx, mid, tw, fields=FIELDS)
    ctx.destroy_model(mid)


def test_lumped_models_batched_with_beams(ctx):
    """Spring-mass models stepped in the same kyn_step call as beams advance
    exactly as they do alone."""
    from openturbine_b200 import workloads as W
    m, p = spring_mass_model()
    pm = m.pack()
    alone = ctx.create_model(pm)
    mixed = [ctx.create_model(pm) for _ in range(3)]
    draws = W.draw_batch(8, first_id=900)
    beams = [ctx.create_model(W.batch_cantilever_model(d).pack()) for d in draws]
    ids = np.array(mixed[:1] + beams[:4] + mixed[1:] + beams[4:], dtype=np.int32)
    for _ in range(30):
        st, _ = ctx.step([alone], p)
        st2, _ = ctx.step(ids, p)
        assert st[0] == 0
    qa = ctx.state(alone, "q")
    for mid in mixed:
        np.testing.assert_array_equal(ctx.state(mid, "q"), qa)
    for mid in [alone] + mixed + beams:
        ctx.destroy_model(mid)


def test_heavy_top_dense_model(ctx):
    """test_heavy_top.cpp:9-75: a top held at a point by a rigid joint to a
    position-only ground node with a prescribed position (RigidJoint6DOFsTo3DOFs,
    PrescribedBC3DOFs; 15 DOFs).  The model runs as its dense bordered system
    (one CTA, pivoted LU): same CRS, Newton decisions and states as the oracle
    over 400 steps, and the golden q at the test's 1e-10."""
    from tests.workloads_ref import heavy_top_model
    g = load_golden("heavy_top.json")
    m, p, _ = heavy_top_model()
    pm = m.pack()
    mid = ctx.create_model(pm)
    assert ctx.info(mid).num_dofs == 15
    rp, ci, _ = ctx.crs(mid, values=False)
    tw = LumpedTwin(pm)
    orp, oci, _ = tw.crs()
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    for _ in range(g["steps"]):
        st, it = ctx.step([mid], p)
        ost, oit = tw.step(p)
        assert (st[0], it[0]) == (ost, oit) == (0, oit)
        # The top spins at 150 rad/s: a step's first correction is ~1e8 times its
        # last, so rounding in the first (1e-16 of it) reaches the later error
        # norms; they are compared to 1e-12 of the step's largest norm.
        gc, oc = ctx.convergence(mid), tw.convergence()
        assert len(gc) == len(oc)
        for a, b in zip(gc, oc):
            assert (a <= 1.0) == (b <= 1.0)
            assert abs(a - b) <= max(1e-6 * b, 1e-12 * max(oc)), (a, b)
    assert_state_close(ctx, mid, tw, fields=FIELDS, lam=False)
    # The multipliers are unconditioned by 1/(beta h^2) ~ 8e5 at h = 0.002, the
    # amplification the accelerations see: they are held to the same 1e-7 bound
    # as vd and a (the run measures ~2e-10).
    lg, lo = ctx.state(mid, "lambda"), tw.state("lambda")
    assert np.abs(lg - lo).max() <= ACCEL_REL * np.abs(lo).max()
    np.testing.assert_allclose(ctx.state(mid, "q")[0], g["q_mass_node"], rtol=0, atol=g["tolerance"])
    ctx.destroy_model(mid)


def test_dense_models_batched_with_beams_and_fp32_form(ctx):
    """Dense models (heavy tops) stepped in the same kyn_step call as beams
    and spring-mass models advance exactly as they do alone, in both
    precision forms (dense models compute in FP64 in either)."""
    from openturbine_b200 import workloads as W
    from tests.workloads_ref import heavy_top_model
    m, p, _ = heavy_top_model()
    sm, _ = spring_mass_model()
    pm = m.pack()
    for precision in (0, 1):
        pp = type(p)(p.is_dynamic_solve, p.max_iter, p.h, p.rho_inf, p.absolute_convergence_tol,
                     p.relative_convergence_tol, precision=precision)
        alone = ctx.create_model(pm)
        mixed = [ctx.create_model(pm) for _ in range(2)]
        others = [ctx.create_model(sm.pack())] + [
            ctx.create_model(W.batch_cantilever_model(d).pack()) for d in W.draw_batch(4, first_id=950)]
        ids = np.array(mixed[:1] + others[:3] + mixed[1:] + others[3:], dtype=np.int32)
        for _ in range(20):
            st, _ = ctx.step([alone], pp)
            ctx.step(ids, pp)
            assert st[0] == 0
        for mid in mixed:
            for f in ("q", "v", "lambda"):
                np.testing.assert_array_equal(ctx.state(mid, f), ctx.state(alone, f))
        for mid in [alone] + mixed + others:
            ctx.destroy_model(mid)


def test_cfd_floating_platform_models(ctx):
    """The CFD interface's platform models (test_cfd_interface.cpp): the
    spinning platform (mass only, the beam-free lumped path, 600 steps) and the
    moored platform (three position-only fairleads and anchors, six three-row
    constraints: a dense model of 42 DOFs, 101 steps under the test's loads).
    Same Newton decisions and states as the oracle, goldens at 1e-12."""
    from tests.workloads_ref import cfd_platform_loads, cfd_platform_model
    g = load_golden("cfd_platform.json")
    m, p, plat = cfd_platform_model(False)
    mid = _run(ctx, m, p, 600)
    np.testing.assert_allclose(ctx.state(mid, "q")[plat], g["precession"]["q_600"], rtol=0, atol=1e-12)
    ctx.destroy_model(mid)

    m, p, plat = cfd_platform_model(True)
    pm = m.pack()
    mid = ctx.create_model(pm)
    assert ctx.info(mid).num_dofs == 42
    rp, ci, _ = ctx.crs(mid, values=False)
    tw = LumpedTwin(pm)
    orp, oci, _ = tw.crs()
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    f = np.zeros((ctx.info(mid).num_nodes, 6))
    for i in range(g["floating_platform"]["step"] + 1):
        f[plat] = cfd_platform_loads(i)
        ctx.set_state_f(mid, f)
        tw.set_state_f(f)
        st, it = ctx.step([mid], p)
        ost, oit = tw.step(p)
        assert (st[0], it[0]) == (ost, oit) == (0, oit)
    assert_state_close(ctx, mid, tw, fields=FIELDS, lam=False)
    lg, lo = ctx.state(mid, "lambda"), tw.state("lambda")
    assert np.abs(lg - lo).max() <= ACCEL_REL * np.abs(lo).max()
    np.testing.assert_allclose(ctx.state(mid, "q")[plat], g["floating_platform"]["q"], rtol=0, atol=1e-12)
    ctx.destroy_model(mid)


def test_dense_model_with_six_row_joints(ctx):
    """Beam-free models whose nodes are joined by six-row joints run as dense
    models: a spinning body (mass B) carried by a RigidJoint from a body (mass
    A) that hangs from a fixed, position-only pivot (RigidJoint6DOFsTo3DOFs +
    FixedBC3DOFs), and the same with the rigid joint replaced by a
    RotationControl turning B about the joint axis.  Same CRS, Newton
    decisions and states as the oracle over 60 steps."""
    from openturbine_b200.model import Model, StepParameters
    for control in (False, True):
        m = Model()
        m.SetGravity(0., 0., -9.81)
        a = m.AddNode().SetPosition(0., 1., 0., 1., 0., 0., 0.).SetVelocity(0., 0., 0., 0., 0., 2.).Build()
        b = m.AddNode().SetPosition(0., 2., 0., 1., 0., 0., 0.).SetVelocity(-2., 0., 0., 0., 0., 2.).Build()
        pivot = m.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build()
        m.AddMassElement(a, np.diag([5., 5., 5., 0.2, 0.1, 0.2]))
        m.AddMassElement(b, np.diag([2., 2., 2., 0.05, 0.05, 0.08]))
        m.AddRigidJoint6DOFsTo3DOFs([a, pivot])
        m.AddFixedBC3DOFs(pivot)
        rc = (m.AddRotationControl([a, b], [0., 1., 0.]) if control else m.AddRigidJointConstraint([a, b]))
        p = StepParameters(True, 8, 0.005, 0.8, a_tol=1e-6, r_tol=1e-3)
        pm = m.pack()
        mid = ctx.create_model(pm)
        assert ctx.info(mid).num_dofs == 6 + 6 + 3 + 3 + 3 + 6
        rp, ci, _ = ctx.crs(mid, values=False)
        tw = LumpedTwin(pm)
        orp, oci, _ = tw.crs()
        assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
        for k in range(60):
            if control:
                ang = 0.5 * 0.005 * (k + 1)
                ctx.set_control(mid, rc, ang)
                tw.set_prescribed(rc, [ang, 0., 0., 1., 0., 0., 0.])
            st, it = ctx.step([mid], p)
            ost, oit = tw.step(p)
            assert (st[0], it[0]) == (ost, oit) == (0, oit)
        assert_state_close(ctx, mid, tw, fields=FIELDS, lam=False)
        lg, lo = ctx.state(mid, "lambda"), tw.state("lambda")
        assert np.abs(lg - lo).max() <= ACCEL_REL * np.abs(lo).max()
        ctx.destroy_model(mid)
