"""Drive train with a revolute joint (test_rotating_beam.cpp:516-680): a blade
on a hub that turns freely about a shaft axis, held by a revolute joint from a
fixed shaft base, with or without an azimuth node between them and with a
generator torque.  The GPU path eliminates the shaft rotation from the beam's
system (second right-hand side, one projected equation); the oracle solves the
whole bordered system densely.  Same CRS graph, same Newton decisions, states
and multipliers within the parity tolerances, and the reference's golden
values."""
import math

import numpy as np
import pytest

from openturbine_b200.model import StepParameters
from oracle.oracle_py import OracleModel
from tests.test_gpu_hub import HubTwin
from tests.test_gpu_parity import FIELDS, assert_state_close
from tests.workloads_ref import generator_torque_model, load_golden, revolute_joint_test_model

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from openturbine_b200.runtime import Context
    c = Context(0)
    yield c
    c.close()


def _crs_equal(ctx, pm):
    mid = ctx.create_model(pm)
    rp, ci, _ = ctx.crs(mid, values=False)
    orp, oci, _ = OracleModel(pm).crs()
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    return mid


# Multipliers are reaction forces and moments: the beam's internal force at the
# root is the axial stiffness times a strain formed as a difference of O(1)
# terms, so any FP64 evaluation carries an absolute rounding floor of about
# EA x machine epsilon on them, whatever the summation order (the oracle's
# reversed-quadrature twin shares the per-point arithmetic and does not see it).
# With the 0.1 rad/s spin of the revolute test the reactions are ~5e-3, where
# that floor (EA = 1.368e6 N: 3e-10) dominates a relative bound.
EA = 1.36817e6
EPS = np.finfo(np.float64).eps


def assert_multipliers_close(ctx, mid, tw):
    lg, lo = ctx.state(mid, "lambda"), tw.state("lambda")
    tol = max(10.0 * tw.floor("lambda") * np.abs(lo).max(), 1e-10 * np.abs(lo).max(), 10.0 * EA * EPS)
    assert np.abs(lg - lo).max() <= tol, (np.abs(lg - lo).max(), tol)


def _run(ctx, mid, tw, p, rj, torque, steps):
    for _ in range(steps):
        ctx.set_control(mid, rj, torque)
        tw.set_prescribed(rj, [torque, 0., 0., 1., 0., 0., 0.])
        st, it = ctx.step([mid], p)
        ost, oit = tw.step(p)
        assert (st[0], it[0]) == (ost, oit) == (0, oit)
        gc, oc = ctx.convergence(mid), tw.convergence()
        assert len(gc) == len(oc)
        for a, b in zip(gc, oc):
            assert (a <= 1.0) == (b <= 1.0)
            if b > 1.0:
                assert abs(a - b) <= 1e-6 * b, (a, b)


def test_revolute_joint_matches_oracle_and_golden(ctx):
    """RevoluteJointConstraint: ground (fixed) -> revolute about z -> hub ->
    rigid joint -> blade root, zero torque, 5 steps; q of all 8 nodes against
    the golden values at the test's 1e-6."""
    g = load_golden("revolute_joint.json")["revolute"]
    m, p, rj = revolute_joint_test_model()
    pm = m.pack()
    mid = _crs_equal(ctx, pm)
    info = ctx.info(mid)
    assert info.num_dofs == 8 * 6 + 6 + 5 + 6
    tw = HubTwin(pm)
    _run(ctx, mid, tw, p, rj, 0.0, g["steps"])
    assert_state_close(ctx, mid, tw, fields=FIELDS, lam=False)
    assert_multipliers_close(ctx, mid, tw)
    np.testing.assert_allclose(ctx.state(mid, "q").ravel(), g["q"], rtol=0, atol=g["tolerance"])
    ctx.destroy_model(mid)


@pytest.mark.parametrize("key", ["tilt0", "tilt90"])
def test_generator_torque_matches_oracle_and_golden(ctx, key):
    """GeneratorTorque_Tilt0 / _Tilt90: shaft base (fixed) -> revolute about
    the tilted shaft -> azimuth -> rigid -> hub -> rigid -> blade root under a
    100 N m torque, 10 steps; azimuth q and v and the joint output (rotation,
    rate, acceleration about the shaft) against the golden values at 1e-6."""
    g = load_golden("revolute_joint.json")["generator_torque"]
    m, p, rj, az = generator_torque_model(0.0 if key == "tilt0" else math.pi / 2.)
    pm = m.pack()
    mid = _crs_equal(ctx, pm)
    tw = HubTwin(pm)
    _run(ctx, mid, tw, p, rj, g["torque"], g["steps"])
    assert_state_close(ctx, mid, tw, fields=FIELDS, lam=False)
    assert_multipliers_close(ctx, mid, tw)
    out = ctx.state(mid, "output")
    np.testing.assert_allclose(out, tw.o.state("output"), rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(ctx.state(mid, "q")[az], g[key]["azimuth_q"], rtol=0, atol=g["tolerance"])
    np.testing.assert_allclose(ctx.state(mid, "v")[az], g[key]["azimuth_v"], rtol=0, atol=g["tolerance"])
    np.testing.assert_allclose(out[rj], g[key]["output"], rtol=0, atol=g["tolerance"])
    ctx.destroy_model(mid)


def _three_blade_drive_train(with_azimuth: bool):
    """Three blades of the rotating-beam test at 120 degrees about z on a hub
    that turns on a revolute joint about z from a fixed shaft base (directly, or
    through an azimuth node rigidly holding the hub), spinning at 0.1 rad/s
    under a 50 N m torque: the beams form one cluster and share the shaft
    rotation."""
    from openturbine_b200.model import BeamSection, Model, RotationVectorToQuaternion, StepParameters
    from tests.workloads_ref import COMPOSITE_MASS, COMPOSITE_STIFF, GAUSS7, GLL6_S
    m = Model()
    m.SetGravity(0., 0., 0.)
    roots = []
    for b in range(3):
        ids = [m.AddNode().SetElemLocation(s).SetPosition(10 * s, 0., 0., 1., 0., 0., 0.).Build()
               for s in GLL6_S]
        e = m.AddBeamElement(ids, [BeamSection(0., COMPOSITE_MASS, COMPOSITE_STIFF),
                                   BeamSection(1., COMPOSITE_MASS, COMPOSITE_STIFF)], GAUSS7)
        m.TranslateBeam(e, [2.0, 0., 0.])
        m.RotateBeamAboutPoint(e, RotationVectorToQuaternion([0., 0., 2. * math.pi * b / 3.]), [0., 0., 0.])
        m.SetBeamVelocityAboutPoint(e, [0., 0., 0., 0., 0., 0.1], [0., 0., 0.])
        roots.append(ids[0])
    base = m.AddNode().SetPosition(0., 0., -1., 1., 0., 0., 0.).Build()
    az = m.AddNode().SetPosition(0., 0., -0.5, 1., 0., 0., 0.).Build() if with_azimuth else None
    hub = m.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build()
    m.AddFixedBC(base)
    rj = m.AddRevoluteJointConstraint([base, az if with_azimuth else hub], [0., 0., 1.], np.array([50.]))
    if with_azimuth:
        m.AddRigidJointConstraint([az, hub])
    for r in roots:
        m.AddRigidJointConstraint([hub, r])
    return m, StepParameters(True, 6, 0.01, 0.9), rj


@pytest.mark.parametrize("with_azimuth", [False, True])
def test_three_blade_drive_train_matches_oracle(ctx, with_azimuth):
    """Three blades in one cluster on a shared shaft: the CTAs sum their parts
    of the shaft equation in rank order; same CRS, Newton decisions, states and
    multipliers as the oracle's dense solve over 10 steps."""
    m, p, rj = _three_blade_drive_train(with_azimuth)
    pm = m.pack()
    mid = _crs_equal(ctx, pm)
    tw = HubTwin(pm)
    _run(ctx, mid, tw, p, rj, 50.0, 10)
    assert_state_close(ctx, mid, tw, fields=FIELDS, lam=False)
    assert_multipliers_close(ctx, mid, tw)
    np.testing.assert_allclose(ctx.state(mid, "output"), tw.o.state("output"), rtol=1e-10, atol=1e-12)
    ctx.destroy_model(mid)


def test_drive_train_restart_and_state_copy(ctx):
    """The drive-train records travel with the state: a copy made after 3
    steps and stepped 2 more matches the original stepped 2 more; so do a model
    read from the original's restart record and a clone, and the batched
    motion read returns the drive-train nodes' rows."""
    m, p, rj, _ = generator_torque_model(0.0)
    pm = m.pack()
    a = ctx.create_model(pm)
    b = ctx.create_model(pm)
    for _ in range(3):
        ctx.set_control(a, rj, 100.0)
        ctx.step([a], p)
    ctx.copy_state(b, a)
    for _ in range(2):
        for mid in (a, b):
            ctx.set_control(mid, rj, 100.0)
        st, _ = ctx.step([a, b], p)
        assert list(st) == [0, 0]
    for f in ("q", "v", "vd", "a", "lambda"):
        np.testing.assert_array_equal(ctx.state(a, f), ctx.state(b, f))
    # restart record round trip and clone: both continue like the original
    rec = ctx.write_restart(a)
    c = ctx.create_model(pm)
    ctx.read_restart(c, rec)
    d = ctx.clone_model(a)
    for _ in range(2):
        for mid in (a, c, d):
            ctx.set_control(mid, rj, 100.0)
        st, _ = ctx.step([a, c, d], p)
        assert list(st) == [0, 0, 0]
    for f in ("q", "v", "vd", "lambda"):
        np.testing.assert_array_equal(ctx.state(a, f), ctx.state(c, f))
        np.testing.assert_array_equal(ctx.state(a, f), ctx.state(d, f))
    # the batched motion read carries the drive-train nodes' rows too
    n = ctx.info(a).num_nodes
    q = np.zeros((2, n, 7))
    ctx.get_state_batch(np.array([a, c], dtype=np.int32), "q", q.ctypes.data, False)
    np.testing.assert_array_equal(q[0], ctx.state(a, "q"))
    np.testing.assert_array_equal(q[1], ctx.state(c, "q"))
    for mid in (a, b, c, d):
        ctx.destroy_model(mid)


def test_drive_trains_batched_with_beams(ctx):
    """Drive-train models batched with plain cantilevers and hub rotors in one
    step call (one launch bucket per instance and size class): every model's
    state equals the state it reaches stepped alone."""
    from openturbine_b200 import workloads as W
    from tests.workloads_ref import rotation_control_test_model
    specs = [("gen", generator_torque_model(0.0)), ("three", _three_blade_drive_train(True)),
             ("rev", revolute_joint_test_model())]
    beams = [W.batch_cantilever_model(d) for d in W.draw_batch(6, first_id=900)]
    rc_model, rc_p, rc, _ = rotation_control_test_model(False)
    p = W.batch_params(6)

    def build():
        ids, ctl = [], []
        for _, sp in specs:
            ids.append(ctx.create_model(sp[0].pack()))
            ctl.append(sp[2])
        for b in beams:
            ids.append(ctx.create_model(b.pack()))
        ids.append(ctx.create_model(rc_model.pack()))
        return ids, ctl

    def advance(ids, ctl, k, together):
        for mid, cid in zip(ids, ctl):
            ctx.set_control(mid, cid, 20.0)
        ctx.set_control(ids[-1], rc, 0.01 * (k + 1))
        if together:
            return list(ctx.step(ids, p)[0])
        return [int(ctx.step([mid], p)[0][0]) for mid in ids]

    a_ids, ctl = build()
    b_ids, _ = build()
    for k in range(4):
        sa = advance(a_ids, ctl, k, True)
        sb = advance(b_ids, ctl, k, False)
        assert sa == sb
    for ia, ib in zip(a_ids, b_ids):
        for f in ("q", "v", "lambda"):
            np.testing.assert_array_equal(ctx.state(ia, f), ctx.state(ib, f))
    for mid in a_ids + b_ids:
        ctx.destroy_model(mid)


def test_drive_train_fp32_form_close_to_fp64(ctx):
    """The FP32 form (FP32 tangent and LU, FP64 residual and update) on the
    generator-torque drive train: same convergence, azimuth rotation and joint
    output within 1e-8 of the FP64 form."""
    m, p, rj, az = generator_torque_model(0.0)
    pm = m.pack()
    a = ctx.create_model(pm)
    b = ctx.create_model(pm)
    p32 = StepParameters(p.is_dynamic_solve, p.max_iter, p.h, p.rho_inf, p.absolute_convergence_tol,
                         p.relative_convergence_tol, precision=1, refine_iters=1)
    for _ in range(10):
        for mid in (a, b):
            ctx.set_control(mid, rj, 100.0)
        sa, _ = ctx.step([a], p)
        sb, _ = ctx.step([b], p32)
        assert sa[0] == sb[0] == 0
    qa, qb = ctx.state(a, "q"), ctx.state(b, "q")
    assert np.abs(qa - qb).max() <= 1e-8 * np.abs(qa).max()
    oa, ob = ctx.state(a, "output")[rj], ctx.state(b, "output")[rj]
    assert np.abs(oa - ob).max() <= 1e-8 * np.abs(oa).max()
    ctx.destroy_model(a)
    ctx.destroy_model(b)

