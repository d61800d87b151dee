"""Rotor with a hub: blade roots rigidly jointed to a hub node that follows a
prescribed rotation (test_rotor.cpp:191-243, IEA15RotorHub), against the
oracle, which assembles the rigid joints' base- and target-node blocks into
the full bordered system and solves it densely."""
import numpy as np
import pytest

from oracle.oracle_py import OracleModel
from tests.test_gpu_parity import FIELDS, Twin, assert_state_close
from tests.workloads_ref import iea15_hub_displacement, iea15_hub_rotor_model, load_golden

pytestmark = pytest.mark.gpu


class HubTwin(Twin):
    """The oracle twice, both with the dense solve of the whole system (the
    single-node elimination of the other twin does not apply to joints); the
    second sums the quadrature in reverse order (rounding-noise floor)."""

    def __init__(self, pm):
        self.o = OracleModel(pm)
        self.alt = OracleModel(pm, solver_mode=2)
        self.info = self.o.info


@pytest.fixture(scope="module")
def ctx():
    from openturbine_b200.runtime import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def golden():
    return load_golden("iea15_rotor.json")


def test_hub_rotor_crs_graph_bit_exact(ctx, golden):
    m, _, _, _ = iea15_hub_rotor_model(golden)
    pm = m.pack()
    mid = ctx.create_model(pm)
    rp, ci, _ = ctx.crs(mid, values=False)
    orp, oci, _ = OracleModel(pm).crs()
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    ctx.destroy_model(mid)


def test_iea15_hub_rotor_matches_oracle(ctx, golden):
    m, p, hub_bc, hub_id = iea15_hub_rotor_model(golden)
    pm = m.pack()
    mid = ctx.create_model(pm)
    tw = HubTwin(pm)
    for i in range(golden["num_steps"]):
        u = iea15_hub_displacement(i, golden)
        ctx.set_prescribed(mid, hub_bc, u)
        tw.set_prescribed(hub_bc, u)
        st, it = ctx.step([mid], p)
        ost, oit = tw.step(p)
        assert (st[0], it[0]) == (ost, oit) == (0, oit)
        # Same Newton decisions, and equal error norms while the correction is
        # larger than the tolerance.  Below it the norm measures a correction
        # computed from a residual ~1e-12 of the first one, where rounding of
        # the residual shows (the oracle against itself with the quadrature
        # summed in reverse: 5e-5 relative at 0.02).
        g, o = ctx.convergence(mid), tw.convergence()
        assert len(g) == len(o)
        for a, b in zip(g, o):
            assert (a <= 1.0) == (b <= 1.0)
            if b > 1.0:
                assert abs(a - b) <= 1e-6 * b, (a, b)
    assert_state_close(ctx, mid, tw, fields=FIELDS)
    np.testing.assert_allclose(ctx.state(mid, "q")[hub_id],
                               iea15_hub_displacement(golden["num_steps"] - 1, golden), atol=1e-12)
    ctx.destroy_model(mid)


def test_hub_rotor_batched_motion_and_gather(ctx, golden):
    """kyn_set_prescribed_batch feeds the hub BC of every model (one row per
    constraint of each listed model) and kyn_get_state_batch returns the hub
    rows, equal to the per-model calls."""
    m, p, hub_bc, hub_id = iea15_hub_rotor_model(golden)
    pm = m.pack()
    a = np.array([ctx.create_model(pm), ctx.create_model(pm)], dtype=np.int32)
    b = [ctx.create_model(pm), ctx.create_model(pm)]
    nc = pm.desc.num_constraints
    for i in range(3):
        u = np.asarray(iea15_hub_displacement(i, golden), dtype=np.float64)
        vals = np.zeros((2 * nc, 7))
        vals[:, 3] = 1.0
        vals[hub_bc] = u
        vals[nc + hub_bc] = u
        ctx.set_prescribed_batch(a, vals.ctypes.data, False)
        for mid in b:
            ctx.set_prescribed(mid, hub_bc, u)
        sa, ia = ctx.step(a, p)
        sb, ib = ctx.step(b, p)
        assert np.array_equal(sa, sb) and np.array_equal(ia, ib)
    nn = pm.desc.num_nodes
    q = np.zeros((2 * nn, 7))
    ctx.get_state_batch(a, "q", q.ctypes.data, False)
    for k, mid in enumerate(b):
        np.testing.assert_array_equal(q[k * nn:(k + 1) * nn], ctx.state(mid, "q"))
    for mid in list(a) + b:
        ctx.destroy_model(int(mid))


def test_hub_rotor_restart(ctx, golden):
    m, p, hub_bc, _ = iea15_hub_rotor_model(golden)
    pm = m.pack()
    a = ctx.create_model(pm)

    def drive(mid, k0, k1):
        for i in range(k0, k1):
            ctx.set_prescribed(mid, hub_bc, iea15_hub_displacement(i, golden))
            assert ctx.step([mid], p)[0][0] == 0

    drive(a, 0, 4)
    rec = ctx.write_restart(a)
    drive(a, 4, 7)
    b = ctx.create_model(pm)
    ctx.read_restart(b, rec)
    drive(b, 4, 7)
    for f in ("q", "v", "vd", "a", "x"):
        np.testing.assert_array_equal(ctx.state(a, f), ctx.state(b, f))


@pytest.mark.parametrize("prescribed_hub", [False, True])
def test_rotation_control_matches_oracle_and_golden(ctx, prescribed_hub):
    """RotationControl from a hub node to a blade root
    (test_rotating_beam.cpp:390-512): the root is pitched by t pi/2 about x
    while the hub is fixed, or turned about z by a PrescribedBC.  Same Newton
    decisions and states as the oracle; the reference's golden q (fixed hub,
    10 steps, 1e-6) or root rotation vector (prescribed hub, 100 steps, 1e-8)."""
    from tests.workloads_ref import (quaternion_to_rotation_vector, rotation_control_inputs,
                                     rotation_control_test_model)
    g = load_golden("rotation_control.json")["prescribed_hub" if prescribed_hub else "fixed_hub"]
    m, p, rc, bc = rotation_control_test_model(prescribed_hub)
    pm = m.pack()
    mid = ctx.create_model(pm)
    rp, ci, _ = ctx.crs(mid, values=False)
    orp, oci, _ = OracleModel(pm).crs()
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    tw = HubTwin(pm)
    for i in range(g["steps"]):
        pitch, u_hub = rotation_control_inputs(i)
        ctx.set_control(mid, rc, pitch)
        tw.set_prescribed(rc, [pitch, 0., 0., 1., 0., 0., 0.])
        if prescribed_hub:
            ctx.set_prescribed(mid, bc, u_hub)
            tw.set_prescribed(bc, u_hub)
        st, it = ctx.step([mid], p)
        ost, oit = tw.step(p)
        assert (st[0], it[0]) == (ost, oit) == (0, oit)
        gc, oc = ctx.convergence(mid), tw.convergence()
        assert len(gc) == len(oc)
        for a, b in zip(gc, oc):
            assert (a <= 1.0) == (b <= 1.0)
            if b > 1.0:
                assert abs(a - b) <= 1e-6 * b, (a, b)
    assert_state_close(ctx, mid, tw, fields=FIELDS)
    q = ctx.state(mid, "q")
    if prescribed_hub:
        np.testing.assert_allclose(quaternion_to_rotation_vector(q[0, 3:]), g["rv_root"],
                                   rtol=0, atol=g["tolerance"])
    else:
        np.testing.assert_allclose(q.ravel(), g["q"], rtol=0, atol=g["tolerance"])
    ctx.destroy_model(mid)
