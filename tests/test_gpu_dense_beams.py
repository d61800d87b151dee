"""Beams inside one dense bordered system (dense_kernel with beam components)
against the oracle: beams coupled to each other by a joint between their nodes,
and beams carrying three-row constraints (a mooring line at a beam tip).

Bar: identical Newton iteration counts and status at every step, bit-exact CRS
graph, states within 1e-10 relative (accelerations 1e-7, multipliers at the
oracle twin floor), as in tests/test_gpu_parity.py."""
import numpy as np
import pytest

from oracle.oracle_py import OracleModel
from tests.test_gpu_parity import FIELDS, Twin, assert_state_close, rel_err
from tests.workloads_ref import cantilever_test_loads, moored_cantilever_model, two_beams_model

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from openturbine_b200.runtime import Context
    c = Context(0)
    yield c
    c.close()


def test_two_beams_crs_graph_bit_exact(ctx):
    for m, _ in (two_beams_model(), moored_cantilever_model()):
        pm = m.pack()
        mid = ctx.create_model(pm)
        rp, ci, _ = ctx.crs(mid, values=False)
        orp, oci, _ = OracleModel(pm).crs()
        assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
        ctx.destroy_model(mid)


def test_two_beams_rigid_joint_1000_steps(ctx):
    """BladeInterfaceTest.TwoBeams: converged at each of 1000 steps (the
    reference test's assertion), with the oracle's Newton decisions and states."""
    m, p = two_beams_model()
    pm = m.pack()
    mid = ctx.create_model(pm)
    o = Twin(pm)
    for k in range(1000):
        st, it = ctx.step([mid], p)
        ost, oit = o.step(p)
        assert (st[0], it[0]) == (ost, oit) == (0, oit), (k, st[0], it[0], ost, oit)
        if k % 250 == 249:
            assert_state_close(ctx, mid, o)
    # the joint carries the second beam: its root follows the first beam's tip
    q = ctx.state(mid, "q")
    assert np.abs(q[4, :3] - q[3, :3]).max() < 1e-9
    ctx.destroy_model(mid)


def test_moored_cantilever_matches_oracle(ctx):
    """A cantilever whose tip carries a point mass and a mooring line (position-only
    fairlead by a RigidJoint6DOFsTo3DOFs, spring, anchor held by FixedBC3DOFs),
    under the cantilever test's tip loads, in both precision forms (a dense
    system solves in FP64 in both)."""
    for precision in (0, 1):
        m, p = moored_cantilever_model()
        p.precision = precision
        pm = m.pack()
        mid = ctx.create_model(pm)
        o = Twin(pm)
        for k in range(60):
            fx = cantilever_test_loads(k % 3) * (1.0 + 0.1 * k)
            ctx.set_node_fx(mid, fx)
            o.set_node_fx(fx)
            st, it = ctx.step([mid], p)
            ost, oit = o.step(p)
            assert (st[0], it[0]) == (ost, oit), (precision, k, st[0], it[0], ost, oit)
        assert_state_close(ctx, mid, o, fields=FIELDS)
        ctx.destroy_model(mid)


def test_dense_beams_batched_with_beam_systems(ctx):
    """Dense models with beams in one step call with ordinary beams and rotors:
    each result equals the same model stepped alone."""
    from openturbine_b200 import workloads as W
    mk = [lambda: two_beams_model()[0], lambda: moored_cantilever_model()[0],
          lambda: W.batch_cantilever_model(W.draw_batch(1, first_id=41)[0]), lambda: W.rotor_model(2)[0]]
    pms = [f().pack() for f in mk]
    mixed = [ctx.create_model(pm) for pm in pms]
    alone = [ctx.create_model(pm) for pm in pms]
    p = W.batch_params()
    for _ in range(5):
        sm, im = ctx.step(mixed, p)
        for i, mid in enumerate(alone):
            sa, ia = ctx.step([mid], p)
            assert (sm[i], im[i]) == (sa[0], ia[0])
    for a, b in zip(mixed, alone):
        assert rel_err(ctx.state(a, "q"), ctx.state(b, "q")) == 0.0
    for mid in mixed + alone:
        ctx.destroy_model(mid)
