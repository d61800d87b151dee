"""Condensed dense models against the oracle: beams larger than one FP64 beam
system (a 41-node cantilever of four order-10 elements, a 31-node tower of
three elements with a nacelle mass) and two 21-node beams coupled by a rigid
joint (264 unknowns).  Each element's interior nodes are eliminated inside the
element (cond_component_terms in kyn_step_kernel.cuh); the shared element
ends, the nodes with masses or constraints and the constraint rows form the
bordered system.  The oracle factors the whole system as the reference does
(src/solver/compute_system_row_entries.hpp:83-97 gives the element overlap).

Bar: bit-exact CRS graph, identical Newton iteration counts and status at
every step, the same convergence history, states within 1e-10 relative
(accelerations 1e-7, multipliers at the oracle twin floor), as in
tests/test_gpu_parity.py."""
import numpy as np
import pytest

from tests.test_gpu_parity import FIELDS, Twin, assert_convergence_close, assert_state_close, rel_err
from tests.workloads_ref import (chain_tip_loads, four_element_cantilever_model, revolute_pendulum_model,
                                 tower_model, two_long_beams_model)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from openturbine_b200.runtime import Context
    c = Context(0)
    yield c
    c.close()


def _run(ctx, pm, p, steps, loads=None, check_every=0):
    mid = ctx.create_model(pm)
    tw = Twin(pm)
    rp, ci, _ = ctx.crs(mid, values=False)
    orp, oci, _ = tw.crs()
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    for k in range(steps):
        if loads is not None:
            fx = loads(k)
            ctx.set_node_fx(mid, fx)
            tw.set_node_fx(fx)
        st, it = ctx.step([mid], p)
        ost, oit = tw.step(p)
        assert (st[0], it[0]) == (ost, oit) == (0, oit), (k, st[0], it[0], ost, oit)
        assert_convergence_close(ctx.convergence(mid), tw.convergence())
        if check_every and k % check_every == check_every - 1:
            assert_state_close(ctx, mid, tw, fields=FIELDS)
    assert_state_close(ctx, mid, tw, fields=FIELDS)
    return mid, tw


def test_four_element_cantilever_41_nodes(ctx):
    m, p, along, elems = four_element_cantilever_model()
    pm = m.pack()
    mid0 = ctx.create_model(pm)
    info = ctx.info(mid0)
    assert info.condensed_dofs == 30 and info.num_dofs == 252
    ctx.destroy_model(mid0)
    mid, _ = _run(ctx, pm, p, 60, loads=lambda k: chain_tip_loads(elems, along[-1], k), check_every=20)
    q = ctx.state(mid, "q")
    assert np.abs(q[along[-1], 2]).max() > 1e-4   # the tip moved
    ctx.destroy_model(mid)


def test_tower_three_elements_with_nacelle_mass(ctx):
    m, p, along, elems = tower_model()
    pm = m.pack()
    mid0 = ctx.create_model(pm)
    assert ctx.info(mid0).condensed_dofs == 30
    ctx.destroy_model(mid0)

    def loads(k):  # the tip load of the cantilever, as a lateral (x) force on the tower top
        fx = 2.0e3 * chain_tip_loads(elems, along[-1], k, h=p.h)
        fx[:, [0, 2]] = fx[:, [2, 0]]
        return fx
    mid, _ = _run(ctx, pm, p, 40, loads=loads, check_every=20)
    ctx.destroy_model(mid)


def test_two_long_beams_rigid_joint(ctx):
    m, p, beams = two_long_beams_model()
    pm = m.pack()
    mid0 = ctx.create_model(pm)
    assert ctx.info(mid0).condensed_dofs == 30 and ctx.info(mid0).num_dofs == 264
    ctx.destroy_model(mid0)
    mid, _ = _run(ctx, pm, p, 50, check_every=25)
    q = ctx.state(mid, "q")
    assert np.abs(q[beams[1][0], :3] - q[beams[0][-1], :3]).max() < 1e-9
    ctx.destroy_model(mid)


def test_condensed_models_in_both_forms_and_batched(ctx):
    """The bordered system solves in FP64 in both precision forms, so the FP32
    form steps a condensed model bit for bit like the FP64 form; condensed
    models batched with beam systems match themselves stepped alone."""
    from openturbine_b200 import workloads as W
    m, p, along, elems = four_element_cantilever_model()
    pm = m.pack()
    a, b = ctx.create_model(pm), ctx.create_model(pm)
    p32 = four_element_cantilever_model()[1]
    p32.precision = 1
    for k in range(10):
        fx = chain_tip_loads(elems, along[-1], k)
        ctx.set_node_fx(a, fx)
        ctx.set_node_fx(b, fx)
        ctx.step([a], p)
        ctx.step([b], p32)
    assert rel_err(ctx.state(b, "q"), ctx.state(a, "q")) == 0.0
    pms = [tower_model()[0].pack(), two_long_beams_model()[0].pack(),
           W.batch_cantilever_model(W.draw_batch(1, first_id=43)[0]).pack()]
    mixed = [ctx.create_model(x) for x in pms]
    alone = [ctx.create_model(x) for x in pms]
    pb = W.batch_params()
    for _ in range(4):
        sm, im = ctx.step(mixed, pb)
        for i, mid in enumerate(alone):
            sa, ia = ctx.step([mid], pb)
            assert (sm[i], im[i]) == (sa[0], ia[0])
    for x, y in zip(mixed, alone):
        assert rel_err(ctx.state(x, "q"), ctx.state(y, "q")) == 0.0
    for mid in [a, b] + mixed + alone:
        ctx.destroy_model(mid)


def test_revolute_joint_in_a_dense_model(ctx):
    """A revolute joint as five constraint rows of a dense bordered system (the
    turbine's shaft joint sits between nodes of such a system): a pendulum on a
    revolute joint about x, swung by gravity and driven by the joint torque,
    against the oracle for 200 steps, states and the joint's output."""
    m, p = revolute_pendulum_model()
    pm = m.pack()
    mid = ctx.create_model(pm)
    tw = Twin(pm)
    for k in range(200):
        torque = 30.0 * np.sin(0.05 * k)
        u = np.array([torque, 0., 0., 1., 0., 0., 0.])
        ctx.set_prescribed(mid, 1, u)
        tw.set_prescribed(1, u)
        st, it = ctx.step([mid], p)
        ost, oit = tw.step(p)
        assert (st[0], it[0]) == (ost, oit) == (0, oit), (k, st[0], it[0], ost, oit)
        assert_convergence_close(ctx.convergence(mid), tw.convergence())
        if k % 50 == 49:  # the joint output (rotation, rate, acceleration about its axis)
            out = ctx.state(mid, "output")
            np.testing.assert_allclose(out, tw.o.state("output"), rtol=1e-9, atol=1e-10)
            assert abs(out[1, 0]) > 1e-3
    assert_state_close(ctx, mid, tw, fields=FIELDS)
    q = ctx.state(mid, "q")
    assert abs(q[2, 2]) > 1e-2   # the bob swung
    ctx.destroy_model(mid)


def test_condensed_tower_under_base_motion_and_state_f(ctx):
    """The condensed tower with its base moved by its PrescribedBC (a lateral
    ground motion) and external forces given as state.f at an interior node of
    the middle element (eliminated inside that element) and at the top (a
    boundary node), against the oracle for 40 steps."""
    m, p, along, elems = tower_model()
    pm = m.pack()
    mid = ctx.create_model(pm)
    tw = Twin(pm)
    interior = elems[1][4]   # a node of the middle element only
    nn = len(m.nodes_)
    for k in range(40):
        t = (k + 1) * p.h
        u = np.array([0.05 * np.sin(6.0 * t), 0.02 * np.sin(4.0 * t), 0., 1., 0., 0., 0.])
        ctx.set_prescribed(mid, 0, u)
        tw.set_prescribed(0, u)
        f = np.zeros((nn, 6))
        f[interior, 1] = 5.0e4 * np.cos(5.0 * t)
        f[along[-1], 0] = 1.0e5 * np.sin(3.0 * t)
        ctx.set_state_f(mid, f)
        tw.o.set_state_f(f)
        tw.alt.set_state_f(f)
        st, it = ctx.step([mid], p)
        ost, oit = tw.step(p)
        assert (st[0], it[0]) == (ost, oit) == (0, oit), (k, st[0], it[0], ost, oit)
        assert_convergence_close(ctx.convergence(mid), tw.convergence())
    assert_state_close(ctx, mid, tw, fields=FIELDS)
    q = ctx.state(mid, "q")
    assert abs(q[interior, 1]) > 1e-5   # the interior node moved sideways
    ctx.destroy_model(mid)
