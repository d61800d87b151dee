"""FP32 + refinement form (KYN_PRECISION_FP32_REFINED) against the FP64 oracle.

The form computes the tangent blocks, the integration GEMM (3xTF32 tensor
cores) and the LU in FP32 and keeps the residual, the rotation update and the
convergence test in FP64, so each Newton iteration refines the state with an
FP64 residual.  Its iterates are not the reference's, so the checks are on the
stopped states (tolerances below are the measured bars, written here), not on
rounding-level equality.
"""
import numpy as np
import pytest

from oracle.oracle_py import OracleModel
from openturbine_b200 import workloads as W
from openturbine_b200.model import StepParameters

pytestmark = pytest.mark.gpu

TIP_REL_CANTILEVER = 1e-8     # north-star bar, met on the cantilever configuration
TIP_REL_BATCH_MEDIAN = 1e-8   # median over the converged beams of the batch
TIP_REL_BATCH_MAX = 1e-5      # worst beam: Newton stops at a different iterate
ROOT_LOAD_REL = 1e-5


def fp32(p, refine=0):
    return StepParameters(p.is_dynamic_solve, p.max_iter, p.h, p.rho_inf, p.absolute_convergence_tol,
                          p.relative_convergence_tol, precision=1, refine_iters=refine)


@pytest.fixture(scope="module")
def ctx():
    from openturbine_b200.runtime import Context
    c = Context(0)
    yield c
    c.close()


def test_cantilever_fp32_form(ctx):
    pm = W.cantilever_model().pack()
    mid = ctx.create_model(pm)
    o = OracleModel(pm)
    p = W.cantilever_params()
    for k in range(100):
        fx = np.zeros((5, 6))
        fx[4, 2] = W.cantilever_tip_load(k)
        ctx.set_node_fx(mid, fx)
        o.set_node_fx(fx)
        st, it = ctx.step([mid], fp32(p))
        ost, oit = o.step(p)
        assert st[0] == 0 and ost == 0
        assert abs(int(it[0]) - oit) <= 1
    q, qo = ctx.state(mid, "q"), o.state("q")
    assert np.abs(q[4, :3] - qo[4, :3]).max() / np.abs(qo[4, :3]).max() < TIP_REL_CANTILEVER
    lam, lo = ctx.state(mid, "lambda"), o.state("lambda")
    assert np.abs(lam - lo).max() / np.abs(lo).max() < ROOT_LOAD_REL
    ctx.destroy_model(mid)


def test_batch_fp32_form(ctx):
    draws = W.draw_batch(64)
    pms = [W.batch_cantilever_model(d).pack() for d in draws]
    ids = np.array([ctx.create_model(pm) for pm in pms], dtype=np.int32)
    orcs = [OracleModel(pm) for pm in pms]
    p = W.batch_params()
    alive = np.ones(len(draws), dtype=bool)
    for k in range(12):
        fz = W.tip_loads(draws, k)
        for i, d in enumerate(draws):
            fx = W.node_fx_for(d, fz[i])
            ctx.set_node_fx(int(ids[i]), fx)
            orcs[i].set_node_fx(fx)
        st, _ = ctx.step(ids, fp32(p))
        for i, o in enumerate(orcs):
            ost, _ = o.step(p)
            alive[i] &= (st[i] == 0) and (ost == 0)
    assert alive.sum() >= 32
    errs = []
    for i, d in enumerate(draws):
        if not alive[i]:
            continue
        q, qo = ctx.state(int(ids[i]), "q"), orcs[i].state("q")
        tip = d.num_nodes - 1
        errs.append(np.abs(q[tip, :3] - qo[tip, :3]).max() / np.abs(qo[tip, :3]).max())
    errs = np.array(errs)
    assert np.median(errs) < TIP_REL_BATCH_MEDIAN, np.median(errs)
    assert errs.max() < TIP_REL_BATCH_MAX, errs.max()
    for i in ids:
        ctx.destroy_model(int(i))


def test_refinement_correction_counts(ctx):
    """refine_iters adds that many corrections after the convergence test."""
    pm = W.cantilever_model().pack()
    a, b = ctx.create_model(pm), ctx.create_model(pm)
    p = W.cantilever_params()
    fx = np.zeros((5, 6))
    fx[4, 2] = W.cantilever_tip_load(0)
    ctx.set_node_fx(a, fx)
    ctx.set_node_fx(b, fx)
    sa, ia = ctx.step([a], fp32(p, 0))
    sb, ib = ctx.step([b], fp32(p, 1))
    assert sa[0] == 0 and sb[0] == 0
    assert ib[0] == ia[0] + 1


def test_autotune_keeps_results(ctx):
    """The autotuner's choices (threads per CTA; in the FP64 form also the
    panel LU or the register Gauss-Jordan solve per size class) change timing,
    and the results only at the rounding level: the same statuses and Newton
    iterations, converged states within 1e-12."""
    from openturbine_b200.runtime import Context
    draws = W.draw_batch(48, first_id=9000)
    pms = [W.batch_cantilever_model(d).pack() for d in draws]
    p = W.batch_params()
    out = []
    for tune in (False, True):
        c = Context(0)
        ids = np.array([c.create_model(pm) for pm in pms], dtype=np.int32)
        if tune:
            c.autotune(ids, p)
            assert all(c.tuned_threads(int(i)) in (128, 256, 512) for i in ids)
            assert all(c.tuned_solver(int(i)) in (0, 1) for i in ids)
        res = []
        for k in range(4):
            fz = W.tip_loads(draws, k)
            for i, d in enumerate(draws):
                c.set_node_fx(int(ids[i]), W.node_fx_for(d, fz[i]))
            res.append(c.step(ids, p))
        out.append((res, [c.state(int(i), "q") for i in ids]))
        c.close()
    (r0, q0), (r1, q1) = out
    for (s0, i0), (s1, i1) in zip(r0, r1):
        assert np.array_equal(s0, s1) and np.array_equal(i0, i1)
    # states of the beams converged at every step (a diverging iterate left by
    # max_iter is not a result: another thread count's reduction order moves it)
    ok = np.all([s == 0 for s, _ in r0], axis=0)
    assert ok.sum() >= len(draws) // 2
    for i in np.flatnonzero(ok):
        assert np.abs(q0[i] - q1[i]).max() <= 1e-12 * max(1.0, np.abs(q0[i]).max())


def test_cuda_graph_replay_matches_direct_launches():
    """Steps replayed from the captured graph give the same results and
    launch counts as direct launches."""
    from openturbine_b200.runtime import Context
    draws = W.draw_batch(40, first_id=9100)
    pms = [W.batch_cantilever_model(d).pack() for d in draws]
    p = W.batch_params()
    runs = []
    for graph in (False, True):
        c = Context(0)
        c.set_cuda_graph(graph)
        ids = np.array([c.create_model(pm) for pm in pms], dtype=np.int32)
        res = []
        for k in range(5):
            fz = W.tip_loads(draws, k)
            for i, d in enumerate(draws):
                c.set_node_fx(int(ids[i]), W.node_fx_for(d, fz[i]))
            l0 = c.kernel_launches
            res.append(c.step(ids, p) + (c.kernel_launches - l0,))
        runs.append((res, np.concatenate([c.state(int(i), "q") for i in ids])))
        c.close()
    (r0, q0), (r1, q1) = runs
    for (s0, i0, n0), (s1, i1, n1) in zip(r0, r1):
        assert np.array_equal(s0, s1) and np.array_equal(i0, i1) and n0 == n1 > 0
    np.testing.assert_array_equal(q0, q1)
