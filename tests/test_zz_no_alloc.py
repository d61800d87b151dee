"""kyn_set_loads_batch_static (staging in the library's fixed device array, no
allocation) against kyn_set_loads_batch on the same inputs.

Kept in its own file, collected last, so it runs both after every other test
and alone in a fresh process.
"""
import numpy as np
import pytest

from openturbine_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _twin_batch(ctx, n, first_id):
    draws = W.draw_batch(n, first_id=first_id)
    pms = [W.batch_cantilever_model(d).pack() for d in draws]
    a = np.array([ctx.create_model(pm) for pm in pms], dtype=np.int32)
    b = np.array([ctx.create_model(pm) for pm in pms], dtype=np.int32)
    return draws, a, b


def test_static_staging_matches_allocating_entry_point():
    """Two calls in a row (the second over the first one's leftovers), node_FX
    and state.f channels, host and device values: the static path must leave
    the slabs exactly as kyn_set_loads_batch does (tolerance 0: the same copy
    kernel moves the same doubles), so states after a step are identical."""
    import torch
    from openturbine_b200.runtime import LOAD_NODE_FX, LOAD_STATE_F, Context
    ctx = Context(0)
    draws, a, b = _twin_batch(ctx, 24, 700)
    rows = sum(d.num_nodes for d in draws)
    p = W.batch_params()
    rng = np.random.default_rng(7)
    for k in range(2):
        fz = W.tip_loads(draws, k)
        fx = np.concatenate([W.node_fx_for(d, fz[i]) for i, d in enumerate(draws)])
        f = rng.standard_normal((rows, 6)) * 10.0
        if k == 0:
            ctx.set_loads_batch_static(a, LOAD_NODE_FX, fx.ctypes.data, False)
            ctx.set_loads_batch_static(a, LOAD_STATE_F, f.ctypes.data, False)
        else:
            dev_fx = torch.from_numpy(fx).cuda()
            ctx.set_loads_batch_static(a, LOAD_NODE_FX, dev_fx.data_ptr(), True)
            ctx.set_loads_batch_static(a, LOAD_STATE_F, f.ctypes.data, False)
            torch.cuda.synchronize()
        ctx.set_loads_batch(b, LOAD_NODE_FX, fx.ctypes.data, False)
        ctx.set_loads_batch(b, LOAD_STATE_F, f.ctypes.data, False)
        fa = np.zeros((rows, 6))
        ctx.get_state_batch(a, "f", fa.ctypes.data, False)
        np.testing.assert_array_equal(fa, f)
        sa, ia = ctx.step(a, p)
        sb, ib = ctx.step(b, p)
        assert np.array_equal(sa, sb) and np.array_equal(ia, ib)
        qa = np.zeros((rows, 7))
        qb = np.zeros((rows, 7))
        ctx.get_state_batch(a, "q", qa.ctypes.data, False)
        ctx.get_state_batch(b, "q", qb.ctypes.data, False)
        np.testing.assert_array_equal(qa, qb)
    for i in list(a) + list(b):
        ctx.destroy_model(int(i))


def test_static_staging_rejects_oversized_batches():
    """More beam elements than the fixed array holds: a clear error, no copy."""
    from openturbine_b200.runtime import LOAD_NODE_FX, Context, KynError
    ctx = Context(0)
    draws = W.draw_batch(1, first_id=800)
    mid = ctx.create_model(W.batch_cantilever_model(draws[0]).pack())
    ids = np.full(8193, mid, dtype=np.int32)
    vals = np.zeros(8193 * draws[0].num_nodes * 6)
    with pytest.raises(KynError) as e:
        ctx.set_loads_batch_static(ids, LOAD_NODE_FX, vals.ctypes.data, False)
    assert "8192" in str(e.value)
    ctx.destroy_model(mid)
