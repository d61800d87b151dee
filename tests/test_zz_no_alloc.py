"""kyn_set_loads_batch_static (staging in the library's fixed device array, no
allocation) against kyn_set_loads_batch on the same inputs.

Some callers cannot let a library allocate device memory while they run: a CFD
solver that owns the GPU's memory through its own pool, for example, or a code
that must not see cudaMalloc/cudaFree synchronise the device in the middle of
its time step.  The static entry point serves them; these tests check that it
moves the same values as the allocating one and that it allocates nothing.

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


def _pool_bytes():
    """(used, reserved) bytes of the device's default memory pool, which the
    library's stream-ordered allocations come from; None without cuda-python."""
    try:
        from cuda.bindings import driver as drv
    except ImportError:
        return None
    import torch
    err, dev = drv.cuDeviceGet(torch.cuda.current_device())
    assert err == drv.CUresult.CUDA_SUCCESS
    err, pool = drv.cuDeviceGetDefaultMemPool(dev)
    assert err == drv.CUresult.CUDA_SUCCESS
    out = []
    for attr in (drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_CURRENT,
                 drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT):
        err, v = drv.cuMemPoolGetAttribute(pool, attr)
        assert err == drv.CUresult.CUDA_SUCCESS
        out.append(int(v))
    return tuple(out)


def _snapshot(ctx):
    """Everything an allocation would move: the context's allocation counter
    and resident bytes, the default pool's used/reserved bytes and the free
    device memory."""
    import torch
    torch.cuda.synchronize()
    return {"allocations": ctx.allocations, "used_bytes": ctx.used_bytes,
            "pool": _pool_bytes(), "free": torch.cuda.mem_get_info()[0]}


def _static_call_allocates_nothing(ctx, *args):
    before = _snapshot(ctx)
    ctx.set_loads_batch_static(*args)
    after = _snapshot(ctx)
    assert after == before, (before, after)


def test_static_staging_matches_allocating_entry_point():
    """Two calls in a row (the second over the first one's leftovers), node_FX
    and state.f channels, host and device values: the static path must leave
    the slabs exactly as kyn_set_loads_batch does (tolerance 0: the same copy
    kernel moves the same doubles), so states after a step are identical; and
    once the one-time set-up has run, no static call allocates."""
    import torch
    from openturbine_b200.runtime import LOAD_NODE_FX, LOAD_STATE_F, Context
    ctx = Context(0)
    draws, a, b = _twin_batch(ctx, 24, 700)
    rows = sum(d.num_nodes for d in draws)
    p = W.batch_params()
    rng = np.random.default_rng(7)
    # set-up call: looks up the fixed array's device address once per device
    ctx.set_loads_batch_static(a, LOAD_STATE_F, np.zeros((rows, 6)).ctypes.data, False)
    for k in range(2):
        fz = W.tip_loads(draws, k)
        fx = np.concatenate([W.node_fx_for(d, fz[i]) for i, d in enumerate(draws)])
        f = rng.standard_normal((rows, 6)) * 10.0
        if k == 0:
            _static_call_allocates_nothing(ctx, a, LOAD_NODE_FX, fx.ctypes.data, False)
            _static_call_allocates_nothing(ctx, a, LOAD_STATE_F, f.ctypes.data, False)
        else:
            dev_fx = torch.from_numpy(fx).cuda()
            _static_call_allocates_nothing(ctx, a, LOAD_NODE_FX, dev_fx.data_ptr(), True)
            _static_call_allocates_nothing(ctx, a, LOAD_STATE_F, f.ctypes.data, False)
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
    ctx.close()


def test_static_state_f_on_multi_beam_and_hub_models():
    """state.f of models with several beams and a hub node (rows per model =
    its nodes, hub included; the hub carries no load) mixed with single beams:
    the static path goes through the node map, the allocating one through
    per-model offsets; after each of two calls in a row, a step from each
    must give bit-identical states."""
    from openturbine_b200.runtime import LOAD_STATE_F, Context
    from tests.workloads_ref import iea15_hub_rotor_model
    ctx = Context(0)
    hub_rotor, _, _, _ = iea15_hub_rotor_model()
    rotor, _ = W.rotor_model(3)
    pms = [hub_rotor.pack(), W.batch_cantilever_model(W.draw_batch(1, first_id=900)[0]).pack(),
           rotor.pack(), W.batch_cantilever_model(W.draw_batch(1, first_id=901)[0]).pack()]
    a = np.array([ctx.create_model(pm) for pm in pms], dtype=np.int32)
    b = np.array([ctx.create_model(pm) for pm in pms], dtype=np.int32)
    rows = sum(int(pm.desc.num_nodes) for pm in pms)
    rng = np.random.default_rng(11)
    ctx.set_loads_batch_static(a, LOAD_STATE_F, np.zeros((rows, 6)).ctypes.data, False)
    p = W.batch_params()
    for _ in range(2):
        f = rng.standard_normal((rows, 6)) * 100.0
        _static_call_allocates_nothing(ctx, a, LOAD_STATE_F, f.ctypes.data, False)
        ctx.set_loads_batch(b, LOAD_STATE_F, f.ctypes.data, False)
        sa, ia = ctx.step(a, p)
        sb, ib = ctx.step(b, p)
        assert np.array_equal(sa, sb) and np.array_equal(ia, ib)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(ctx.state(int(x), "q"), ctx.state(int(y), "q"))
    for i in list(a) + list(b):
        ctx.destroy_model(int(i))
    ctx.close()


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
    ctx.close()
