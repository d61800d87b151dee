"""Restart records (WriteStateToFile / ReadStateFromFile format) and state copy
(CopyStateData) of resident models."""
import struct

import numpy as np
import pytest

from openturbine_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from openturbine_b200.runtime import Context
    c = Context(0)
    yield c
    c.close()


def _drive(ctx, mid, k0, k1):
    p = W.cantilever_params()
    for k in range(k0, k1):
        fx = np.zeros((5, 6))
        fx[4, 2] = W.cantilever_tip_load(k)
        ctx.set_node_fx(mid, fx)
        st, _ = ctx.step([mid], p)
        assert st[0] == 0


def test_restart_record_layout(ctx):
    mid = ctx.create_model(W.cantilever_model().pack())
    _drive(ctx, mid, 0, 7)
    rec = ctx.write_restart(mid)
    (nn,) = struct.unpack_from("N", rec, 0)   # size_t, native order
    assert nn == 5
    off = struct.calcsize("N")
    for field, w in (("x0", 7), ("x", 7), ("q_delta", 6), ("q_prev", 7), ("q", 7), ("v", 6),
                     ("vd", 6), ("a", 6), ("f", 6)):
        arr = np.frombuffer(rec, dtype=np.float64, count=nn * w, offset=off).reshape(nn, w)
        np.testing.assert_array_equal(arr, ctx.state(mid, field))
        off += nn * w * 8
    assert off == len(rec)


def test_restart_continues_bit_identically(ctx):
    pm = W.cantilever_model().pack()
    a = ctx.create_model(pm)
    _drive(ctx, a, 0, 20)
    rec = ctx.write_restart(a)
    _drive(ctx, a, 20, 30)
    b = ctx.create_model(pm)
    ctx.read_restart(b, rec)
    _drive(ctx, b, 20, 30)
    for f in ("q", "v", "vd", "a", "x"):
        np.testing.assert_array_equal(ctx.state(a, f), ctx.state(b, f))


def test_restart_rejects_other_node_count(ctx):
    from openturbine_b200.runtime import KynError
    a = ctx.create_model(W.cantilever_model().pack())
    d = W.draw_batch(1, first_id=77)[0]
    d = W.BeamDraw(d.model_id, 9, d.length, d.amp, d.freq)
    b = ctx.create_model(W.batch_cantilever_model(d).pack())
    with pytest.raises(KynError) as e:
        ctx.read_restart(b, ctx.write_restart(a))
    assert e.value.code == -1


def test_predictor_corrector_with_state_copy(ctx):
    """Save, take a predictor step, restore, take the corrector step: the result
    equals one step from the saved state (src/interfaces/cfd/interface.cpp:312-327)."""
    pm = W.cantilever_model().pack()
    a, save, twin = ctx.create_model(pm), ctx.create_model(pm), ctx.create_model(pm)
    _drive(ctx, a, 0, 10)
    _drive(ctx, twin, 0, 10)
    p = W.cantilever_params()
    ctx.copy_state(save, a)
    fx = np.zeros((5, 6))
    fx[4, 2] = 3e3
    ctx.set_node_fx(a, fx)
    ctx.step([a], p)                 # predictor
    ctx.copy_state(a, save)          # restore
    fx[4, 2] = -2e3
    ctx.set_node_fx(a, fx)
    ctx.set_node_fx(twin, fx)
    ctx.step([a], p)                 # corrector
    ctx.step([twin], p)
    for f in ("q", "v", "vd", "a"):
        np.testing.assert_array_equal(ctx.state(a, f), ctx.state(twin, f))


def test_clone_continues_like_the_original(ctx):
    """kyn_model_clone of a model part-way through a run: the clone has the
    original's state and, stepped with the same loads, stays identical to it
    bit for bit; the source is unaffected and both can be destroyed."""
    from openturbine_b200 import workloads as W
    d = W.draw_batch(1, first_id=4242)[0]
    p = W.batch_params()
    src = ctx.create_model(W.batch_cantilever_model(d).pack())
    for k in range(3):
        ctx.set_node_fx(src, W.node_fx_for(d, W.tip_loads([d], k)[0]))
        ctx.step([src], p)
    cl = ctx.clone_model(src)
    for f in ("q", "v", "vd", "a", "x", "lambda"):
        np.testing.assert_array_equal(ctx.state(cl, f), ctx.state(src, f))
    for k in range(3, 8):
        fx = W.node_fx_for(d, W.tip_loads([d], k)[0])
        ctx.set_node_fx(src, fx)
        ctx.set_node_fx(cl, fx)
        st, it = ctx.step([src, cl], p)
        assert st[0] == st[1] and it[0] == it[1]
    for f in ("q", "v", "vd", "a", "x", "lambda"):
        np.testing.assert_array_equal(ctx.state(cl, f), ctx.state(src, f))
    ctx.destroy_model(cl)
    ctx.destroy_model(src)
