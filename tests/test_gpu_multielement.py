"""Beams of several elements sharing nodes: one CTA's system over all the
elements' nodes, the elements' integrals adding up at the shared node
(src/solver/compute_system_row_entries.hpp:83-97), against the oracle, which
assembles every element into the CRS system like the reference."""
import numpy as np
import pytest

from oracle.oracle_py import OracleModel
from tests.test_gpu_parity import FIELDS, Twin, assert_state_close
from tests.workloads_ref import two_element_cantilever_loads, two_element_cantilever_model

pytestmark = pytest.mark.gpu


class DenseTwin(Twin):
    """The oracle with the dense solve of the whole system, and again with the
    quadrature sums reversed (the rounding-noise floor)."""

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


def test_two_element_cantilever_matches_oracle(ctx):
    m, p = two_element_cantilever_model()
    pm = m.pack()
    mid = ctx.create_model(pm)
    info = ctx.info(mid)
    assert info.num_beams == 2
    rp, ci, _ = ctx.crs(mid, values=False)
    tw = DenseTwin(pm)
    orp, oci, _ = tw.crs()
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    for k in range(20):
        fx = two_element_cantilever_loads(k)
        ctx.set_node_fx(mid, fx)
        tw.set_node_fx(fx)
        st, it = ctx.step([mid], p)
        ost, oit = tw.step(p)
        assert (st[0], it[0]) == (ost, oit) == (0, oit)
        g, o = ctx.convergence(mid), tw.convergence()
        assert len(g) == len(o)
        for x, y in zip(g, o):
            assert (x <= 1.0) == (y <= 1.0)
            if y > 1.0:
                assert abs(x - y) <= 1e-6 * y, (x, y)
    assert_state_close(ctx, mid, tw, fields=FIELDS)
    ctx.destroy_model(mid)


def test_two_element_beams_in_a_batch_and_batched_loads_rejected(ctx):
    """Several two-element beams step together with single-element beams and
    match their lone twin; the batched node_FX path (one row per beam-local
    node) refuses models whose nodes are shared between elements."""
    from openturbine_b200 import workloads as W
    from openturbine_b200.runtime import LOAD_NODE_FX, KynError
    m, p = two_element_cantilever_model()
    pm = m.pack()
    alone = ctx.create_model(pm)
    twins = [ctx.create_model(pm) for _ in range(3)]
    draws = W.draw_batch(4, first_id=950)
    beams = [ctx.create_model(W.batch_cantilever_model(d).pack()) for d in draws]
    ids = np.array(beams[:2] + twins + beams[2:], dtype=np.int32)
    for k in range(10):
        fx = two_element_cantilever_loads(k)
        for mid in [alone] + twins:
            ctx.set_node_fx(mid, fx)
        ctx.step([alone], p)
        ctx.step(ids, p)
    for mid in twins:
        np.testing.assert_array_equal(ctx.state(mid, "q"), ctx.state(alone, "q"))
    vals = np.zeros((6 * 3, 6))
    with pytest.raises(KynError):
        ctx.set_loads_batch(np.array(twins, dtype=np.int32), LOAD_NODE_FX, vals.ctypes.data, False)
    for mid in [alone] + twins + beams:
        ctx.destroy_model(mid)
