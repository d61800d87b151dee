"""The synthetic workloads: seeded and reproducible, and the precision batch
spans the intended range of tangent conditioning (measured on the oracle)."""
import numpy as np

from oracle.oracle_py import OracleModel
from openturbine_b200 import workloads as W


def test_draws_are_seeded():
    a, b = W.draw_batch(16), W.draw_batch(16)
    assert [(x.num_nodes, x.length, x.amp, x.freq) for x in a] == \
        [(x.num_nodes, x.length, x.amp, x.freq) for x in b]
    assert all(5 <= d.num_nodes <= 21 for d in W.draw_batch(200))


def _first_tangent_cond(d, scale):
    o = OracleModel(W.batch_cantilever_model(d, stiffness_scale=scale).pack())
    o.set_node_fx(W.node_fx_for(d, W.tip_loads([d], 0)[0]))
    o.predict_and_assemble(W.batch_params())
    rp, ci, v = o.crs()
    n = len(rp) - 1
    A = np.zeros((n, n))
    for r in range(n):
        A[r, ci[rp[r]:rp[r + 1]]] = v[rp[r]:rp[r + 1]]
    return np.linalg.cond(A)


def test_precision_batch_condition_span():
    """The conditioned system of the first Newton iteration over the EI-swept
    batch spans more than a decade and a half, inside 1e6..1e10."""
    draws = W.draw_batch(24)
    scales = [W.precision_scale(d) for d in draws]
    assert 0.1 <= min(scales) and max(scales) <= 100.0
    conds = [_first_tangent_cond(d, s) for d, s in zip(draws, scales)]
    assert 1e6 <= min(conds) and max(conds) <= 1e10
    assert np.log10(max(conds) / min(conds)) >= 1.5, conds
