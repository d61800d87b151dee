"""Per-phase SM cycles of the step kernel (tracing).

    python -m openturbine_b200.phase_profile --beams 2048 --steps 3 --nodes 13 [--precision 1]

Creates a batch of cantilevers (uniform node count, or the mixed batch with
--nodes 0), takes two untimed steps, switches on KYN_OPT_PHASE_TIMING and
prints the SM cycles per beam and Newton iteration of each kernel phase (one
CTA's clock, summed over beams by the kernel).  Phase "factor" is the whole
Gauss-Jordan elimination (--solver 0) or the panel LU's barrier wait
(--solver 1, whose own sub-phases follow as lu_*).
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import workloads as W
from .runtime import LOAD_NODE_FX, OPT_LINEAR_SOLVER, OPT_PHASE_TIMING, Context

PHASES = ["load_predict", "quadrature", "integrate_gemm", "constraints", "eliminate",
          "factor", "substitute", "update", "store", "lu_warp0_next_rows",
          "lu_warp0_diag_factor", "lu_l21_all_threads", "refine"]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--beams", type=int, default=2048)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--nodes", type=int, default=13, help="0: the mixed batch (U{5..21})")
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--solver", type=int, default=1,
                    help="1: panel LU (default), 0: Gauss-Jordan in registers where it fits")
    ap.add_argument("--bulk-sections", type=int, default=1,
                    help="1: sections staged by one bulk copy per iteration, 0: per-point loads")
    args = ap.parse_args()
    ctx = Context(0)
    ctx.lib.kyn_ctx_set_option(ctx.h, OPT_LINEAR_SOLVER, args.solver)
    ctx.set_bulk_sections(bool(args.bulk_sections))
    draws = W.draw_batch(args.beams)
    if args.nodes:
        draws = [W.BeamDraw(d.model_id, args.nodes, d.length, d.amp, d.freq) for d in draws]
    ids = np.array([ctx.create_model(W.batch_cantilever_model(d).pack()) for d in draws],
                   dtype=np.int32)
    p = W.batch_params()
    p.precision = args.precision

    def step(k):
        fx = np.concatenate([W.node_fx_for(d, f) for d, f in zip(draws, W.tip_loads(draws, k))])
        ctx.set_loads_batch(ids, LOAD_NODE_FX, fx.ctypes.data, False)
        return ctx.step(ids, p)

    for k in range(2):
        step(k)
    ctx.lib.kyn_ctx_set_option(ctx.h, OPT_PHASE_TIMING, 1)
    iters = 0
    for k in range(2, 2 + args.steps):
        _, it = step(k)
        iters += int(it.sum())
    cyc = [ctx.stat(100 + i) for i in range(len(PHASES))]
    print(json.dumps({"beams": args.beams, "nodes": args.nodes or "mixed",
                      "precision": args.precision, "solver": args.solver,
                      "bulk_sections": args.bulk_sections,
                      "beam_iterations": iters,
                      "cycles_per_beam_iteration": {n: round(c / max(iters, 1))
                                                    for n, c in zip(PHASES, cyc)}}))
    ctx.close()


if __name__ == "__main__":
    main()
