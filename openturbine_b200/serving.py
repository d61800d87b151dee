"""Continuous-batching step server for resident beam and rotor models.

Requests (a model description, a number of time steps and a load schedule)
arrive over time.  The server keeps every admitted model's state resident on
the device and runs iterations: each iteration advances every admitted model
by one time step in one batched kyn_step call, and while that step runs on the
GPU the host admits newly arrived requests (as the HBM budget and the slot
limit allow) and prepares the next iteration's loads.  A model leaves the
batch when its requested steps are done; its final state is read back first.

Per model the arithmetic does not depend on which other models share the
batch, so a request's result is the same alone and in any mix.

Loads follow the benchmark workloads: a single beam gets a tip force
amp*sin(2 pi f t) along z; a rotor's three blade roots follow the hub rotation
exp(omega t z) as prescribed motion (the reference's turbine interface sets
both per step, src/interfaces/turbine/turbine_interface.cpp:117-150).
"""
from __future__ import annotations

import gc
import math
import time
from dataclasses import dataclass, field

import numpy as np

from .runtime import LOAD_NODE_FX, Context, KynError

KYN_ERR_BUDGET = -4


@dataclass
class Request:
    """A model to advance `steps` time steps.

    kind "beam": `packed` is one beam element with a fixed root; the tip
    (its last element node) gets amp*sin(2 pi freq t).  kind "rotor": three
    blades whose roots follow the hub rotation at `omega` rad/s; `roots`
    holds the root reference positions [3][3]."""
    rid: int
    kind: str
    packed: object
    nodes: int                  # element nodes of the model (rows of node_FX)
    steps: int
    amp: float = 0.0
    freq: float = 0.0
    omega: float = 0.0
    roots: np.ndarray | None = None
    arrival: float = 0.0
    # filled by the server
    model_id: int = -1
    done: int = 0
    admitted_at: float = math.nan
    finished_at: float = math.nan
    statuses: list = field(default_factory=list)   # (step, status) of non-converged steps
    final_q: np.ndarray | None = None


class StepServer:
    """One context, one GPU.  `params` applies to every model (one kyn_step).

    The active set is kept as arrays (model ids, load parameters, step
    counters, node-row offsets), so building one iteration's loads and
    bookkeeping costs a few vector operations, not a pass over Python
    objects; only admitted and finishing requests are touched one by one.

    Requests that carry the same (pooled) model description share one
    resident template model: the first one builds it, every admission clones
    it on the device (kyn_model_clone), so admitting costs a device copy, not
    a rebuild of shape tables, sections and CRS graph.  Templates count
    against the HBM budget and are never stepped."""

    def __init__(self, ctx: Context, params, h: float = 0.01, max_active: int | None = None,
                 reserve_rows: int = 16384 * 22):
        self.ctx = ctx
        self.params = params
        self.h = h
        self.max_active = max_active
        self.queue: list[Request] = []
        self.active: list[Request] = []       # same order as the arrays below
        self.finished: list[Request] = []
        self.step_ms: list[float] = []        # iteration wall time (submit -> results)
        self.step_models: list[int] = []      # models advanced by that iteration
        self.beam_steps_converged = 0
        self.beam_steps_total = 0
        self.max_active_seen = 0
        # host time per iteration part (ms, summed): loads and motion in, step
        # submission, admission while the step runs, wait for results, retire
        self.host_ms = {"inputs": 0.0, "submit": 0.0, "admit": 0.0, "wait": 0.0, "retire": 0.0}
        # pinned staging of the per-iteration loads, sized up front: growing it
        # (a page-locked allocation) inside the loop stalls an iteration
        import torch
        self._pinned = torch.zeros((max(int(reserve_rows), 1024), 6), dtype=torch.float64).pin_memory()
        self._templates: dict = {}      # id(packed description) -> resident template model
        self._template_refs: list = []  # keeps those descriptions alive (their ids stay unique)
        self._ids = np.zeros(0, dtype=np.int32)
        self._rotor = np.zeros(0, dtype=bool)
        self._amp = np.zeros(0)
        self._freq = np.zeros(0)
        self._omega = np.zeros(0)
        self._done = np.zeros(0, dtype=np.int64)
        self._steps = np.zeros(0, dtype=np.int64)
        self._nodes = np.zeros(0, dtype=np.int64)
        self._roots = np.zeros((0, 3, 3))

    # ---- admission -------------------------------------------------------------
    def submit(self, req: Request) -> None:
        self.queue.append(req)

    def _admit(self, now: float) -> None:
        keep, new = [], []
        blocked = False
        for r in self.queue:
            if blocked or r.arrival > now or (self.max_active and len(self.active) + len(new) >= self.max_active):
                keep.append(r)
                continue
            try:
                r.model_id = self._new_model(r.packed)
            except KynError as e:
                if e.code != KYN_ERR_BUDGET:
                    raise
                # the templates are a cache: give their memory back and build
                # this model directly before waiting for active models to leave
                try:
                    if not self._templates:
                        raise
                    self._drop_templates()
                    r.model_id = self.ctx.create_model(r.packed)
                except KynError as e2:
                    if e2.code != KYN_ERR_BUDGET:
                        raise
                    blocked = True  # wait for memory to free up
                    keep.append(r)
                    continue
            r.admitted_at = now
            new.append(r)
        self.queue = keep
        if new:
            self.active.extend(new)
            self._ids = np.concatenate([self._ids, np.array([r.model_id for r in new], dtype=np.int32)])
            self._rotor = np.concatenate([self._rotor, np.array([r.kind == "rotor" for r in new])])
            self._amp = np.concatenate([self._amp, [r.amp for r in new]])
            self._freq = np.concatenate([self._freq, [r.freq for r in new]])
            self._omega = np.concatenate([self._omega, [r.omega for r in new]])
            self._done = np.concatenate([self._done, np.array([r.done for r in new], dtype=np.int64)])
            self._steps = np.concatenate([self._steps, np.array([r.steps for r in new], dtype=np.int64)])
            self._nodes = np.concatenate([self._nodes, np.array([r.nodes for r in new], dtype=np.int64)])
            self._roots = np.concatenate(
                [self._roots, np.stack([r.roots if r.roots is not None else np.zeros((3, 3)) for r in new])])

    def _new_model(self, packed) -> int:
        """First request of a description builds a resident template; every
        request then gets a device copy of it."""
        tid = self._templates.get(id(packed))
        if tid is None:
            tid = self.ctx.create_model(packed)
            self._templates[id(packed)] = tid
            self._template_refs.append(packed)
        return self.ctx.clone_model(tid)

    def _drop_templates(self) -> None:
        for tid in self._templates.values():
            self.ctx.destroy_model(tid)
        self._templates.clear()
        self._template_refs.clear()

    def _remove(self, idx: np.ndarray) -> None:
        keep = np.ones(len(self.active), dtype=bool)
        keep[idx] = False
        self.active = [r for r, k in zip(self.active, keep) if k]
        for name in ("_ids", "_rotor", "_amp", "_freq", "_omega", "_done", "_steps", "_nodes", "_roots"):
            setattr(self, name, getattr(self, name)[keep])

    # ---- per-iteration inputs -----------------------------------------------------
    def _loads(self, n: int):
        nodes = self._nodes[:n]
        rows = int(nodes.sum())
        if self._pinned.shape[0] < rows:
            import torch
            self._pinned = torch.zeros((2 * rows, 6), dtype=torch.float64).pin_memory()
        fx = self._pinned.numpy()[:rows]
        fx[:] = 0.0
        t = self.h * (self._done[:n] + 1)
        rotor = self._rotor[:n]
        beam = ~rotor
        tip = np.cumsum(nodes) - 1
        fx[tip[beam], 2] = self._amp[:n][beam] * np.sin(2.0 * np.pi * self._freq[:n][beam] * t[beam])
        presc, rot_ids = None, None
        rot = np.flatnonzero(rotor)
        if rot.size:
            ang = self._omega[rot] * t[rot]                              # [R]
            c, s = np.cos(ang)[:, None], np.sin(ang)[:, None]
            x0 = self._roots[rot]                                        # [R][3][3]
            vals = np.zeros((rot.size, 3, 7))
            vals[:, :, 0] = c * x0[:, :, 0] - s * x0[:, :, 1] - x0[:, :, 0]
            vals[:, :, 1] = s * x0[:, :, 0] + c * x0[:, :, 1] - x0[:, :, 1]
            vals[:, :, 3] = np.cos(ang / 2.0)[:, None]
            vals[:, :, 6] = np.sin(ang / 2.0)[:, None]
            presc = np.ascontiguousarray(vals.reshape(-1, 7))
            rot_ids = np.ascontiguousarray(self._ids[rot])
        return fx, presc, rot_ids

    # ---- one iteration ------------------------------------------------------------
    def iterate(self, now_fn) -> None:
        if not self.active:
            self._admit(now_fn())
            return
        n = len(self.active)
        ids = np.ascontiguousarray(self._ids[:n])
        fx, presc, rot_ids = self._loads(n)
        t0 = time.perf_counter()
        self.ctx.set_loads_batch(ids, LOAD_NODE_FX, fx.ctypes.data, False)
        if presc is not None:
            self.ctx.set_prescribed_batch(rot_ids, presc.ctypes.data, False)
        t1 = time.perf_counter()
        self.ctx.step_async(ids, self.params)
        t2 = time.perf_counter()
        self._admit(now_fn())               # overlaps the step on the GPU (appends after n)
        t3 = time.perf_counter()
        st, it = self.ctx.step_wait()
        t4 = time.perf_counter()
        self.step_ms.append((t4 - t0) * 1e3)
        for k, dt in (("inputs", t1 - t0), ("submit", t2 - t1), ("admit", t3 - t2), ("wait", t4 - t3)):
            self.host_ms[k] += dt * 1e3
        self.step_models.append(n)
        self.max_active_seen = max(self.max_active_seen, n)
        conv = st == 0
        nb = np.where(self._rotor[:n], 3, 1)
        self.beam_steps_total += int(nb.sum())
        self.beam_steps_converged += int(nb[conv].sum())
        for i in np.flatnonzero(~conv):     # the rare non-converged model-steps
            self.active[i].statuses.append((int(self._done[i]), int(st[i])))
        self._done[:n] += 1
        leave = np.flatnonzero(self._done[:n] >= self._steps[:n])
        if leave.size:
            t5 = time.perf_counter()
            now = now_fn()
            # final displacements of all leaving models in one batched read
            lids = np.ascontiguousarray(self._ids[leave])
            rows = [self.ctx.info(int(mid)).num_nodes for mid in lids]
            qall = np.empty((sum(rows), 7))
            self.ctx.get_state_batch(lids, "q", qall.ctypes.data, False)
            start = 0
            for i, nr in zip(leave, rows):
                r = self.active[i]
                r.done = int(self._done[i])
                r.final_q = qall[start:start + nr].copy()
                start += nr
                self.ctx.destroy_model(r.model_id)
                r.finished_at = now
                self.finished.append(r)
            self._remove(leave)
            self.host_ms["retire"] += (time.perf_counter() - t5) * 1e3

    def run(self, until_s: float, drain: bool = False) -> None:
        """Serve in real time for until_s seconds (requests become visible at
        their arrival times); with drain, then finish every admitted model."""
        # The request objects and model descriptions made before serving stay
        # alive throughout; keep the cyclic collector from walking them inside an
        # iteration (a full collection over them stalls the loop).
        gc.freeze()
        t_start = time.perf_counter()
        now = lambda: time.perf_counter() - t_start  # noqa: E731
        while now() < until_s:
            if not self.active and not any(r.arrival <= now() for r in self.queue):
                if not self.queue:
                    break
                time.sleep(min(0.001, max(0.0, min(r.arrival for r in self.queue) - now())))
            self.iterate(now)
        if drain:
            while self.active or self.queue:
                if not self.active:
                    self._admit(float("inf"))
                    if not self.active:
                        raise KynError(KYN_ERR_BUDGET, "a queued model does not fit the HBM budget")
                self.iterate(lambda: float("inf"))

    def summary(self) -> dict:
        ms = np.repeat(np.asarray(self.step_ms), np.asarray(self.step_models)) if self.step_ms else np.zeros(1)
        wall = float(np.sum(self.step_ms)) * 1e-3 if self.step_ms else 0.0
        return {"iterations": len(self.step_ms),
                "model_steps": int(np.sum(self.step_models)) if self.step_models else 0,
                "beam_steps_converged": self.beam_steps_converged,
                "beam_steps_total": self.beam_steps_total,
                "converged_beam_steps_per_s": self.beam_steps_converged / wall if wall else 0.0,
                "step_latency_ms": {"p50": float(np.percentile(ms, 50)),
                                    "p99": float(np.percentile(ms, 99))},
                "max_active": self.max_active_seen,
                "host_ms_total": {k: round(v, 1) for k, v in self.host_ms.items()},
                "active_end": len(self.active), "queued_end": len(self.queue),
                "finished": len(self.finished)}


# ---- synthetic request stream (Poisson arrivals, beams and rotors) ---------------
def request_pool(n_beams: int, n_rotors: int, first_id: int = 7_000_000):
    """Packed model descriptions reused by the request stream (packing is the
    client's work and stays out of the served loop)."""
    from . import workloads as W
    beams = []
    for d in W.draw_batch(n_beams, first_id=first_id):
        beams.append((W.batch_cantilever_model(d).pack(), d.num_nodes))
    rotors = []
    spec = W.RotorSpec()
    roots = np.array([[spec.hub_radius * math.cos(2 * math.pi * b / 3),
                       spec.hub_radius * math.sin(2 * math.pi * b / 3), 0.0] for b in range(3)])
    for k in range(n_rotors):
        m, _ = W.rotor_model(first_id + n_beams + k, spec)
        rotors.append((m.pack(), 3 * spec.num_nodes, roots, spec.omega))
    return beams, rotors


def poisson_requests(rate: float, duration: float, beams, rotors, rotor_fraction: float = 0.1,
                     steps_lo: int = 50, steps_hi: int = 500, seed: int = 20261203) -> list[Request]:
    """Arrivals at `rate` per second for `duration` seconds; each request picks a
    pooled model, U{steps_lo..steps_hi} steps and (beams) a tip load with
    amplitude U(1e3, 1e5) N and frequency U(0.1, 5) Hz."""
    rng = np.random.default_rng(seed)
    t, out, rid = 0.0, [], 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        steps = int(rng.integers(steps_lo, steps_hi + 1))
        if rotors and rng.random() < rotor_fraction:
            packed, nodes, roots, omega = rotors[int(rng.integers(len(rotors)))]
            out.append(Request(rid, "rotor", packed, nodes, steps, omega=omega, roots=roots, arrival=t))
        else:
            packed, nodes = beams[int(rng.integers(len(beams)))]
            out.append(Request(rid, "beam", packed, nodes, steps, amp=float(rng.uniform(1e3, 1e5)),
                               freq=float(rng.uniform(0.1, 5.0)), arrival=t))
        rid += 1
    return out
