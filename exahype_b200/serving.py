"""Continuous-batching serving loop for independent Euler solves.

Requests (dimension, order, cells, problem, steps) arrive over time. The
server keeps every admitted solve resident on the device and keeps all of
them advancing:

* small pulse (unlimited) solves share one :class:`exahype_b200.Batch` --
  instances of one order in common arrays, one CUDA graph launch per step
  for all of them;
* large pulse solves run on their own :class:`exahype_b200.Mesh`, explosion
  solves (a-posteriori limiter) on their own
  :class:`exahype_b200.LimitingMesh`, each on its own stream, so their
  kernels overlap the batch's on the device.

Admission is first-come first-served by device-memory budget: a waiting
request is admitted at the next tick as soon as its state fits beside the
admitted ones; finished solves leave between ticks and free their memory. A
request whose state alone exceeds the budget is rejected. The time to
solution of a request is from its arrival to the moment its result is on the
host.

The process should set CUDA_DEVICE_MAX_CONNECTIONS=32 before CUDA starts:
with the default of 8 hardware queues, kernels of unrelated streams wait
behind each other and neither overlap nor stream priorities work.

Each solve computes exactly what it computes alone (a Mesh or LimitingMesh
of the same problem with the same predictor variant): batching never changes
a result.
"""
import math
import time

import numpy as np

from . import BC_OUTFLOW, BC_PERIODIC, Batch, LimitingMesh, Mesh, Solver, problems


class Request:
    __slots__ = ("rid", "arrival", "dim", "order", "cells", "kind", "steps", "seed", "luh", "fv", "result",
                 "admitted", "finished", "done_steps", "handle", "bytes", "state", "enq", "inflight", "stream")

    def __init__(self, rid, arrival, dim, order, cells, kind, steps, seed):
        self.rid, self.arrival, self.dim, self.order = rid, arrival, dim, order
        self.cells, self.kind, self.steps, self.seed = tuple(cells), kind, steps, seed
        self.luh = self.fv = self.result = self.handle = self.state = None
        self.admitted = self.finished = None
        self.done_steps = self.enq = 0
        self.bytes = 0
        self.inflight, self.stream = [], None

    @property
    def ncells(self):
        return int(np.prod(self.cells))

    @property
    def dof_updates(self):
        return self.ncells * (self.order + 1) ** self.dim * 5 * self.steps

    def build_initial(self):
        if self.luh is not None:
            return
        if self.kind == "explosion":
            self.luh, self.fv, _ = problems.explosion(self.dim, self.order, self.cells, seed=self.seed)
        elif self.dim == 2:
            rng = np.random.default_rng(self.seed)
            amp = float(rng.uniform(0.1, 0.5))
            self.luh, _ = problems.gaussian_pulse_2d(self.order, self.cells, seed=self.seed + 1, amplitude=amp)
        else:
            self.luh, _ = problems.gaussian_pulses_3d(self.order, self.cells, seed=self.seed)


def request_stream(n, rate, seed=0, sides_2d=(27, 243), sides_3d=(9, 81), orders=(3, 5, 7), p3d=0.3,
                   p_limiter=0.2, steps=(10, 200)):
    """n requests with Poisson arrivals at `rate` per second (seeded): 70 % 2D
    with sides in sides_2d, 30 % 3D with sides in sides_3d (log-uniform),
    order uniform in `orders`, 20 % explosions with the limiter (outflow), the
    rest Gaussian pulses (periodic), steps uniform in `steps`."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        dim = 3 if rng.random() < p3d else 2
        lo, hi = sides_3d if dim == 3 else sides_2d
        side = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        order = int(rng.choice(orders))
        kind = "explosion" if rng.random() < p_limiter else "pulse"
        nsteps = int(rng.integers(steps[0], steps[1] + 1))
        out.append(Request(i, t, dim, order, (side,) * dim, kind, nsteps, int(rng.integers(0, 2 ** 31 - 1))))
    return out


def limiting_bytes(dim, order, ncells):
    """device bytes of one LimitingMesh (dense FV patches)"""
    b = order + 1
    P, F = b ** dim, b ** (dim - 1)
    E = 2 * order + 5
    per = 8 * (3 * P * 5 + P * 5 + 2 * 2 * dim * F * 5 + 2 * E ** dim * 5 + 2 * 2 * dim * 5) + 4 * (8 + 2 * dim)
    return ncells * per


def priority_level(dof_updates):
    """stream priority level of a dedicated solve: the less total work, the
    more urgent (4 below 1e9 DoF-updates down to 0 above 3e10)"""
    for level, limit in ((4, 1e9), (3, 3e9), (2, 1e10), (1, 3e10)):
        if dof_updates < limit:
            return level
    return 0


class Server:
    """Serves requests with continuous batching under a device-memory budget.

    Small pulse solves (at most `batch_dof` DoF per step) share the Batch:
    batching pays where single solves are too small to fill the GPU. Larger
    solves and every limiter solve run on their own mesh and stream, at a
    stream priority that is higher the less work the solve has. Work is
    enqueued in chunks of up to `chunk` steps, at most two chunks in flight
    per stream, and completion is polled with CUDA events, so the host never
    waits on one solve while others could be fed."""

    def __init__(self, budget_bytes, variants=None, batch_dof=1 << 18, chunk=8):
        self.budget = int(budget_bytes)
        self.batch = Batch()
        self.batch_stream = None
        self.batch_inflight = []  # (event, [(request, steps done after the chunk)])
        self.solvers = {}
        self.variants = dict(variants or {})
        self.active = []  # admitted, unfinished
        self.used = 0
        self.batch_dof = batch_dof
        self.chunk = chunk
        for (dim, order), v in self.variants.items():  # no autotuning inside the batch
            self.batch.set_variant(dim, order, v)

    def _solver(self, dim, order):
        k = (dim, order)
        if k not in self.solvers:
            s = Solver(dim, order)
            if k in self.variants:
                s.variant = self.variants[k]
            else:
                self.variants[k] = s.autotune(4096)[0]
            self.solvers[k] = s
        return self.solvers[k]

    def bytes_for(self, r):
        if r.kind == "explosion":
            return limiting_bytes(r.dim, r.order, r.ncells)
        return Batch.instance_bytes(r.dim, r.order, r.cells)

    def batched(self, r):
        return r.kind == "pulse" and r.ncells * (r.order + 1) ** r.dim * 5 <= self.batch_dof

    def _admit(self, r, now):
        import torch
        r.build_initial()
        s = self._solver(r.dim, r.order)  # fixes the predictor variant of this order
        r.enq = 0
        r.inflight = []
        if self.batched(r):
            self.batch.set_variant(r.dim, r.order, self.variants[(r.dim, r.order)])
            r.handle = self.batch.add(r.dim, r.order, r.cells, [1.0] * r.dim, BC_PERIODIC, r.luh)
            if self.batch_stream is None:
                self.batch_stream = torch.cuda.ExternalStream(self.batch.stream_handle)
        else:
            if r.kind == "explosion":
                m = LimitingMesh(s, r.cells, [0.0] * r.dim, [1.0] * r.dim, BC_OUTFLOW)
                m.set_solution(r.luh)
                m.set_fv_initial(r.fv)
            else:
                m = Mesh(s, r.cells, [0.0] * r.dim, [1.0] * r.dim, BC_PERIODIC)
                m.set_solution(r.luh)
            # smaller solves first where streams compete for SMs (the batch ranks above all)
            m.set_priority(priority_level(r.dof_updates))
            m.init(0.0)
            r.handle = m
            r.stream = torch.cuda.ExternalStream(m.stream_handle)
        r.admitted = now
        self.used += r.bytes
        self.active.append(r)

    def _finish(self, r, t, keep_results):
        if self.batched(r):
            r.result = self.batch.get_solution(r.handle) if keep_results else None
            r.state = self.batch.state(r.handle)
            self.batch.remove(r.handle)
        else:
            r.result = r.handle.get_solution() if keep_results else None
            r.state = r.handle.state()
            r.handle = None
        r.finished = t
        self.used -= r.bytes
        self.active.remove(r)

    def _feed(self):
        """enqueue chunks where streams have room; returns True if any work was enqueued"""
        import torch
        fed = False
        for r in self.active:
            if self.batched(r):
                continue
            while r.enq < r.steps and len(r.inflight) < 2:
                k = min(self.chunk, r.steps - r.enq)
                r.handle.step(k)
                r.enq += k
                ev = torch.cuda.Event()
                ev.record(r.stream)
                r.inflight.append((ev, r.enq))
                fed = True
        members = [r for r in self.active if self.batched(r)]
        # a batch chunk never runs past the end of any member: a member that
        # reached its steps leaves the batch before the next chunk
        if members and all(r.enq < r.steps for r in members) and len(self.batch_inflight) < 2:
            k = min(self.chunk, min(r.steps - r.enq for r in members))
            self.batch.step(k)
            for r in members:
                r.enq += k
            ev = torch.cuda.Event()
            ev.record(self.batch_stream)
            self.batch_inflight.append((ev, [(r, r.enq) for r in members]))
            fed = True
        return fed

    def _poll(self, t, keep_results):
        done = False
        for r in list(self.active):
            if self.batched(r):
                continue
            while r.inflight and r.inflight[0][0].query():
                r.done_steps = r.inflight.pop(0)[1]
            if r.done_steps >= r.steps:
                self._finish(r, t(), keep_results)
                done = True
        while self.batch_inflight and self.batch_inflight[0][0].query():
            for r, n in self.batch_inflight.pop(0)[1]:
                r.done_steps = n
        for r in list(self.active):
            if self.batched(r) and r.done_steps >= r.steps:
                self._finish(r, t(), keep_results)
                done = True
        return done

    def run(self, requests, clock=time.perf_counter, keep_results=True):
        """Serves `requests` (arrival times in seconds from the start) in real
        time. Returns (requests, rejected); a rejected request's state alone
        exceeds the budget and it keeps finished = None."""
        pending = sorted(requests, key=lambda r: r.arrival)
        for r in pending:
            r.bytes = self.bytes_for(r)
        rejected = [r for r in pending if r.bytes > self.budget]
        queue = [r for r in pending if r.bytes <= self.budget]
        t0 = clock()
        now = lambda: clock() - t0  # noqa: E731
        waiting = []
        while queue or waiting or self.active:
            while queue and queue[0].arrival <= now():
                waiting.append(queue.pop(0))
            # first come, first served while the state fits
            while waiting and self.used + waiting[0].bytes <= self.budget:
                self._admit(waiting.pop(0), now())
            if not self.active:
                if queue:  # idle until the next arrival
                    time.sleep(max(0.0, queue[0].arrival - now()))
                continue
            fed = self._feed()
            done = self._poll(now, keep_results)
            if not fed and not done:
                time.sleep(5e-5)
        return pending, rejected


def run_one_at_a_time(requests, variants, clock=time.perf_counter, keep_results=True):
    """The same requests served one at a time, in arrival order, each on its
    own Mesh / LimitingMesh (the plain FP64 path); each waits for the previous
    one. Returns the requests with finished times (seconds from the start)."""
    pending = sorted(requests, key=lambda r: r.arrival)
    solvers = {}
    t0 = clock()
    for r in pending:
        now = clock() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        r.build_initial()
        k = (r.dim, r.order)
        if k not in solvers:
            solvers[k] = Solver(r.dim, r.order)
            solvers[k].variant = variants[k]
        s = solvers[k]
        if r.kind == "explosion":
            m = LimitingMesh(s, r.cells, [0.0] * r.dim, [1.0] * r.dim, BC_OUTFLOW)
            m.set_solution(r.luh)
            m.set_fv_initial(r.fv)
        else:
            m = Mesh(s, r.cells, [0.0] * r.dim, [1.0] * r.dim, BC_PERIODIC)
            m.set_solution(r.luh)
        m.init(0.0)
        m.step(r.steps)
        r.result = m.get_solution() if keep_results else None
        r.state = m.state()
        r.finished = clock() - t0
        del m
    return pending


def summarise(requests, wall):
    """p50/p99 time to solution (arrival to result on the host) and the
    aggregate DoF-updates/s of the served requests"""
    done = [r for r in requests if r.finished is not None]
    tts = np.array([r.finished - r.arrival for r in done])
    dof = sum(r.dof_updates for r in done)
    return {"requests": len(requests), "served": len(done),
            "p50_s": float(np.percentile(tts, 50)) if len(tts) else None,
            "p99_s": float(np.percentile(tts, 99)) if len(tts) else None,
            "dof_updates": int(dof), "wall_s": wall, "value": dof / wall if wall > 0 else None}
