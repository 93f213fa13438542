"""BCLP on many independent targets at once (targets of uneven size).

``MultiTargetBCLP`` runs one BCLP problem per target -- each with its own
geometry, angle count, absorption and response options, exactly as
``BCLPNorm`` (vamtoolbox/optimizer/BCLP.py:277-534) runs it -- but issues the
projections of all targets together: every iteration is one batched
backprojection (all targets' g -> dose in persistent launches), the
per-target fused dose passes, one batched forward (all operands -> gradients),
and the per-target clamped updates, all captured once in a CUDA graph.  Each
target's sequence of operations is the one its own ``DeviceIteration`` issues,
so the per-target results equal running the targets one at a time.
"""
from __future__ import annotations

import torch

from ..batch import ProjectionBatch
from ..fused import capture
from .BCLP import BCLPNorm


class MultiTargetBCLP:
    """problems: sequence of (target_geo, proj_geo, options), parallel-beam projectors.

    schedule:
      "persistent" -- per iteration one batched backprojection and one batched
                      forward over all targets (vam_batch_submit: a persistent
                      launch per kernel-body family, the families on forked
                      streams), with the per-target fused passes between, each
                      on its target's stream;
      "streams"    -- each target's whole iteration chain on its own stream inside
                      the graph, so the hardware interleaves the targets' own
                      specialised kernels with no barrier between phases;
      "auto"       -- time one captured iteration of each and keep the faster.
    """

    def __init__(self, problems, schedule="auto"):
        if schedule not in ("auto", "persistent", "streams"):
            raise ValueError(f"unknown schedule {schedule!r}")
        self.solvers = [BCLPNorm(tg, pg, o) for tg, pg, o in problems]
        if not self.solvers:
            raise ValueError("MultiTargetBCLP needs at least one problem")
        for s in self.solvers:
            plan = getattr(s.P, "plan", None)
            if plan is None or not hasattr(plan, "backward_ref"):
                raise NotImplementedError("MultiTargetBCLP batches parallel-beam projectors only")
        self.its = [s.device_iteration() for s in self.solvers]
        self.device = self.its[0].device
        if any(it.device != self.device for it in self.its):
            raise ValueError("all targets of a MultiTargetBCLP must live on one device")
        self.back = ProjectionBatch(self.device)
        self.fwd = ProjectionBatch(self.device)
        self.back_work = [(it.bclp.P.plan, "backward_ref", it.g, it.dose) for it in self.its]
        self.fwd_work = [(it.bclp.P.plan, "forward", it.operand, it.grad) for it in self.its]
        self.streams = [torch.cuda.Stream(device=self.device) for _ in self.its]
        self.fork = torch.cuda.Event()
        self.joins = [torch.cuda.Event() for _ in self.its]
        self.schedule = schedule
        self.timings = None
        if schedule == "auto":
            self.schedule = self._pick()

    # -- persistent schedule: phases over all targets
    # (the per-target passes between the batched launches run on the targets' own streams, so
    # the small ones overlap instead of queueing one after another)
    def state(self):
        self.back.submit(self.back_work)
        self._fork_join(self._dose)

    def update(self):
        self.fwd.submit(self.fwd_work)
        self._fork_join(self._update)

    @staticmethod
    def _dose(it):
        it.ws.bclp_dose_pass(it.dose, it.fT, it.prm, it.mapped, it.operand, it.stats)
        it.ws.append(it.stats, it.log, it.counter)

    @staticmethod
    def _update(it):
        b = it.bclp
        it.ws.bclp_update(it.g, it.grad, b.learning_rate, b.p, b.q, b.glb, b.gub, it.stats)

    # -- streams schedule: one chain per target, forked from and joined to the current stream
    def _fork_join(self, fn):
        main = torch.cuda.current_stream(self.device)
        self.fork.record(main)
        for it, s, ev in zip(self.its, self.streams, self.joins):
            s.wait_event(self.fork)
            with torch.cuda.stream(s):
                fn(it)
            ev.record(s)
        for ev in self.joins:
            main.wait_event(ev)

    def step(self):
        if self.schedule == "persistent":
            self.state()
            self.update()
        else:
            self._fork_join(lambda it: it.step())

    def capture(self):
        """The whole multi-target iteration as one CUDA graph (lists validated first, nothing run)."""
        self.back.prepare(self.back_work)
        self.fwd.prepare(self.fwd_work)
        return capture(self.step, self.device)

    def _pick(self, reps=3):
        """Time both schedules on captured iterations from the same starting sinograms; keep the faster."""
        saved = [it.g.clone() for it in self.its]
        st = torch.cuda.current_stream(self.device)
        times = {}
        for sched in ("persistent", "streams"):
            self.schedule = sched
            gr = self.capture()
            gr.replay()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(reps):
                gr.replay()
            e1.record(st)
            e1.synchronize()
            times[sched] = e0.elapsed_time(e1) / reps
            del gr
            for it, g in zip(self.its, saved):
                it.g.copy_(g)
                it.counter.zero_()
                it.log.fill_(float("nan"))
        torch.cuda.synchronize(self.device)
        self.timings = times
        return min(times, key=times.get)

    def run(self, n_iter=None, graph=True):
        """Iterate every target ``n_iter`` times (default: each problem's options.n_iter, which must agree);
        returns the per-target (sinogram, dose, loss log) like ``BCLPNorm.gradientDescent``."""
        if n_iter is None:
            counts = {s.logs.options.n_iter for s in self.solvers}
            if len(counts) != 1:
                raise ValueError("problems disagree on n_iter; pass n_iter explicitly")
            n_iter = counts.pop()
        st = torch.cuda.current_stream(self.device)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(n_iter + 1)]
        ev[0].record(st)
        if graph:
            gr = self.capture()
            for k in range(n_iter):
                gr.replay()
                ev[k + 1].record(st)
            del gr
        else:
            for k in range(n_iter):
                self.step()
                ev[k + 1].record(st)
        self.state()  # the final dose of every target (persistent schedule's first phase)
        torch.cuda.synchronize(self.device)
        times = [ev[0].elapsed_time(ev[k + 1]) / 1e3 for k in range(n_iter)]
        out = []
        for s, it in zip(self.solvers, self.its):
            g = s.finish_device(it, n_iter, times)
            out.append((s.checkSinogramShape(g, "cylindrical"), s.dose, s.logs.loss))
        return out
