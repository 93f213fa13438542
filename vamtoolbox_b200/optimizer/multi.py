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
      "phased"     -- the targets in two halves (A, B, alternating by cost) with B
                      half an iteration ahead: each persistent batch holds A's
                      backprojections with B's forwards, then A's forwards with
                      B's backprojections, so both kernel-body families share the
                      device in every phase; every target still runs back, dose
                      pass, forward, update in its own order (B's first state is
                      computed before the loop, A's last one after it);
      "auto"       -- time one captured iteration of each and keep the fastest.
    """

    def __init__(self, problems, schedule="auto"):
        if schedule not in ("auto", "persistent", "streams", "phased"):
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
        # phased schedule: halves by cost (largest first, alternating), their mixed batch lists
        cost = [it.g.numel() * it.dose.shape[-1] for it in self.its]
        order = sorted(range(len(self.its)), key=lambda k: -cost[k])
        self.half_a = [self.its[k] for k in order[0::2]]
        self.half_b = [self.its[k] for k in order[1::2]]
        self.phase1 = ProjectionBatch(self.device)
        self.phase2 = ProjectionBatch(self.device)
        back = lambda it: (it.bclp.P.plan, "backward_ref", it.g, it.dose)
        fwd = lambda it: (it.bclp.P.plan, "forward", it.operand, it.grad)
        self.phase1_work = [back(it) for it in self.half_a] + [fwd(it) for it in self.half_b]
        self.phase2_work = [fwd(it) for it in self.half_a] + [back(it) for it in self.half_b]
        self._b_primed = False
        self.schedule = schedule
        self.timings = None
        if schedule == "auto":
            self.schedule = self._pick()

    # -- persistent schedule: phases over all targets
    # (the per-target passes between the batched launches run on the targets' own streams, so
    # the small ones overlap instead of queueing one after another)
    @staticmethod
    def _zero_dose(its):
        # the targets' zero-dose sinogram entries set to 0 before their batched backprojections, as each
        # target's own projector does (nothing is launched for a target without a zero-dose region)
        for it in its:
            zd = getattr(it.bclp.P, "zero_dose_", None)
            if zd is not None:
                zd(it.g)

    def state(self):
        self._zero_dose(self.its)
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

    def _fork_join_over(self, its, fn):
        main = torch.cuda.current_stream(self.device)
        self.fork.record(main)
        for k, it in enumerate(its):
            s, ev = self.streams[k], self.joins[k]
            s.wait_event(self.fork)
            with torch.cuda.stream(s):
                fn(it)
            ev.record(s)
        for ev in self.joins[:len(its)]:
            main.wait_event(ev)

    def prime(self):
        """Phased schedule: half B's first backprojection and dose pass (its state for iteration 0),
        issued once before the loop; a no-op when already issued."""
        if self._b_primed or not self.half_b:
            self._b_primed = True
            return
        for it in self.half_b:
            it.back(it.g, it.dose)
        self._fork_join_over(self.half_b, self._dose)
        self._b_primed = True

    def step(self):
        if self.schedule == "persistent":
            self.state()
            self.update()
        elif self.schedule == "phased":
            self._zero_dose(self.half_a)
            self.phase1.submit(self.phase1_work)
            self._fork_join_over(self.half_a, self._dose)
            self._fork_join_over(self.half_b, self._update)
            self._zero_dose(self.half_b)
            self.phase2.submit(self.phase2_work)
            self._fork_join_over(self.half_a, self._update)
            self._fork_join_over(self.half_b, self._dose)
        else:
            self._fork_join(lambda it: it.step())

    def finish_state(self):
        """The final dose of every target after the loop: all targets' (persistent / streams) or half
        A's (phased: half B's is the last phase of the loop)."""
        if self.schedule == "phased":
            for it in self.half_a:
                it.back(it.g, it.dose)
            self._fork_join_over(self.half_a, self._dose)
        else:
            self.state()

    def capture(self):
        """The whole multi-target iteration as one CUDA graph (lists validated first, nothing run).
        The phased schedule's half B is primed on the current stream first (outside the graph)."""
        self.back.prepare(self.back_work)
        self.fwd.prepare(self.fwd_work)
        if self.schedule == "phased":
            self.phase1.prepare(self.phase1_work)
            self.phase2.prepare(self.phase2_work)
            self.prime()
        return capture(self.step, self.device)

    def reset(self, saved):
        """Restore every target's sinogram and log (and the phased schedule's priming) to a saved start."""
        for it, g in zip(self.its, saved):
            it.g.copy_(g)
            it.counter.zero_()
            it.log.fill_(float("nan"))
        self._b_primed = False

    def _pick(self, reps=3):
        """Time the schedules on captured iterations from the same starting sinograms; keep the fastest."""
        saved = [it.g.clone() for it in self.its]
        st = torch.cuda.current_stream(self.device)
        times = {}
        for sched in ("persistent", "streams", "phased"):
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
            self.reset(saved)
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
        if self.schedule == "phased":
            self.prime()
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
        self.finish_state()  # the final dose of every target
        torch.cuda.synchronize(self.device)
        times = [ev[0].elapsed_time(ev[k + 1]) / 1e3 for k in range(n_iter)]
        out = []
        for s, it in zip(self.solvers, self.its):
            g = s.finish_device(it, n_iter, times)
            out.append((s.checkSinogramShape(g, "cylindrical"), s.dose, s.logs.loss))
        return out
