"""Band-constrained Lp-norm minimisation (BCLP): the reference's vamtoolbox/optimizer/BCLP.py.

Iteration (BCLP.py:277-386, 477-534), with P the projector:
    dose = P.backward(g); mapped = response(dose); e = mapped - f_T
    eb = |e| - eps; v = eb > 0; loss = (sum v w |eb|^p)^(q/p)
    grad = q loss^((q-p)/q) P.forward(v w |eb|^(p-1) sign(e) dresponse(dose))   (no prefactor if loss == 0)
    g <- clip(g - lr grad, blb, bub)
For the parallel beam, P.backward is the reference-parity backprojection
(not the transpose of P.forward), exactly as the reference pairs them.

engine="device": g, dose and every intermediate stay on the GPU; one
iteration is five kernel launches (backprojection, fused dose pass with the
loss / norm reductions, log append, forward projection, fused clamped
update) captured once into a CUDA graph and replayed n_iter times; the loss
scalar never leaves the device (the prefactor and the loss == 0 branch are a
select inside the update kernel).  engine="host" is the reference's numpy
loop calling the projector with host arrays (the plain per-call path).
"""
from __future__ import annotations

import logging
import time
import warnings

import numpy as np
import torch

from .. import geometry
from ..fused import Workspace, bclp_params, capture, to_device_f64, to_host_f64
from ..projectorconstructor import projectorconstructor
from ..util import data as udata


class LogPerf:
    """Per-iteration loss and norm log (BCLP.py:14-135)."""

    def __init__(self, options):
        self.options = options
        self.curr_iter = 0
        n = options.n_iter + 1
        for k in ("loss", "l0", "l1", "l2", "lf", "l0_eps0", "l1_eps0", "l2_eps0", "lf_eps0", "ver"):
            setattr(self, k, np.full(n, np.nan))
        self.iter_times = np.zeros(n)
        self.t0 = np.nan
        self.is_converged = False

    def startTiming(self):
        self.t0 = time.perf_counter()

    def recordIterTime(self):
        self.iter_times[self.curr_iter] = time.perf_counter() - self.t0

    def show(self, *args, **kwargs):
        """The reference plots the loss and norm histories (BCLP.py:94-135); this package has no display:
        it logs that nothing is drawn and returns (the histories are the arrays on this object)."""
        logging.getLogger(__name__).warning("LogPerf.show(): no display in this package; see .loss, .l0 ... .lf_eps0")

    def save(self, filename):
        np.savetxt(filename, np.column_stack([range(self.options.n_iter + 1), self.iter_times, self.loss, self.l0,
                                              self.l1, self.l2, self.lf, self.l0_eps0, self.l1_eps0, self.l2_eps0,
                                              self.lf_eps0]), delimiter=",",
                   header="n,compute time,loss,L0 norm,L1 norm,L2 norm,Linf norm,L0 norm eps=0,L1 norm eps=0,"
                          "L2 norm eps=0,Linf norm eps=0,",
                   fmt=["%5.0i"] + ["%10.2f"] + ["%10.4f"] * 9)

    def fill_from_stats(self, stats, q, p, upto):
        """stats: [rows, 9] float array from vam_bclp_dose_pass."""
        s = np.asarray(stats, dtype=np.float64)[:upto]
        n = s.shape[0]
        self.loss[:n] = s[:, 0] ** (q / p)
        self.l0[:n], self.l0_eps0[:n] = s[:, 1], s[:, 2]
        self.l1[:n], self.l1_eps0[:n] = s[:, 3], s[:, 4]
        self.l2[:n], self.l2_eps0[:n] = np.sqrt(s[:, 5]), np.sqrt(s[:, 6])
        self.lf[:n], self.lf_eps0[:n] = s[:, 7], s[:, 8]


class BCLPNorm:
    def __init__(self, target_geo, proj_geo, options):
        self.logger = logging.getLogger(__name__)
        self.target_geo = target_geo
        self.target_geo.array = np.atleast_3d(self.target_geo.array)
        self.proj_geo = proj_geo
        self.options = options
        self.logs = LogPerf(options)
        self.logs.startTiming()
        self.response_model = options.response_model
        self.eps, self.weight = options.eps, options.weight
        self.p, self.q = options.p, options.q
        self.learning_rate = options.learning_rate
        self.optim_alg = options.optim_alg
        self.g0 = options.g0
        self.glb, self.gub = options.blb, options.bub
        self.bit_depth = options.bit_depth
        self.dvol = 1
        self.exit_param = options.exit_param
        self.verbose = options.verbose
        self.test_alternate_handling = getattr(options, "test_alternate_handling", False)
        self.dose = None
        self._mapped_dose = None
        self.mapped_t = None
        # state of the reference's step interface (updateVariables: each quantity computed once per
        # iteration index, BCLP.py:203-216)
        self.v = self.loss = self.loss_grad = None
        self.mapped_dose_error_from_f_T = self.mapped_dose_error_from_band = None
        self.dose_iter = self.mapped_dose_iter = self.mapped_dose_error_from_f_T_iter = -1
        self.mapped_dose_error_from_band_iter = self.v_iter = self.weight_iter = -1
        self.loss_iter = self.loss_grad_iter = -1
        self.g0_t = self.fT_t = None
        self.P = projectorconstructor(self.target_geo, self.proj_geo)
        if self._device_init_ok():
            self._init_device()
            return
        if self.response_model.checkResponseTarget(self.target_geo.array) is False:
            warnings.warn("Target is either out of range of response function over non-negative real dose input, "
                          "or contains inf/nan.")
        if self.g0 is None:
            f0 = self.response_model.map_inv(self.target_geo.array)
            if callable(getattr(self.P, "inverseBackward", None)):
                self.g0 = self.P.inverseBackward(f0, filter_option=options.filter)
            elif hasattr(getattr(self.P, "plan", None), "backward_ref"):  # parallel beam: cuFFT filter on the device
                g0 = udata.filterSinogram_t(self.P.forward_t(f0).to(torch.float64), options.filter)
                self.g0 = (g0 * (np.pi / (2 * proj_geo.n_angles))).cpu().numpy()
            else:
                self.g0 = udata.filterSinogram(self.P.forward(f0), options.filter)
                self.g0 *= np.pi / (2 * proj_geo.n_angles)
        self.g0 = np.asarray(self.g0)
        self.g0_shape = self.g0.shape
        self.g0 = self.imposeSinogramConstraints(self.g0)

    # -- device-resident set-up (engine="device", parallel beam) -------------------
    def _device_init_ok(self):
        """The target, the initial sinogram and the constraints stay on the device when the device engine
        runs a parallel-beam plan with a device response form and no bit-depth quantisation."""
        return (getattr(self.options, "engine", "device") == "device" and self.bit_depth is None
                and hasattr(getattr(self.P, "plan", None), "backward_ref") and self._device_response_ok()
                and getattr(self.response_model, "device_map_inv_ok", lambda: False)())

    def _init_device(self):
        """BCLP.py's set-up (response-target check, g0 = filter(forward(map_inv(f_T))) * pi / (2 n_angles),
        imposeSinogramConstraints) on the device: the float64 target is uploaded once, the checks reduce
        on the device, and g0 is filtered, scaled and clipped into a float32 device tensor (no host
        round trip of the 3-D arrays)."""
        dev = self.P.device
        tgt = to_device_f64(self.target_geo.array, dev)
        if self.response_model.checkResponseTarget_t(tgt) is False:
            warnings.warn("Target is either out of range of response function over non-negative real dose input, "
                          "or contains inf/nan.")
        self.fT_t = tgt.to(torch.float32)
        n_angles = self.proj_geo.n_angles
        if self.g0 is None:
            f0 = self.response_model.map_inv_t(tgt)
            b = self.P.forward_t(f0)
            g0 = udata.filterSinogram_t(b, self.options.filter, scale=np.pi / (2 * n_angles), lo=self.glb, hi=self.gub)
        else:
            g0 = torch.as_tensor(np.asarray(self.g0)).to(dev, torch.float32).reshape(self.P.plan.shape_sino)
            if self.glb is not None or self.gub is not None:
                g0 = g0.clamp(min=self.glb, max=self.gub)
        self.g0_t = g0.contiguous()
        self.g0_shape = tuple(self.g0_t.shape)
        self.g0 = None  # the host copy is made on demand (host_g0)

    def host_g0(self):
        """The initial sinogram as a host float64 array (a download when it lives on the device)."""
        if self.g0 is None and self.g0_t is not None:
            self.g0 = self.g0_t.double().cpu().numpy()
        return self.g0

    @property
    def mapped_dose(self):
        if self._mapped_dose is None and self.mapped_t is not None:
            self._mapped_dose = self.mapped_t.double().cpu().numpy()
        return self._mapped_dose

    @mapped_dose.setter
    def mapped_dose(self, value):
        self._mapped_dose = value

    # -- shared helpers (BCLP.py:528-590) ------------------------------------
    def imposeSinogramConstraints(self, g):
        if self.bit_depth is not None:
            g = udata.discretize(g, self.bit_depth, [0.0, np.amax(g)])
        return np.clip(g, a_min=self.glb, a_max=self.gub)

    def checkSinogramShape(self, g, desired_shape="flattened"):
        if desired_shape == "flattened" and g.ndim > 1:
            return np.reshape(g, -1)
        if desired_shape == "cylindrical" and g.ndim == 1:
            return np.reshape(g, self.g0_shape)
        return g

    def checkConvergence(self):
        it = self.logs.curr_iter
        zero = self.logs.loss[it] == 0.0
        conv = False
        if it >= 5 and self.exit_param is not None:
            ch = np.abs(np.diff(self.logs.loss[it - 5:it + 1]))
            conv = bool(np.mean(ch) <= self.exit_param * self.logs.loss[it])
        return conv or zero

    # -- the reference's step interface (BCLP.py:277-475) -----------------------------
    # The same quantities as the host engine below, held as attributes and refreshed once per iteration
    # index (logs.curr_iter), so a caller can drive the problem with its own iteration loop as with the
    # reference: every getLoss / getLossGrad between two callback calls sees the state of the first
    # sinogram queried at that index (callback advances the index).
    def updateVariables(self, g_iter):
        """Bring dose, mapped dose, its errors from the target and from the tolerance band, the violation
        set, the loss and its gradient up to date for g_iter, each computed once per iteration index and
        in that order (BCLP.py:277-330)."""
        it = self.logs.curr_iter
        if self.dose_iter != it:
            g = self.checkSinogramShape(np.asarray(g_iter), desired_shape="cylindrical")
            self.dose = np.asarray(self.P.backward(g)).reshape(self.target_geo.array.shape)
            self.dose_iter = it
        if self.mapped_dose_iter != it:
            self.mapped_dose = self.response_model.map(self.dose)
            self.mapped_dose_iter = it
        if self.mapped_dose_error_from_f_T_iter != it:
            self.mapped_dose_error_from_f_T = self.mapped_dose - self.target_geo.array
            self.mapped_dose_error_from_f_T_iter = it
        if self.mapped_dose_error_from_band_iter != it:
            # positive exactly where the band constraint is violated
            self.mapped_dose_error_from_band = np.abs(self.mapped_dose_error_from_f_T) - self.eps
            self.mapped_dose_error_from_band_iter = it
        if self.v_iter != it:
            self.v = self.mapped_dose_error_from_band > 0
            self.v_iter = it
        if self.test_alternate_handling and self.weight_iter != it:
            inside = self.target_geo.array > 0
            self.weight = (inside if it % 2 == 0 else ~inside).astype(float)
            self.weight_iter = it
        if self.loss_iter != it:
            self.loss = self.computeLoss()
            self.loss_iter = it
        if self.loss_grad_iter != it:
            self.loss_grad = self.computeLossGradient()
            self.loss_grad_iter = it

    def computeLoss(self):
        """(sum over violating voxels of weight * |band error|^p * dvol)^(q/p), logged at the current
        iteration (BCLP.py:332-351)."""
        integrand = self.v * self.weight * np.abs(self.mapped_dose_error_from_band) ** self.p
        loss = (np.sum(integrand) * self.dvol) ** (self.q / self.p)
        self.logs.loss[self.logs.curr_iter] = loss
        return loss

    def computeLossGradient(self):
        """The loss gradient with respect to the sinogram, flattened: q loss^((q-p)/q) times the forward
        projection of v * weight * |band error|^(p-1) * sign(error) * dmap/df(dose); the forward alone
        when the loss is zero, where the factor is not finite (BCLP.py:353-386)."""
        operand = (self.v * self.weight * (np.abs(self.mapped_dose_error_from_band) ** (self.p - 1))
                   * np.sign(self.mapped_dose_error_from_f_T) * self.response_model.dmapdf(self.dose))
        fwd = np.asarray(self.P.forward(operand))
        grad = (self.q * self.loss ** ((self.q - self.p) / self.q)) * fwd if self.loss != 0.0 else fwd
        return self.checkSinogramShape(grad, desired_shape="flattened")

    def getLoss(self, g_iter):
        self.updateVariables(g_iter)
        return self.loss

    def getLossGrad(self, g_iter):
        self.updateVariables(g_iter)
        return self.loss_grad

    def evaluateNormMetrics(self):
        """l0 / l1 / l2 / l-infinity norms of the band violation and of the error itself (eps = 0), times
        dvol, logged at the current iteration (BCLP.py:396-437)."""
        i, L = self.logs.curr_iter, self.logs
        e, eb, v = self.mapped_dose_error_from_f_T, self.mapped_dose_error_from_band, self.v
        v0 = np.abs(e) > 0
        L.l0[i], L.l0_eps0[i] = np.sum(v) * self.dvol, np.sum(v0) * self.dvol
        L.l1[i], L.l1_eps0[i] = np.sum(v * np.abs(eb)) * self.dvol, np.sum(np.abs(e)) * self.dvol
        L.l2[i] = np.sqrt(np.sum(v * eb ** 2) * self.dvol)
        L.l2_eps0[i] = np.sqrt(np.sum(e ** 2) * self.dvol)
        L.lf[i], L.lf_eps0[i] = np.amax(v * np.abs(eb)), np.amax(v0 * np.abs(e))

    def callback(self, g_iter):
        """Norms and iteration time of the current iteration, then the next iteration index
        (BCLP.py:439-475; the live plots of verbose='plot' are not drawn here)."""
        self.updateVariables(g_iter)
        self.evaluateNormMetrics()
        self.logs.recordIterTime()
        if self.verbose in ("time", "plot", "plot_demo"):
            self.logger.info(f"Iteration {self.logs.curr_iter: 4.0f} at time: "
                             f"{self.logs.iter_times[self.logs.curr_iter]: 6.1f} s. "
                             f"Loss = {self.logs.loss[self.logs.curr_iter]}")
        self.logs.curr_iter += 1

    # -- host engine: the reference's numpy loop (BCLP.py:277-526) ---------------
    def _host_state(self, g):
        g = self.checkSinogramShape(g, "cylindrical")
        dose = np.asarray(self.P.backward(g)).reshape(self.target_geo.array.shape)
        mapped = self.response_model.map(dose)
        e = mapped - self.target_geo.array
        eb = np.abs(e) - self.eps
        v = eb > 0
        loss = (np.sum(v * self.weight * np.abs(eb) ** self.p) * self.dvol) ** (self.q / self.p)
        return dose, mapped, e, eb, v, loss

    def _host_norms(self, e, eb, v):
        i = self.logs.curr_iter
        L = self.logs
        v0 = np.abs(e) > 0
        L.l0[i], L.l0_eps0[i] = np.sum(v), np.sum(v0)
        L.l1[i], L.l1_eps0[i] = np.sum(v * np.abs(eb)), np.sum(np.abs(e))
        L.l2[i], L.l2_eps0[i] = np.sqrt(np.sum(v * eb ** 2)), np.sqrt(np.sum(e ** 2))
        L.lf[i], L.lf_eps0[i] = np.amax(v * np.abs(eb)), np.amax(v0 * np.abs(e))

    def gradientDescentHost(self):
        g = self.checkSinogramShape(self.host_g0(), "flattened")
        for _ in range(self.logs.options.n_iter):
            dose, mapped, e, eb, v, loss = self._host_state(g)
            self.logs.loss[self.logs.curr_iter] = loss
            operand = v * self.weight * (np.abs(eb) ** (self.p - 1)) * np.sign(e) * self.response_model.dmapdf(dose)
            fwd = np.asarray(self.P.forward(operand))
            grad = (self.q * loss ** ((self.q - self.p) / self.q)) * fwd if loss != 0.0 else fwd
            g = self.imposeSinogramConstraints(g - self.learning_rate * self.checkSinogramShape(grad, "flattened"))
            conv = self.checkConvergence() if self.exit_param is not None else False
            self._host_norms(e, eb, v)
            self.logs.recordIterTime()
            self.logs.curr_iter += 1
            if conv:
                self.logs.is_converged = True
                break
        dose, mapped, e, eb, v, loss = self._host_state(g)
        self.logs.loss[self.logs.curr_iter] = loss
        self._host_norms(e, eb, v)
        self.dose, self.mapped_dose = dose, mapped
        return g

    # -- device engine ---------------------------------------------------------
    def _device_projector_ops(self):
        from ._device_ops import device_ops

        ops = device_ops(self.P, self.target_geo, self.logs.options.n_iter)
        if ops is None:
            raise TypeError("the device engine needs a vamtoolbox_b200 projector")
        return ops

    def _device_response_ok(self):
        return getattr(self.response_model, "has_device_form", lambda: False)()

    def device_iteration(self, reduce_stats=None):
        """A :class:`DeviceIteration` holding this problem's device state (g = g0)."""
        return DeviceIteration(self, reduce_stats=reduce_stats)

    def gradientDescentDevice(self, graph=True, reduce_stats=None):
        """The device engine's loop; ``reduce_stats`` (see DeviceIteration) runs it eagerly with the loss /
        norm sums combined across ranks every iteration (vamtoolbox_b200.distributed.optimize_bclp_zslab)."""
        it = self.device_iteration(reduce_stats=reduce_stats)
        n_iter = self.logs.options.n_iter
        q, p = self.q, self.p
        dev = it.device
        st = torch.cuda.current_stream(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(n_iter + 1)]
        ev[0].record(st)
        eager = (not graph) or self.bit_depth is not None or self.exit_param is not None or reduce_stats is not None
        done = n_iter
        if eager:
            for k in range(n_iter):
                it.step()
                if self.bit_depth is not None:
                    it.g.copy_(udata.discretize_t(it.g, self.bit_depth, 0.0, torch.amax(it.g)))
                    it.g.clamp_(min=self.glb, max=self.gub)
                ev[k + 1].record(st)
                if self.exit_param is not None:
                    self.logs.fill_from_stats(it.log.cpu().numpy(), q, p, k + 1)
                    self.logs.curr_iter = k
                    if self.checkConvergence():
                        self.logs.is_converged = True
                        done = k + 1
                        break
        else:
            gr = it.capture()
            for k in range(n_iter):
                gr.replay()
                ev[k + 1].record(st)
            del gr
        it.state()  # dose / mapped dose / norms of the final sinogram
        torch.cuda.synchronize(dev)
        # device time per iteration of the loop (CUDA events on the engine's stream)
        self.options.device_iteration_ms = ev[0].elapsed_time(ev[done]) / done if done else None
        return self.finish_device(it, done, [ev[0].elapsed_time(ev[k + 1]) / 1e3 for k in range(done)])

    def finish_device(self, it, done, iter_times):
        """Logs, dose and sinogram of a device run from its iteration state (after a final ``it.state()``)."""
        n_iter = self.logs.options.n_iter
        self.logs.curr_iter = done
        rows = min(int(it.counter.item()), n_iter + 1)
        self.logs.fill_from_stats(it.log[:rows].cpu().numpy(), self.q, self.p, rows)
        for k in range(done):
            self.logs.iter_times[k] = iter_times[k]
        tshape = self.target_geo.array.shape
        self.dose_t, self.mapped_t, self.g_t = it.dose.reshape(tshape), it.mapped.reshape(tshape), it.g
        self._mapped_dose = None  # downloaded on first use (output="full" / "components")
        self.dose, g = to_host_f64(self.dose_t, it.g)
        return g.reshape(-1)

    def _device_engine_ok(self):
        """The fused engine serves this problem: a projector of this package with device entry points
        (parallel-beam plan, ray plan, vector geometry, algebraic propagator) and a device form of the
        response model."""
        P, plan = self.P, getattr(self.P, "plan", None)
        from ..projector.pyTorchAlgebraicPropagation import PyTorchAlgebraicPropagator

        proj_ok = (plan is not None and (hasattr(plan, "backward_ref") or hasattr(plan, "deposit")
                                         or (hasattr(P, "backward_t") and hasattr(P, "forward_t")))
                   or isinstance(P, PyTorchAlgebraicPropagator))
        return proj_ok and self._device_response_ok()

    def gradientDescent(self):
        """The fused device engine where it serves the problem, else the reference's host loop (response
        models without a device form, or engine="host")."""
        if getattr(self.options, "engine", "device") == "host" or not self._device_engine_ok():
            return self.gradientDescentHost()
        return self.gradientDescentDevice()


class DeviceIteration:
    """Device state and kernels of one BCLP iteration (the fused engine).

    ``step()`` issues, on the current stream: the backprojection of g into
    the dose, the fused dose pass (response, band error, operand and the 9
    loss / norm sums), the log append, the forward projection of the operand
    and the clamped sinogram update.  Nothing is allocated and nothing syncs,
    so ``capture()`` records it once as a CUDA graph.  ``reduce_stats`` (a
    callable on the 9-float stats tensor) is the hook where a z-sharded run
    all-reduces the loss sums before the update.
    """

    def __init__(self, bclp, reduce_stats=None):
        self.bclp = bclp
        back, fwd, vol_shape, sino_shape, dev = bclp._device_projector_ops()
        self.back, self.fwd, self.device = back, fwd, dev
        self.vol_shape, self.sino_shape = vol_shape, sino_shape
        n_iter = bclp.logs.options.n_iter
        self.ws = Workspace(dev)
        f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)
        if bclp.fT_t is not None:
            self.fT = bclp.fT_t.reshape(vol_shape).contiguous()
        else:
            self.fT = f32(bclp.target_geo.array).reshape(vol_shape).contiguous()
        if bclp.g0_t is not None:
            self.g = bclp.g0_t.reshape(sino_shape).clone()
        else:
            self.g = f32(bclp.host_g0()).reshape(sino_shape).contiguous()
        self.dose = torch.empty(vol_shape, dtype=torch.float32, device=dev)
        self.mapped = torch.empty(vol_shape, dtype=torch.float32, device=dev)
        self.operand = torch.empty(vol_shape, dtype=torch.float32, device=dev)
        self.grad = torch.empty(sino_shape, dtype=torch.float32, device=dev)
        self.stats = self.ws.scalar(9)
        self.log = torch.full((n_iter + 1, 9), float("nan"), dtype=torch.float32, device=dev)
        self.counter = torch.zeros(1, dtype=torch.int32, device=dev)
        self._keep = []
        if not bclp._device_response_ok():
            raise NotImplementedError(
                "the fused BCLP pass evaluates interpolation tables with increasing sample points and the "
                "analytical gen_log_fun / linear / identity forms; use engine='host' for other response models")
        eps = f32(bclp.eps).reshape(vol_shape) if np.ndim(bclp.eps) else bclp.eps
        weight = f32(bclp.weight).reshape(vol_shape) if np.ndim(bclp.weight) else bclp.weight
        self.prm = bclp_params(bclp.response_model, eps, weight, bclp.p, dev, self._keep)
        self.reduce_stats = reduce_stats

    def state(self):
        self.back(self.g, self.dose)
        self.ws.bclp_dose_pass(self.dose, self.fT, self.prm, self.mapped, self.operand, self.stats)
        if self.reduce_stats is not None:
            self.reduce_stats(self.stats)
        self.ws.append(self.stats, self.log, self.counter)

    def update(self):
        b = self.bclp
        self.fwd(self.operand, self.grad)
        self.ws.bclp_update(self.g, self.grad, b.learning_rate, b.p, b.q, b.glb, b.gub, self.stats)

    def step(self):
        self.state()
        self.update()

    def capture(self):
        return capture(self.step, self.device)


def minimizeBCLP(target_geo, proj_geo, options, output="packaged"):
    bclp = BCLPNorm(target_geo, proj_geo, options)
    g_opt = bclp.checkSinogramShape(bclp.gradientDescent(), "cylindrical")
    if output == "packaged":
        return (geometry.Sinogram(g_opt, proj_geo, options), geometry.Reconstruction(bclp.dose, proj_geo, options),
                bclp.logs.loss)
    if output == "full":
        return (geometry.Sinogram(g_opt, proj_geo, options), geometry.Reconstruction(bclp.dose, proj_geo, options),
                geometry.Reconstruction(bclp.mapped_dose, proj_geo, options), bclp.logs)
    if output == "components":
        return g_opt, bclp.dose, bclp.mapped_dose, bclp.logs
    raise ValueError(f"unknown output {output!r}")
