"""Per-problem launch-shape tuning for the parallel-beam kernels.

The fastest vector width (slices per lane) and backprojection angle batch
depend on the slice count, the number of angles and the device, so a plan can
time every candidate once on its own device and keep the winner.  Winners are
cached in a JSON file keyed by device name and problem shape, so later plans of
the same shape apply the cached shape without timing anything.

The cache file is ``$VAMTOOLBOX_B200_TUNE_CACHE`` when set, else
``~/.cache/vamtoolbox_b200/tuning.json``.  Tuning changes launch shapes only:
every candidate computes the same sums in the same order per slice, and the
tests check each candidate against the oracle.
"""
from __future__ import annotations

import json
import os
import threading

import torch

from . import _lib

# slices per lane: 1 = the generic kernel, 4 / 8 = the fast kernels (nZ % 4 == 0), 6 / 5 = the fast forward
# on 192- / 160-slice chunks (nZ % 192 == 0 / nZ % 160 == 0)
FORWARD_VZ = (1, 4, 5, 6, 8)
# (slices per lane, angles per batch, bin table): the block table serves four or eight slices per lane,
# and 0 (automatic) adds six / five on 192- / 160-slice chunks
BACKWARD = ((1, 1, 0), (4, 1, 0), (8, 1, 0), (4, 2, 0), (8, 2, 0), (4, 4, 0), (4, 2, 1), (8, 2, 1), (0, 2, 1))
ADJOINT = ((1, 0), (4, 1), (8, 1), (4, 0), (8, 0))           # (slices per lane, weight table on)

_lock = threading.Lock()


def cache_path():
    p = os.environ.get("VAMTOOLBOX_B200_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "vamtoolbox_b200", "tuning.json")


def problem_key(plan):
    name = torch.cuda.get_device_name(plan.device).replace(" ", "_")
    ny, nx, nz = plan.shape_vol
    return f"{name}|{ny}x{nx}x{nz}|na{plan.angles.size}|abs={plan.absorption or 'none'}|occ={int(plan.has_occlusion)}"


def _load(path):
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def _store(path, key, value):
    with _lock:
        d = _load(path)
        d[key] = value
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        tmp = f"{path}.{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, path)


def _time(fn, reps, warm):
    for _ in range(warm):
        fn()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(reps):
        s.record()
        fn()
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    return best


def measure(plan, reps=3, warm=1, ops=("forward", "backward", "adjoint")):
    """Time every candidate of ``ops`` on the plan's device; returns (tuning dict, timings in ms).
    Ops left out keep the plan's current shape (the adjoint's weight table is then not built)."""
    dev = plan.device
    with torch.cuda.device(dev):
        g = torch.Generator(device=dev).manual_seed(0)
        x = torch.rand(plan.shape_vol, device=dev, generator=g)
        b = torch.rand(plan.shape_sino, device=dev, generator=g)
        ob, ox = torch.empty_like(b), torch.empty_like(x)
        table = plan.prepare_adjoint() if "adjoint" in ops else False
        times = {"forward": {}, "backward": {}, "adjoint": {}}
        base = plan.get_tuning()
        for vz in FORWARD_VZ if "forward" in ops else ():
            if (vz == 6 and plan.shape_vol[2] % 192) or (vz == 5 and plan.shape_vol[2] % 160):
                continue
            plan.set_tuning(dict(base, forward_vz=vz))
            times["forward"][str(vz)] = _time(lambda: plan.forward(x, ob), reps, warm)
        for vz, bt, tb in BACKWARD if "backward" in ops else ():
            if tb and not getattr(plan, "has_backward_table", False):
                continue
            plan.set_tuning(dict(base, backward_vz=vz, backward_batch=bt, backward_table=tb))
            times["backward"][f"{vz},{bt},{tb}"] = _time(lambda: plan.backward_ref(b, ox), reps, warm)
        for vz, tb in ADJOINT if "adjoint" in ops else ():
            if tb and not table:
                continue
            plan.set_tuning(dict(base, adjoint_vz=vz, adjoint_table=tb))
            times["adjoint"][f"{vz},{tb}"] = _time(lambda: plan.adjoint(b, ox), reps, warm)
        plan.set_tuning(base)
    best = dict(base)
    if times["forward"]:
        best["forward_vz"] = int(min(times["forward"], key=times["forward"].get))
    if times["backward"]:
        best["backward_vz"], best["backward_batch"], best["backward_table"] = map(
            int, min(times["backward"], key=times["backward"].get).split(","))
    if times["adjoint"]:
        best["adjoint_vz"], best["adjoint_table"] = map(int, min(times["adjoint"], key=times["adjoint"].get).split(","))
    return best, times


def autotune(plan, use_cache=True, reps=3, warm=1, ops=("forward", "backward", "adjoint")):
    """Apply the cached or freshly measured best launch shapes to ``plan``; returns them."""
    path = cache_path()
    key = problem_key(plan) + ("" if len(ops) == 3 else "|" + ",".join(ops))
    if use_cache:
        hit = _load(path).get(key)
        if isinstance(hit, dict) and "tuning" in hit:
            try:
                plan.set_tuning(hit["tuning"])
                return plan.get_tuning()
            except (_lib.VamError, TypeError, KeyError):
                pass
    best, times = measure(plan, reps, warm, ops)
    plan.set_tuning(best)
    if use_cache:
        try:
            _store(path, key, {"tuning": best, "ms": times})
        except OSError:
            pass
    return plan.get_tuning()
