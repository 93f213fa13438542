"""Every public option of the ray tracer that reaches a kernel, against the
reference's own tracer (tests/golden/options.npz, made by
tests/golden/make_golden.py): the three eikonal parametrisations
(physical path length, canonical sigma, optical path length) x the three ODE
solvers (forward symplectic Euler, forward Euler, leapfrog), the analytic
Luneburg-lens index (surrounding index 1 and 1.2) and the analytic
homogeneous-ball attenuation.  Tolerance: relative L2 <= 1e-4 (float32
atomics, float32 fields against the reference's float64 fields)."""
import numpy as np
import pytest
import torch

from tests.conftest import relL2

pytestmark = pytest.mark.gpu
TOL = 1e-4

PARAMS = ("physical_path_length", "canonical", "optical_path_length")
SOLVERS = ("forward_symplectic_euler", "forward_euler", "leapfrog")


def _prop(G, im, am, param="physical_path_length", solver="forward_symplectic_euler"):
    from vamtoolbox_b200 import geometry
    from vamtoolbox_b200.projector.pyTorchRayTrace import PyTorchRayTracingPropagator

    tg = geometry.TargetGeometry(target=np.zeros((G["xv"].size, G["yv"].size, G["zv"].size)))
    pg = geometry.ProjectionGeometry(G["angles"], "ray_trace", CUDA=True, index_model=im, attenuation_model=am,
                                     absorption_model=am, ray_trace_method="eikonal", eikonal_parametrization=param,
                                     ray_trace_ode_solver=solver, ray_trace_ray_config="parallel",
                                     inclination_angle=0.0, ray_density=1)
    return PyTorchRayTracingPropagator(tg, pg)


def _coords(G):
    from vamtoolbox_b200 import geometry

    tg = geometry.TargetGeometry(target=np.zeros((G["xv"].size, G["yv"].size, G["zv"].size)))
    cv = tg.constructCoordVec()
    assert all(np.array_equal(a, G[k]) for a, k in zip(cv, ("xv", "yv", "zv")))
    return cv


def _check(G, P, key):
    assert relL2(P.forward(G[key + "_f"]), G[key + "_fwd"]) < TOL
    assert relL2(P.backward(G[key + "_g"]), G[key + "_bwd"]) < TOL


@pytest.mark.parametrize("solver", SOLVERS)
@pytest.mark.parametrize("param", PARAMS)
def test_integrator_and_parametrisation_match_reference(golden, param, solver):
    from vamtoolbox_b200 import medium

    G = golden["options"]
    cv = _coords(G)
    am = medium.AttenuationModel(cv, type="interpolation", form="freeform", alpha_x=torch.as_tensor(G["alpha"]))
    if solver == "leapfrog":  # the reference's leapfrog runs with analytic index models only
        im = medium.IndexModel(cv, type="analytical", form="luneburg_lens", R=0.9, p=2, n_sur=1.2)
    else:
        im = medium.IndexModel(cv, type="interpolation", form="freeform", n_x=torch.as_tensor(G["n"]))
    _check(G, _prop(G, im, am, param, solver), f"{param}__{solver}")


@pytest.mark.parametrize("tag", ["lune1", "lune12"])
def test_luneburg_lens_matches_reference(golden, tag):
    from vamtoolbox_b200 import medium

    G = golden["options"]
    cv = _coords(G)
    R, p, n_sur = G[tag + "_params"]
    im = medium.IndexModel(cv, type="analytical", form="luneburg_lens", R=float(R), p=float(p), n_sur=float(n_sur))
    am = medium.AttenuationModel(cv, type="analytical", form="homogeneous_cylinder", R=1, alpha_internal=15.0)
    _check(G, _prop(G, im, am), tag)


def test_homogeneous_ball_attenuation_matches_reference(golden):
    from vamtoolbox_b200 import medium

    G = golden["options"]
    cv = _coords(G)
    R, a = G["ball_params"]
    im = medium.IndexModel(cv, type="analytical", form="homogeneous", n_sur=1.0)
    am = medium.AttenuationModel(cv, type="analytical", form="homogeneous_ball", R=float(R), alpha_internal=float(a))
    _check(G, _prop(G, im, am), "ball")
