"""GPU parity: the CUDA stepping path against the CPU oracle (restated hpGEM).

Every case runs the same seeded initial coefficients through
``computeOneTimeStep`` on both sides and compares the solution (and, where
stated, the stage derivatives) in the max norm relative to the largest
coefficient.  Tolerance: 1e-12 relative for the FP64 path (the accuracy
target of the FP64 form; both sides round differently only in summation order
and in the mass solve, which hpGEM does by LU per element and the GPU path
by the precomputed reference inverse).
"""
import math

import numpy as np
import pytest

from oracle.dg import ADVECTION, WAVE, Problem
from oracle.mesh import mesh_from_description

import hpgem_b200
from hpgem_b200 import _native

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def desc(n, triangular=False, periodic=True):
    dim = len(n)
    return hpgem_b200.structured_description(n, [0.0] * dim, [1.0] * dim, triangular, periodic)


def sine_field(x):
    return np.prod(np.sin(2 * np.pi * x), axis=1)


def run_pair(description, p, physics, params, tableau, dt, nsteps, seed=0, stages=False):
    mesh = mesh_from_description(description)
    dim = mesh.dim
    if physics == "advection":
        prob = Problem(mesh, p, ADVECTION, a=params)
        u0 = prob.project(lambda x: sine_field(x)[:, None])
        solver = hpgem_b200.Advection(dim, p, params, tableau=tableau)
    else:
        prob = Problem(mesh, p, WAVE, cinv=params[0])
        rng = np.random.default_rng(seed)
        k = rng.integers(1, 3, size=(dim,))
        u0 = prob.project(lambda x: np.stack(
            [np.sin(2 * np.pi * (x @ k))] + [0.3 * np.cos(2 * np.pi * x[:, i]) for i in range(dim)],
            axis=1))
        solver = hpgem_b200.AcousticWave(dim, p, c_inv=params[0], tableau=tableau)
    solver.readMesh(description)
    solver.setTimeIntegrationVector(0, u0)
    t = solver.computeTimeSteps(0.0, dt, nsteps)
    assert math.isclose(t, nsteps * dt, rel_tol=1e-12)
    got = solver.getTimeIntegrationVector(0)
    if stages:
        ref, ref_k = prob.step(u0, dt, nsteps, tableau, return_stages=True)
        got_k = [solver.getTimeIntegrationVector(i + 1) for i in range(len(ref_k))]
        return got, ref, solver, got_k, ref_k
    ref = prob.step(u0, dt, nsteps, tableau)
    return got, ref, solver


def rel_err(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def test_config1_quads_p2_rk4_100_steps():
    """2D advection, 32x32 periodic quads, p=2, a=(1,0.5), RK4, dt=1e-3, 100 steps."""
    got, ref, solver = run_pair(desc([32, 32]), 2, "advection", [1.0, 0.5], "RK4_4", 1e-3, 100)
    assert solver.handle.kernel_kind == "tensor"
    assert rel_err(got, ref) < RTOL


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_hex_tensor_kernel(p):
    n = 4 if p <= 3 else 3
    got, ref, solver, gk, rk = run_pair(desc([n, n, n]), p, "advection", [1.0, 0.7, 0.3], "RK4_4",
                                        2e-3, 3, stages=True)
    assert solver.handle.kernel_kind == "tensor"
    assert rel_err(got, ref) < RTOL
    for a, b in zip(gk, rk):
        assert rel_err(a, b) < RTOL


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_quad_tensor_kernel_negative_velocity(p):
    got, ref, solver = run_pair(desc([6, 5]), p, "advection", [-0.8, 0.45], "RK4_4", 2e-3, 4)
    assert solver.handle.kernel_kind == "tensor"
    assert rel_err(got, ref) < RTOL


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_triangles_dense_kernel(p):
    theta = 0.3 + p
    a = [math.cos(theta), math.sin(theta)]
    got, ref, solver = run_pair(desc([6, 6], triangular=True), p, "advection", a, "RK4_4", 1e-3, 4)
    assert solver.handle.kernel_kind == "dense"
    assert rel_err(got, ref) < RTOL


@pytest.mark.parametrize("p", [1, 2, 3])
def test_tets_wave_dense_kernel(p):
    got, ref, solver, gk, rk = run_pair(desc([2, 2, 2], triangular=True), p, "wave", [1.0], "RK4_4",
                                        5e-3, 3, stages=True)
    assert solver.handle.kernel_kind == "dense"
    assert rel_err(got, ref) < RTOL
    for a, b in zip(gk, rk):
        assert rel_err(a, b) < RTOL


def test_tets_wave_config3_shape_small():
    """Config-3 physics (tets p=2, 4 fields, c=1, RK4, dt=5e-4) on a 4^3x5 mesh, 20 steps."""
    got, ref, _ = run_pair(desc([4, 4, 4], triangular=True), 2, "wave", [1.0], "RK4_4", 5e-4, 20)
    assert rel_err(got, ref) < RTOL


def test_wave_on_squares_and_cubes():
    got, ref, _ = run_pair(desc([4, 4]), 2, "wave", [0.7], "RK4_4", 2e-3, 3)
    assert rel_err(got, ref) < RTOL
    got, ref, _ = run_pair(desc([3, 3, 3]), 2, "wave", [1.0], "RK4_4", 2e-3, 2)
    assert rel_err(got, ref) < RTOL


def test_advection_on_tets_and_lines():
    got, ref, _ = run_pair(desc([2, 2, 2], triangular=True), 2, "advection", [1.0, 0.7, 0.3],
                           "RK4_4", 2e-3, 3)
    assert rel_err(got, ref) < RTOL
    for p in (1, 3, 5):
        got, ref, _ = run_pair(desc([7]), p, "advection", [0.6], "RK4_4", 2e-3, 5)
        assert rel_err(got, ref) < RTOL


@pytest.mark.parametrize("tableau", ["DormandPrince", "ForwardEuler", "MidPoint", "RK2TVD",
                                     "RK3TVD", "BogackiShampine"])
def test_every_tableau(tableau):
    got, ref, _ = run_pair(desc([4, 4], triangular=True), 2, "advection", [0.1, 0.2], tableau,
                           1e-2, 3)
    assert rel_err(got, ref) < RTOL


def test_axis_aligned_velocity_takes_average_flux():
    # a . n = 0 on the y-faces: hpGEM averages both traces there (|A| < 1e-12)
    got, ref, _ = run_pair(desc([5, 5]), 2, "advection", [1.0, 0.0], "RK4_4", 1e-3, 5)
    assert rel_err(got, ref) < RTOL


def test_time_derivative_matches_oracle():
    description = desc([3, 3, 3])
    mesh = mesh_from_description(description)
    prob = Problem(mesh, 3, ADVECTION, a=[1.0, 0.7, 0.3])
    rng = np.random.default_rng(7)
    u = rng.standard_normal((mesh.n_elements, prob.nB))
    solver = hpgem_b200.Advection(3, 3, [1.0, 0.7, 0.3], tableau="RK4_4").readMesh(description)
    solver.setTimeIntegrationVector(0, u)
    solver.computeTimeDerivative(0, 1)
    assert rel_err(solver.getTimeIntegrationVector(1), prob.time_derivative(u)) < 1e-11


def test_state_round_trip_and_store_last_stage():
    description = desc([4, 4, 4])
    solver = hpgem_b200.Advection(3, 3, [1.0, 0.7, 0.3], tableau="RK4_4").readMesh(description)
    rng = np.random.default_rng(3)
    u = rng.standard_normal(solver.handle.vector_length)
    solver.setTimeIntegrationVector(0, u)
    assert np.array_equal(solver.getTimeIntegrationVector(0).reshape(-1), u)
    solver.computeTimeSteps(0.0, 1e-3, 3)
    a = solver.getTimeIntegrationVector(0)
    solver.setTimeIntegrationVector(0, u)
    solver.handle.set_store_last_stage(False)
    solver.computeTimeSteps(0.0, 1e-3, 3)
    assert np.array_equal(solver.getTimeIntegrationVector(0), a)


def test_advection_selftest_goldens_through_gpu():
    """090Advection_SelfTest goldens (Dormand-Prince, p=1) through the library's own
    projection, stepping and error norm."""
    import json
    import os
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "advection_goldens.json")))
    for dim, sizes in (("1", [4, 8, 16, 32]), ("2", [4, 8, 16, 32, 64]), ("3", [4, 8, 16])):
        par = g[dim]
        D = int(dim)
        a = [0.1 + 0.1 * i for i in range(D)]
        for level, N in enumerate(sizes):
            solver = hpgem_b200.Advection(D, par["p"], a, tableau="DormandPrince")
            solver.readMesh(desc([N] * D, triangular=(D == 2)))
            _, steps, dt = solver.solve(0.0, par["end_time"], par["end_time"] / par["time_steps"],
                                        1, u0=sine_field)
            assert steps == par["time_steps"]
            err = solver.computeTotalError(
                lambda x, t: sine_field(x - np.asarray(a) * t), par["end_time"])
            gold = par["errors"][level]
            assert abs(err - gold) < 0.01 * gold, (dim, N, err, gold)


def test_invalid_inputs_fail_loudly():
    with pytest.raises(_native.NativeError):
        hpgem_b200.Advection(2, 2, [1.0, 0.5]).readMesh("structured 1 2\n4 4\n0 0\n1 1\nrectangular\nfalse false\n")
    with pytest.raises(_native.NativeError):
        hpgem_b200.Advection(2, 6, [1.0, 0.5]).readMesh(desc([4, 4]))
    with pytest.raises(_native.NativeError):
        hpgem_b200.Advection(2, 2, [1.0, 0.5], tableau="NoSuchTableau").readMesh(desc([4, 4]))
