"""GPU parity: the CUDA stepping path against the CPU oracle (restated hpGEM).

Every case runs the same seeded initial coefficients through
``computeOneTimeStep`` on both sides and compares the solution (and, where
stated, the stage derivatives) in the max norm relative to the largest
coefficient.

Tolerances:
* solution coefficients after N steps: 1e-12 relative (the FP64 target),
  widened only where the mass-solve rounding below, carried into the solution
  through dt once per stage and step, exceeds it (hexahedra at p = 5);
* stage derivatives k_i = M^{-1} R: max(1e-12, 4 cond(Mhat) eps).  hpGEM
  solves the element mass system by LU in every stage; the forward error of
  that solve is the condition number of the reference mass matrix times a
  small multiple of the unit round-off (cond = 1.9e5 for hexahedra at p = 3,
  1.6e7 at p = 5), while the GPU path applies the inverse through exactly
  factorised reference operators.  The factor 4 covers the maximum over the
  1e5 coefficients of the larger meshes (1.4 cond eps observed for the
  Dormand-Prince stages on 1287 hexahedra at p = 3).  In the solution the
  same error is damped by dt.
"""
import math

import numpy as np
import pytest

from oracle.dg import ADVECTION, WAVE, WAVE_UPWIND, Problem
from oracle.mesh import mesh_from_description

import hpgem_b200
from hpgem_b200 import _native

pytestmark = pytest.mark.gpu

RTOL = 1e-12
EPS = np.finfo(float).eps


def mass_cond_eps(prob):
    M = np.einsum("q,qi,qj->ij", prob.rule.weights, prob.phi, prob.phi)
    return np.linalg.cond(M) * EPS


def stage_rtol(prob):
    return max(RTOL, 4.0 * mass_cond_eps(prob))


def solution_rtol(prob, dt, nsteps, stages=4):
    return max(RTOL, mass_cond_eps(prob) * dt * nsteps * stages)


def desc(n, triangular=False, periodic=True):
    dim = len(n)
    return hpgem_b200.structured_description(n, [0.0] * dim, [1.0] * dim, triangular, periodic)


def sine_field(x):
    return np.prod(np.sin(2 * np.pi * x), axis=1)


def run_pair(description, p, physics, params, tableau, dt, nsteps, seed=0, stages=False, variant=0):
    mesh = mesh_from_description(description)
    dim = mesh.dim
    if physics == "advection":
        prob = Problem(mesh, p, ADVECTION, a=params)
        u0 = prob.project(lambda x: sine_field(x)[:, None])
        solver = hpgem_b200.Advection(dim, p, params, tableau=tableau)
    else:
        prob = Problem(mesh, p, WAVE_UPWIND if physics == "wave_upwind" else WAVE, cinv=params[0])
        rng = np.random.default_rng(seed)
        k = rng.integers(1, 3, size=(dim,))
        u0 = prob.project(lambda x: np.stack(
            [np.sin(2 * np.pi * (x @ k))] + [0.3 * np.cos(2 * np.pi * x[:, i]) for i in range(dim)],
            axis=1))
        solver = hpgem_b200.AcousticWave(dim, p, c_inv=params[0], tableau=tableau,
                                         flux="upwind" if physics == "wave_upwind" else "central")
    solver.readMesh(description)
    solver.handle.set_kernel_variant(variant)
    solver.setTimeIntegrationVector(0, u0)
    t = solver.computeTimeSteps(0.0, dt, nsteps)
    assert math.isclose(t, nsteps * dt, rel_tol=1e-12)
    got = solver.getTimeIntegrationVector(0)
    if stages:
        ref, ref_k = prob.step(u0, dt, nsteps, tableau, return_stages=True)
        got_k = [solver.getTimeIntegrationVector(i + 1) for i in range(len(ref_k))]
        solver.stage_rtol = stage_rtol(prob)
        solver.solution_rtol = solution_rtol(prob, dt, nsteps, len(ref_k))
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


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_hex_tensor_kernel(p, variant):
    if p == 3 and variant != 0:
        pytest.skip("hexahedra of order 3 have the slice kernel only")
    n = 4 if p <= 3 else 3
    got, ref, solver, gk, rk = run_pair(desc([n, n, n]), p, "advection", [1.0, 0.7, 0.3], "RK4_4",
                                        2e-3, 3, stages=True, variant=variant)
    assert solver.handle.kernel_kind == "tensor"
    assert rel_err(got, ref) < solver.solution_rtol
    for a, b in zip(gk, rk):
        assert rel_err(a, b) < solver.stage_rtol


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_quad_tensor_kernel_negative_velocity(p, variant):
    got, ref, solver = run_pair(desc([6, 5]), p, "advection", [-0.8, 0.45], "RK4_4", 2e-3, 4,
                                variant=variant)
    assert solver.handle.kernel_kind == "tensor"
    assert rel_err(got, ref) < RTOL


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_triangles_dense_kernel(p):
    theta = 0.3 + p
    a = [math.cos(theta), math.sin(theta)]
    got, ref, solver = run_pair(desc([6, 6], triangular=True), p, "advection", a, "RK4_4", 1e-3, 4)
    # too few elements per operator group for the folded form: the dense kernel runs
    assert solver.handle.kernel_kind == "dense"
    assert rel_err(got, ref) < RTOL


@pytest.mark.parametrize("p", [4, 5])
def test_triangles_folded_operator(p):
    """From p = 4 on a mesh whose elements fill tiles of equal operators, the
    advection operator is folded into per-element matrices and applied by the
    stored-matrix tensor-core kernel."""
    theta = 0.7 + p
    a = [math.cos(theta), math.sin(theta)]
    got, ref, solver, gk, rk = run_pair(desc([32, 32], triangular=True), p, "advection", a, "RK4_4", 2e-4, 3,
                                        stages=True)
    assert solver.handle.kernel_kind == "linear"
    assert rel_err(got, ref) < solver.solution_rtol
    # the folded operator applies an explicit inverse of the mass matrix multiplied
    # into the assembled operator: twice the forward-error bound of one LU solve
    for x, y in zip(gk, rk):
        assert rel_err(x, y) < 2 * solver.stage_rtol


@pytest.mark.parametrize("p", [1, 2, 3])
def test_tets_wave_dense_kernel(p):
    got, ref, solver, gk, rk = run_pair(desc([2, 2, 2], triangular=True), p, "wave", [1.0], "RK4_4",
                                        5e-3, 3, stages=True)
    assert solver.handle.kernel_kind == "dense"
    assert rel_err(got, ref) < RTOL
    for a, b in zip(gk, rk):
        assert rel_err(a, b) < solver.stage_rtol


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


@pytest.mark.parametrize("p", [2, 4])
def test_pipelined_and_one_shot_kernels_agree_on_a_large_ragged_mesh(p):
    """Many tiles per block, a last tile that is only partly filled, every Dormand-Prince
    stage (more than one stage vector in the input): the two organisations of the
    sum-factorised kernel give the same numbers."""
    description = desc([13, 11, 9])
    res = []
    # at p = 4 the last Dormand-Prince stage reads more vectors than the pipelined
    # kernel's ring holds: variant 2 refuses it and the automatic choice takes variant 1
    for variant in ((0, 1, 2) if p == 2 else (0, 1)):
        s = hpgem_b200.Advection(3, p, [-0.4, 0.9, 0.25], tableau="DormandPrince").readMesh(description)
        s.handle.set_kernel_variant(variant)
        s.setInitialSolution(sine_field)
        s.computeTimeSteps(0.0, 1e-3, 5)
        res.append([s.getTimeIntegrationVector(i) for i in range(8)])
    for other in res[1:]:
        for a, b in zip(res[0], other):
            assert rel_err(a, b) < RTOL


def test_hex_p3_slice_kernel_dormand_prince_ragged():
    """Hexahedra p = 3, every Dormand-Prince stage (up to six stage vectors in the input
    and five in the final update), 1287 elements (last tile partly filled), stage
    vectors and solution against the oracle."""
    got, ref, solver, gk, rk = run_pair(desc([13, 11, 9]), 3, "advection", [-0.4, 0.9, 0.25],
                                        "DormandPrince", 1e-3, 2, stages=True)
    assert rel_err(got, ref) < RTOL
    for a, b in zip(gk, rk):
        assert rel_err(a, b) < solver.stage_rtol


def test_hex_p3_kernel_ragged_mesh_rk4():
    """Hexahedra p = 3 with RK4: element count not a multiple of the tile, negative and
    positive velocity components, against the oracle."""
    got, ref, solver = run_pair(desc([7, 5, 3]), 3, "advection", [-0.6, 0.8, -0.3], "RK4_4", 2e-3, 4)
    assert rel_err(got, ref) < RTOL


def test_hex_p3_rejects_other_kernel_organisations():
    s = hpgem_b200.Advection(3, 3, [1.0, 0.7, 0.3]).readMesh(desc([4, 4, 4]))
    with pytest.raises(_native.NativeError) as ex:
        s.handle.set_kernel_variant(1)
    assert ex.value.code == -2  # HGG_ERR_UNSUPPORTED
    s.handle.set_kernel_variant(0)


@pytest.fixture(scope="module")
def many_tiles_reference():
    description = desc([23, 17, 13])
    prob = Problem(mesh_from_description(description), 3, ADVECTION, a=[0.9, -0.5, 0.35])
    u0 = prob.project(lambda x: sine_field(x)[:, None])
    ref, ref_k = prob.step(u0, 1e-3, 2, "RK4_4", return_stages=True)
    return description, u0, ref, ref_k, stage_rtol(prob)


def test_hex_p3_many_tiles(many_tiles_reference):
    """More tiles than SMs, x-neighbours inside and outside each tile, periodic wrap in
    every direction, a last tile that is only partly filled."""
    description, u0, ref, ref_k, srtol = many_tiles_reference
    solver = hpgem_b200.Advection(3, 3, [0.9, -0.5, 0.35], tableau="RK4_4").readMesh(description)
    solver.setTimeIntegrationVector(0, u0)
    solver.computeTimeSteps(0.0, 1e-3, 2)
    assert rel_err(solver.getTimeIntegrationVector(0), ref) < RTOL
    for i, b in enumerate(ref_k):
        assert rel_err(solver.getTimeIntegrationVector(i + 1), b) < srtol


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
    assert rel_err(solver.getTimeIntegrationVector(1), prob.time_derivative(u)) < stage_rtol(prob)


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


UPWIND_CASES = [
    # cells, triangular, order, c_inv: every dense wave body (1D rows, 2D/3D shared rows)
    ([2, 2, 2], True, 2, 1.0),
    ([4, 4], True, 3, 0.5),
    ([4, 3], False, 2, 2.0),
    ([6], False, 3, 1.5),
]


@pytest.mark.parametrize("case", UPWIND_CASES, ids=lambda c: "%dD-%s-p%d" % (len(c[0]), "tri" if c[1] else "box", c[2]))
def test_wave_upwind_flux_against_oracle(case):
    """The upwind (Riemann) flux of the acoustic wave, restated (the reference has the
    central flux): solution and stage derivatives against the oracle's restatement."""
    cells, tri, p, cinv = case
    got, ref, solver, gk, rk = run_pair(desc(cells, triangular=tri), p, "wave_upwind", [cinv], "RK4_4",
                                        2e-3, 4, stages=True)
    assert solver.handle.kernel_kind == "dense"
    assert rel_err(got, ref) < solver.solution_rtol
    for a, b in zip(gk, rk):
        assert rel_err(a, b) < solver.stage_rtol
