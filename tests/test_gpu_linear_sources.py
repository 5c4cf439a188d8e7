"""GPU: HpgemAPILinear's source terms (addSourceTerm, addSourceTermAtBoundary,
kernel/Base/HpgemAPILinear_Impl.h:437-498) through the C ABI.

* The reference's own stored-matrix self-test, run unchanged through the
  library: tests/self/Basic/080AdvectionLinear_SelfTest.cpp (non-periodic
  meshes, inflow boundary values through the boundary source term,
  Dormand-Prince, the library's projection and L2 error): all four golden
  tables (080:255-297, 16 levels including p = 2 triangles) at the test's 1 %
  tolerance and to every printed digit.
* Coefficients after the steps equal the oracle's (LinearOracle with the same
  source) to the solution tolerance of the parity tests.
* hgg_time_derivative_at with an element source and a boundary source, on
  advection and on the wave, equals the oracle's time derivative at that time.
* A handle with source terms refuses calls that have no time."""
import ctypes

import numpy as np
import pytest

import hpgem_b200
from hpgem_b200 import _native
from oracle.dg import ADVECTION, WAVE, Problem
from oracle.linear import LinearOracle, assemble
from oracle.mesh import mesh_from_description

from test_oracle_pins import _linear_cases, linear_advection_run

pytestmark = pytest.mark.gpu

RTOL = 1e-12
EPS = np.finfo(float).eps


def rel_err(a, b):
    a, b = np.asarray(a).reshape(-1), np.asarray(b).reshape(-1)
    return float(np.abs(a - b).max() / np.abs(b).max())


def stage_rtol(prob):
    M = np.einsum("q,qi,qj->ij", prob.rule.weights, prob.phi, prob.phi)
    return max(RTOL, 4.0 * np.linalg.cond(M) * EPS)


def description_of(mesh_dims, triangular):
    D = len(mesh_dims)
    return hpgem_b200.structured_description(mesh_dims, [0.0] * D, [1.0] * D, triangular, False)


def _gpu_solver(results):
    """The library's run of 080's set-up; also keeps the oracle's coefficients for comparison."""
    def solve(cells, triangular, prob, a, inflow, exact, u0, dt, nT):
        s = hpgem_b200.HpgemAPILinear(prob.dim, prob.p, "advection", advection=a, tableau="DormandPrince")
        s.readMesh(description_of(cells, triangular))
        assert s.n_elements == prob.mesh.n_elements
        s.setInitialSolution(lambda x: exact(x, 0.0))  # the library's own projection
        assert rel_err(s.getTimeIntegrationVector(0), u0) < RTOL
        s.setSourceTermAtBoundary(inflow)
        s.computeTimeSteps(0.0, dt, nT)
        u = s.getTimeIntegrationVector(0).reshape(-1)
        results["gpu"] = s
        lin = LinearOracle(*assemble(prob)).set_sources(prob, boundary_source=inflow)
        results["oracle"] = lin.step(u0, dt, nT, "DormandPrince")
        results["prob"] = prob
        return u
    return solve


@pytest.mark.parametrize("key,level", list(_linear_cases()))
def test_080_goldens_through_the_library(key, level):
    results = {}
    err, gold = linear_advection_run(key, level, _gpu_solver(results))
    assert abs(err - gold) < 0.01 * gold  # ConvergenceTest.h:113-122
    assert abs(err - gold) < 1e-8 * gold  # every printed digit
    u = results["gpu"].getTimeIntegrationVector(0)
    assert rel_err(u, results["oracle"]) < RTOL
    # the library's own L2 error (computeTotalError on the device) agrees
    a = np.array([0.1 + 0.1 * i for i in range(results["prob"].dim)])
    T = {"dim1": 0.1, "dim2P1": 0.1, "dim2P2": 0.1, "dim3": 0.02}[key]
    dev_err = results["gpu"].computeTotalError(
        lambda x, t: np.prod(np.sin(2 * np.pi * (x - a * t)), axis=1), T)
    assert abs(dev_err - err) < 1e-12 * err


# (cells, triangular, periodic, order, physics, params)
DERIV_CASES = [
    ([4, 3], True, False, 2, "advection", [0.6, -0.4]),
    ([3, 3, 2], False, False, 2, "advection", [0.3, 0.5, -0.2]),
    ([4, 4], False, [True, False], 2, "wave", [0.8]),
    ([2, 2, 2], True, False, 1, "wave", [1.2]),
]


@pytest.mark.parametrize("cells,tri,periodic,p,physics,params", DERIV_CASES)
def test_time_derivative_at_with_both_sources(cells, tri, periodic, p, physics, params):
    D = len(cells)
    desc = hpgem_b200.structured_description(cells, [0.0] * D, [1.0] * D, tri, periodic)
    mesh = mesh_from_description(desc)
    prob = Problem(mesh, p, ADVECTION if physics == "advection" else WAVE,
                   a=params if physics == "advection" else (0, 0, 0),
                   cinv=params[0] if physics == "wave" else 1.0)
    V = prob.V

    def elem_src(x, t):
        return np.stack([np.sin(3 * x[:, 0] + v) * np.cos(2 * t) + x[:, -1] for v in range(V)], axis=1)

    def face_src(x, n, t):
        return np.stack([(1.0 + v) * n[:, 0] * np.exp(-t) + x[:, 0] * n[:, -1] for v in range(V)], axis=1)

    lin = LinearOracle(*assemble(prob)).set_sources(prob, element_source=elem_src, boundary_source=face_src)
    u = np.random.default_rng(5).standard_normal(prob.n_dof)
    t = 0.37
    ref = lin.time_derivative(u, t)
    if physics == "advection":
        s = hpgem_b200.HpgemAPILinear(D, p, "advection", advection=params, tableau="RK4_4")
    else:
        s = hpgem_b200.HpgemAPILinear(D, p, "wave", c_inv=params[0], tableau="RK4_4")
    s.readMesh(desc)
    s.setSourceTerm(elem_src)
    s.setSourceTermAtBoundary(face_src)
    s.setTimeIntegrationVector(0, u.reshape(s.n_elements, -1))
    s.computeTimeDerivative(0, 1, t)
    assert rel_err(s.getTimeIntegrationVector(1), ref) < stage_rtol(prob)

    # RK4 steps with both sources against the oracle's steps
    u0 = u * 1e-2
    s.setTimeIntegrationVector(0, u0.reshape(s.n_elements, -1))
    t_end = s.computeTimeSteps(0.25, 1e-3, 7)
    assert abs(t_end - 0.257) < 1e-15
    want = lin.step(u0, 1e-3, 7, "RK4_4", t0=0.25)
    assert rel_err(s.getTimeIntegrationVector(0), want) < RTOL

    # calls without a time are refused; the static right-hand side too
    lib = _native.load()
    assert lib.hgg_time_derivative(s.handle._raw, 0, 1) == -1
    assert b"hgg_time_derivative_at" in lib.hgg_last_error(s.handle._raw)
    assert lib.hgg_step(s.handle._raw, None, ctypes.c_double(1e-3), 1) == -1
    # removing both sources restores the plain operator
    s.setSourceTerm(None)
    s.setSourceTermAtBoundary(None)
    s.setTimeIntegrationVector(0, u.reshape(s.n_elements, -1))
    s.computeTimeDerivative(0, 1)
    plain = LinearOracle(*assemble(prob)).time_derivative(u)
    assert rel_err(s.getTimeIntegrationVector(1), plain) < stage_rtol(prob)


def test_sources_refused_where_the_mesh_is_unknown():
    lib = _native.load()
    s = hpgem_b200.Advection(2, 2, [1.0, 0.5]).readMesh(
        hpgem_b200.structured_description([4, 4], [0, 0], [1, 1]))
    assert lib.hgg_set_boundary_source(s.handle._raw, None, None) == -2  # matrix-free: no source terms
