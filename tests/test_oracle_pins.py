"""Pins of the CPU oracle against the reference's own golden data.

* meshes: bit-exact against the Preprocessor output committed in hpGEM's
  tests/files (tests/golden/meshes.json);
* basis functions + quadrature rules: the known-answer integrals of hpGEM's
  quadrature unit tests (tests/unit/Integration/QuadratureRules/0[2-6]0*.cpp),
  at their 1e-12 tolerance;
* the whole time-stepping pipeline: the L2-error goldens of
  tests/self/Basic/090Advection_SelfTest.cpp:303-337 (Dormand-Prince, p = 1,
  periodic 1D lines, 2D triangles, 3D cubes), at that test's 1 % tolerance;
* the stored-matrix pipeline with its boundary source term: the four L2-error
  tables of tests/self/Basic/080AdvectionLinear_SelfTest.cpp:255-297
  (HpgemAPILinear, Dormand-Prince, non-periodic meshes whose inflow boundary
  enters through addSourceTermAtBoundary; p = 1 lines, triangles and cubes,
  p = 2 triangles), at that test's 1 % tolerance and to every printed digit.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle.basis import tabulate
from oracle.dg import ADVECTION, Problem
from oracle.linear import LinearOracle, assemble
from oracle.mesh import structured_mesh
from oracle.quadrature import _tensor_rule, rule_by_name

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.mark.parametrize("name", sorted(_load("meshes.json")))
def test_structured_mesh_matches_preprocessor(name):
    ref = _load("meshes.json")[name]
    s = ref["source"]
    mesh = structured_mesh(s["n"], s["lower"], s["upper"], s["triangular"], s["periodic"])
    assert np.array_equal(mesh.element_nodes, np.array(ref["element_nodes"]))
    assert np.array_equal(mesh.element_coords, np.array(ref["element_coords"]))
    # every face has two sides on periodic meshes; none is shared by three
    table = mesh.faces["table"]
    if all(s["periodic"]):
        assert (table[:, 1] >= 0).all()


_TENSOR = {"line": ("Cn1_1_1", "Cn1_3_2", "Cn1_5_3", "C1_7_4", "C1_9_5", "C1_11_6"),
           "square": ("Cn2_1_1", "Cn2_3_4", "Cn2_5_9", "C2_7_4", "C2_9_5", "C2_11_6"),
           "cube": ("Cn3_1_1", "Cn3_3_4", "Cn3_5_9", "C3_7_2", "C3_9_2", "C3_11_2")}


def _cases():
    q = _load("quadrature_integrals.json")
    for shape, spec in q.items():
        for rname, order in spec["rules"]:
            yield shape, rname, order


@pytest.mark.parametrize("shape,rname,order", list(_cases()))
def test_basis_integrals_known_answers(shape, rname, order):
    spec = _load("quadrature_integrals.json")[shape]
    if shape in _TENSOR:
        rule = _tensor_rule(shape, _TENSOR[shape].index(rname) + 1)
    else:
        rule = rule_by_name(shape, rname)
    assert rule.order >= order
    assert (rule.weights >= 0).all()
    phi, _ = tabulate(shape, order, rule.points)
    integrals = rule.weights @ phi
    for i, v in enumerate(integrals):
        for cond, expected in spec["chain"]:
            if eval(cond, {"i": i, "math": math}):
                assert abs(v - expected) < 1e-12, (i, v, expected)
                break


def test_basis_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    for shape, d in (("square", 2), ("triangle", 2), ("cube", 3), ("tetrahedron", 3)):
        x = rng.uniform(0.05, 0.3, size=(5, d))
        _, g = tabulate(shape, 4, x)
        h = 1e-6
        for k in range(d):
            xp, xm = x.copy(), x.copy()
            xp[:, k] += h
            xm[:, k] -= h
            fd = (tabulate(shape, 4, xp)[0] - tabulate(shape, 4, xm)[0]) / (2 * h)
            assert np.allclose(g[:, :, k], fd, atol=1e-7)


_SIZES = {"1": [4, 8, 16, 32], "2": [4, 8, 16, 32, 64], "3": [4, 8, 16]}


@pytest.mark.parametrize("dim,level", [(d, i) for d in ("1", "2", "3")
                                       for i in range(len(_SIZES[d]))])
def test_advection_selftest_goldens(dim, level):
    par = _load("advection_goldens.json")[dim]
    D = int(dim)
    N = _SIZES[dim][level]
    if D == 3 and N > 8:
        pytest.skip("16^3 level runs in the slow suite")
    a = np.array([0.1 + 0.1 * i for i in range(D)])  # 090Advection_SelfTest.cpp:83-86
    mesh = structured_mesh([N] * D, [0.0] * D, [1.0] * D, D == 2, [True] * D)
    prob = Problem(mesh, par["p"], ADVECTION, a=a)
    u = prob.project(lambda x: np.prod(np.sin(2 * np.pi * x), axis=1)[:, None])
    T, nT = par["end_time"], par["time_steps"]
    u = prob.step(u, T / nT, nT, "DormandPrince")
    err = prob.l2_error(u, lambda x, t: np.prod(np.sin(2 * np.pi * (x - a * t)), axis=1)[:, None], T)
    gold = par["errors"][level]
    assert abs(err - gold) < 0.01 * gold  # ConvergenceTest.h:113-122
    assert abs(err - gold) < 1e-7 * gold  # and in fact to every printed digit


def _linear_cases():
    g = _load("advection_linear_goldens.json")
    for key in ("dim1", "dim2P1", "dim2P2", "dim3"):
        for level in range(len(g[key]["errors"])):
            yield key, level


def linear_advection_run(key, level, solver):
    """080AdvectionLinear_SelfTest's set-up (080:58-103, 108-168, 255-297): a_i = 0.1 + 0.1 i,
    u0 = prod sin(2 pi x_i) projected, inflow boundary value through the boundary source term
    g = -u_exact(x, t) (a . n) where a . n < 0, Dormand-Prince, nT steps to T; returns
    (L2 error at T, golden).  ``solver(cells, triangular, prob, a, g, exact, u0, dt, nT)``
    runs the steps on the structured mesh of ``cells`` per direction, not periodic, from
    the projection of exact(x, 0) (``u0``: the oracle's projection)."""
    par = _load("advection_linear_goldens.json")[key]
    D = {"dim1": 1, "dim2P1": 2, "dim2P2": 2, "dim3": 3}[key]
    name = par["files"][par["levels"][0] + level]   # e.g. unitSquareTrianglesN8
    N = int(name.rsplit("N", 1)[1])
    a = np.array([0.1 + 0.1 * i for i in range(D)])
    triangular = "Triangles" in name
    mesh = structured_mesh([N] * D, [0.0] * D, [1.0] * D, triangular, [False] * D)
    prob = Problem(mesh, par["p"], ADVECTION, a=a)

    def exact(x, t):
        return np.prod(np.sin(2 * np.pi * (x - a * t)), axis=1)[:, None]

    def inflow(x, n, t):
        flow = n @ a
        return np.where(flow < 0, -exact(x, t)[:, 0] * flow, 0.0)[:, None]

    u0 = prob.project(lambda x: exact(x, 0.0)).reshape(-1)
    T, nT = par["end_time"], par["time_steps"]
    u = solver([N] * D, triangular, prob, a, inflow, exact, u0, T / nT, nT)
    return prob.l2_error(u, exact, T), par["errors"][level]


def _oracle_solver(cells, triangular, prob, a, inflow, exact, u0, dt, nT):
    lin = LinearOracle(*assemble(prob)).set_sources(prob, boundary_source=inflow)
    return lin.step(u0, dt, nT, "DormandPrince")


@pytest.mark.parametrize("key,level", list(_linear_cases()))
def test_linear_advection_selftest_goldens(key, level):
    if key == "dim3" and level == 2:
        pytest.skip("16^3 level takes a few seconds; the GPU test runs it")
    err, gold = linear_advection_run(key, level, _oracle_solver)
    assert abs(err - gold) < 0.01 * gold  # ConvergenceTest.h:113-122
    assert abs(err - gold) < 1e-8 * gold  # and to every printed digit
