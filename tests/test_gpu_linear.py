"""GPU: HpgemAPILinear's stored-matrix stages against the oracle restatement
(oracle/linear.py: the reference's matrices, multiplied and mass-solved in
every stage).

Tolerances follow the matrix-free parity tests: stage derivatives
max(1e-12, 4 cond(Mhat) eps) (hpGEM solves with the stored mass matrix every
stage, the device applies the folded inverse), solutions 1e-12 relative
after N steps."""
import numpy as np
import pytest

from oracle.dg import ADVECTION, WAVE, Problem
from oracle.linear import LinearOracle, assemble
from oracle.mesh import mesh_from_description

import hpgem_b200
from hpgem_b200 import _native
from hpgem_b200.descriptor import linear_descriptor

pytestmark = pytest.mark.gpu

RTOL = 1e-12
EPS = np.finfo(float).eps


def desc(n, triangular=False):
    d = len(n)
    return hpgem_b200.structured_description(n, [0.0] * d, [1.0] * d, triangular, True)


def rel_err(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def stage_rtol(prob):
    M = np.einsum("q,qi,qj->ij", prob.rule.weights, prob.phi, prob.phi)
    return max(RTOL, 4.0 * np.linalg.cond(M) * EPS)


# (name, cells, triangular, order, physics, params, dt, steps)
CASES = [
    ("1D p3 advection", [8], False, 3, "advection", [0.7], 2e-3, 20),
    ("quads p2 advection", [6, 5], False, 2, "advection", [1.0, 0.5], 2e-3, 20),
    ("triangles p3 advection", [4, 6], True, 3, "advection", [0.3, -0.7], 1e-3, 20),
    ("hexahedra p2 advection", [3, 4, 3], False, 2, "advection", [1.0, 0.7, 0.3], 2e-3, 10),
    ("hexahedra p3 advection", [3, 3, 3], False, 3, "advection", [0.2, -0.9, 0.4], 1e-3, 10),
    ("tetrahedra p2 advection", [2, 2, 2], True, 2, "advection", [0.4, -0.3, 0.8], 1e-3, 10),
    ("quads p2 wave", [4, 4], False, 2, "wave", [0.7], 2e-3, 20),
    ("triangles p2 wave", [4, 4], True, 2, "wave", [1.0], 2e-3, 20),
    ("tetrahedra p2 wave", [2, 2, 2], True, 2, "wave", [1.3], 1e-3, 10),
    ("hexahedra p3 wave", [2, 2, 2], False, 3, "wave", [1.0], 1e-3, 5),
    # large enough for the grouped tensor-core kernel (64-element tiles of equal matrices):
    # one 64-row pass, several groups, four passes (256 rows), two passes (75 rows)
    ("hexahedra p3 advection tiles", [8, 8, 8], False, 3, "advection", [1.0, 0.7, 0.3], 1e-3, 4),
    ("tetrahedra p2 wave tiles", [4, 4, 4], True, 2, "wave", [1.3], 1e-3, 4),
    ("hexahedra p3 wave tiles", [4, 4, 4], False, 3, "wave", [1.0], 1e-3, 2),
    ("quads p4 wave tiles", [8, 8], False, 4, "wave", [0.7], 1e-3, 4),
]


def problem(cells, triangular, order, physics, params):
    mesh = mesh_from_description(desc(cells, triangular))
    if physics == "advection":
        return Problem(mesh, order, ADVECTION, a=params)
    return Problem(mesh, order, WAVE, cinv=params[0])


@pytest.mark.parametrize("name,cells,tri,order,physics,params,dt,steps", CASES, ids=[c[0] for c in CASES])
def test_linear_steps_match_oracle(name, cells, tri, order, physics, params, dt, steps):
    prob = problem(cells, tri, order, physics, params)
    lin = LinearOracle(*assemble(prob))
    u0 = np.random.default_rng(5).standard_normal(prob.n_dof)
    s = hpgem_b200.HpgemAPILinear(len(cells), order, physics, advection=params if physics == "advection" else None,
                                  c_inv=params[0] if physics == "wave" else 1.0, tableau="RK4_4")
    s.readMesh(desc(cells, tri))
    assert s.handle.kernel_kind == "linear"
    h = s.handle
    # one stage derivative
    h.set_state(0, u0)
    h.time_derivative(0, 1)
    assert rel_err(h.get_state(1), lin.time_derivative(u0)) < stage_rtol(prob), name
    # N steps
    h.set_state(0, u0)
    h.step(0.0, dt, steps)
    assert rel_err(h.get_state(0), lin.step(u0, dt, steps)) < RTOL, name


def test_generic_matrices_match_the_structured_route():
    """hgg_create_linear on the matrices hgg_linear_descriptor returns gives the
    same steps as hgg_create_linear_structured (the same matrices either way)."""
    d = desc([4, 6], True)
    D = linear_descriptor(d, 3, _native.PHYSICS_ADVECTION, [0.3, -0.7])
    g = hpgem_b200.Handle.linear(D["mass"], D["element_stiffness"], D["face_elements"], D["face_stiffness"],
                                 D["rk_a"], D["rk_b"], D["rk_c"])
    s = hpgem_b200.Handle.linear_structured(d, 3, _native.PHYSICS_ADVECTION, [0.3, -0.7])
    u0 = np.random.default_rng(2).standard_normal(g.vector_length)
    for h in (g, s):
        h.set_state(0, u0)
        h.step(0.0, 1e-3, 10)
    assert np.array_equal(g.get_state(0), s.get_state(0))


def test_boundary_faces_use_their_left_block_only():
    """Faces whose right element is -1 (a mesh boundary in hpGEM) contribute only
    their (LEFT, LEFT) block (HpgemAPILinear_Impl.h:410-430)."""
    d = desc([6, 5])
    D = linear_descriptor(d, 2, _native.PHYSICS_ADVECTION, [1.0, 0.5])
    fe = D["face_elements"].copy()
    fe[::3, 1] = -1  # every third face becomes a boundary face of its left element
    lin = LinearOracle(D["mass"], D["element_stiffness"], fe, D["face_stiffness"])
    h = hpgem_b200.Handle.linear(D["mass"], D["element_stiffness"], fe, D["face_stiffness"],
                                 D["rk_a"], D["rk_b"], D["rk_c"])
    u0 = np.random.default_rng(3).standard_normal(h.vector_length)
    h.set_state(0, u0)
    h.step(0.0, 1e-3, 10)
    assert rel_err(h.get_state(0), lin.step(u0, 1e-3, 10)) < RTOL


def test_linear_and_matrix_free_solvers_agree():
    """The stored-matrix and the matrix-free solver of the same physics step alike."""
    d = desc([8, 8])
    a = [1.0, 0.5]
    lin = hpgem_b200.HpgemAPILinear(2, 2, "advection", advection=a).readMesh(d)
    free = hpgem_b200.Advection(2, 2, a, tableau="RK4_4").readMesh(d)
    for s in (lin, free):
        s.setInitialSolution(lambda x: np.sin(2 * np.pi * x[:, 0]) * np.cos(2 * np.pi * x[:, 1]))
        s.handle.step(0.0, 1e-3, 50)
    assert rel_err(lin.getTimeIntegrationVector(0), free.getTimeIntegrationVector(0)) < 1e-11


def test_linear_mixed_form():
    """FP32 stage vectors (and FP32 contractions up to 20 rows): the solution stays
    within 1e-6 (L2) of the FP64 stored-matrix solution."""
    d = desc([6, 6], True)
    out = []
    for prec in (_native.PRECISION_FP64, _native.PRECISION_FP32):
        s = hpgem_b200.HpgemAPILinear(2, 2, "advection", advection=[1.0, 0.5], precision=prec).readMesh(d)
        s.setInitialSolution(lambda x: np.sin(2 * np.pi * x[:, 0]) * np.cos(2 * np.pi * x[:, 1]))
        s.handle.step(0.0, 1e-3, 50)
        out.append((s, s.getTimeIntegrationVector(0)))
    (s64, u64), (_, u32) = out
    assert s64.l2Distance(u32, u64) < 1e-6
    assert np.isfinite(u32).all()
