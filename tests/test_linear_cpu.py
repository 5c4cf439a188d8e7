"""HpgemAPILinear's stored matrices on the CPU (no kernel runs).

* The matrices the library assembles (hgg_linear_descriptor) equal the
  oracle's numpy assembly of the same integrands (080AdvectionLinear_SelfTest,
  AcousticWaveLinear_Impl.h) entry by entry.
* The oracle's stored-matrix time derivative (multiply, then mass solve) equals
  the matrix-free oracle's right-hand side of the same physics: the two
  reference classes compute the same operator, so the linear restatement is
  pinned through the pinned matrix-free oracle.
* Invalid inputs are rejected before any device is touched."""
import ctypes

import numpy as np
import pytest

from oracle.dg import ADVECTION, WAVE, Problem
from oracle.linear import LinearOracle, assemble
from oracle.mesh import mesh_from_description

import hpgem_b200
from hpgem_b200 import _native
from hpgem_b200.descriptor import linear_descriptor

# (description, order, physics, params)
CASES = [
    ("structured 1 1\n6\n0\n1\nrectangular\ntrue\n", 3, 0, [0.7]),
    ("structured 1 2\n4 4\n0 0\n1 1\nrectangular\ntrue true\n", 2, 0, [1.0, 0.5]),
    ("structured 1 2\n4 6\n0 0\n1 2\ntriangular\ntrue true\n", 3, 0, [0.3, -0.7]),
    ("structured 1 2\n4 4\n0 0\n1 1\nrectangular\ntrue true\n", 2, 0, [1.0, 0.0]),  # flow along faces
    ("structured 1 3\n3 3 3\n0 0 0\n1 1 1\nrectangular\ntrue true true\n", 2, 0, [1.0, 0.7, 0.3]),
    ("structured 1 3\n2 2 2\n0 0 0\n1 1 1\ntriangular\ntrue true true\n", 2, 0, [0.4, -0.3, 0.8]),
    ("structured 1 2\n4 4\n0 0\n1 1\nrectangular\ntrue true\n", 2, 1, [0.7]),
    ("structured 1 2\n4 4\n0 0\n1 1\ntriangular\ntrue true\n", 2, 1, [1.0]),
    ("structured 1 3\n2 2 2\n0 0 0\n1 1 1\ntriangular\ntrue true true\n", 2, 1, [1.3]),
]
IDS = ["%dD-%s-p%d-%s" % (int(c[0].split()[2]), "tri" if "triangular" in c[0] else "rect", c[1],
                          "adv" if c[2] == 0 else "wave") for c in CASES]


# meshes with boundary faces (non-periodic directions): the stored-matrix path takes them
BOUNDARY_CASES = [
    ("structured 1 1\n4\n0\n1\nrectangular\nfalse\n", 1, 0, [0.1]),
    ("structured 1 2\n4 4\n0 0\n1 1\ntriangular\nfalse false\n", 2, 0, [0.1, 0.2]),
    ("structured 1 2\n3 4\n0 0\n1 1\nrectangular\ntrue false\n", 2, 0, [1.0, -0.5]),
    ("structured 1 3\n3 2 2\n0 0 0\n1 1 1\nrectangular\nfalse false false\n", 1, 0, [0.1, 0.2, 0.3]),
    ("structured 1 3\n2 2 2\n0 0 0\n1 1 1\ntriangular\nfalse false false\n", 2, 0, [0.4, -0.3, 0.8]),
    ("structured 1 2\n4 4\n0 0\n1 1\ntriangular\nfalse false\n", 2, 1, [1.0]),
    ("structured 1 3\n2 3 2\n0 0 0\n1 1 1\nrectangular\nfalse true false\n", 2, 1, [0.7]),
]


def oracle_problem(description, p, physics, params):
    mesh = mesh_from_description(description)
    if physics == 0:
        return Problem(mesh, p, ADVECTION, a=params)
    return Problem(mesh, p, WAVE, cinv=params[0])


@pytest.mark.parametrize("description,p,physics,params", CASES, ids=IDS)
def test_library_matrices_match_oracle_assembly(description, p, physics, params):
    prob = oracle_problem(description, p, physics, params)
    mass, K, fe, faces = assemble(prob)
    D = linear_descriptor(description, p, physics, params)
    scale = max(np.abs(K).max(), np.abs(faces).max())
    assert np.array_equal(D["face_elements"], fe)
    assert np.allclose(D["mass"], mass, rtol=0, atol=1e-15 * np.abs(mass).max() * 10)
    assert np.allclose(D["element_stiffness"], K, rtol=0, atol=1e-14 * scale)
    assert np.allclose(D["face_stiffness"], faces, rtol=0, atol=1e-14 * scale)


@pytest.mark.parametrize("description,p,physics,params", BOUNDARY_CASES)
def test_boundary_face_matrices_match_oracle_assembly(description, p, physics, params):
    """Boundary faces carry only their (LEFT, LEFT) block, with the application's
    boundary integrand (080:125-168 outflow term; AcousticWaveLinear_Impl.h:254-272)."""
    prob = oracle_problem(description, p, physics, params)
    mass, K, fe, faces = assemble(prob)
    boundary = fe[:, 1] < 0
    assert boundary.any()
    faces[boundary, 1:] = 0.0  # only (LEFT, LEFT) exists on a boundary face
    D = linear_descriptor(description, p, physics, params)
    scale = max(np.abs(K).max(), np.abs(faces).max())
    assert np.array_equal(D["face_elements"], fe)
    assert np.allclose(D["mass"], mass, rtol=0, atol=1e-15 * np.abs(mass).max() * 10)
    assert np.allclose(D["element_stiffness"], K, rtol=0, atol=1e-14 * scale)
    assert np.allclose(D["face_stiffness"], faces, rtol=0, atol=1e-14 * scale)


@pytest.mark.parametrize("description,p", [(CASES[7][0], 2), (CASES[8][0], 2), (CASES[6][0], 3)])
def test_upwind_wave_matrices_give_the_matrix_free_upwind_operator(description, p):
    """The folded form of the upwind wave (split-BF16 runs the wave as folded
    tensor-core tiles; HpgemAPILinear takes 'wave_upwind'): its stored matrices,
    applied as HpgemAPILinear applies them, give the matrix-free oracle's upwind
    right-hand side."""
    from oracle.dg import WAVE_UPWIND
    prob = Problem(mesh_from_description(description), p, WAVE_UPWIND, cinv=0.7)
    D = linear_descriptor(description, p, 2, [0.7])
    lin = LinearOracle(D["mass"], D["element_stiffness"], D["face_elements"], D["face_stiffness"])
    u = np.random.default_rng(12).standard_normal(prob.n_dof)
    k_lin, k_free = lin.time_derivative(u), prob.time_derivative(u)
    M = np.einsum("q,qi,qj->ij", prob.rule.weights, prob.phi, prob.phi)
    tol = max(1e-12, 8 * np.linalg.cond(M) * np.finfo(float).eps)
    assert np.abs(k_lin - k_free).max() <= tol * np.abs(k_free).max()


@pytest.mark.parametrize("description,p,physics,params", CASES, ids=IDS)
def test_stored_matrices_give_the_matrix_free_operator(description, p, physics, params):
    prob = oracle_problem(description, p, physics, params)
    lin = LinearOracle(*assemble(prob))
    u = np.random.default_rng(11).standard_normal(prob.n_dof)
    k_lin, k_free = lin.time_derivative(u), prob.time_derivative(u)
    M = np.einsum("q,qi,qj->ij", prob.rule.weights, prob.phi, prob.phi)
    tol = max(1e-12, 8 * np.linalg.cond(M) * np.finfo(float).eps)
    assert np.abs(k_lin - k_free).max() <= tol * np.abs(k_free).max()


def test_stored_matrix_steps_match_the_matrix_free_steps():
    description, p = CASES[2][0], 2
    prob = oracle_problem(description, p, 0, [0.3, -0.7])
    lin = LinearOracle(*assemble(prob))
    u0 = prob.project(lambda x: np.sin(2 * np.pi * x[:, :1]) * np.cos(2 * np.pi * x[:, 1:]))
    a = lin.step(u0, 1e-3, 5)
    b = prob.step(u0, 1e-3, 5).reshape(-1)
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_invalid_linear_inputs_are_rejected():
    lib = _native.load()
    desc = _native.LinearDesc()
    owner = ctypes.c_void_p()
    quads = b"structured 1 2\n4 4\n0 0\n1 1\nrectangular\ntrue true\n"
    a = (ctypes.c_double * 3)(1.0, 0.5, 0.0)
    # physics the stored-matrix form does not assemble
    rc = lib.hgg_linear_descriptor(quads, 2, 7, a, b"RK4_4", 0, ctypes.byref(desc), ctypes.byref(owner))
    assert rc == -2
    assert lib.hgg_linear_descriptor(quads, 2, 0, a, b"NoSuchTableau", 0, ctypes.byref(desc),
                                     ctypes.byref(owner)) == -1
    # a face that names an element out of range, and too many rows
    R, E = 3, 2
    m = np.tile(np.eye(R), (E, 1, 1))
    fe = np.array([[0, 5]], dtype=np.int64)
    fs = np.zeros((1, 4, R, R))
    rk_a, rk_b = np.zeros((1, 1)), np.ones(1)
    for rows, faces in ((R, fe), (300, np.array([[0, 1]], dtype=np.int64))):
        d = _native.LinearDesc(n_rows=rows, precision=0, n_elements=E, mass=m.ctypes.data,
                               element_stiffness=m.ctypes.data, n_faces=1, face_elements=faces.ctypes.data,
                               face_stiffness=fs.ctypes.data, n_stages=1, rk_a=rk_a.ctypes.data,
                               rk_b=rk_b.ctypes.data, rk_c=None)
        h = ctypes.c_void_p()
        assert lib.hgg_create_linear(ctypes.byref(d), ctypes.byref(h)) == -1
        assert lib.hgg_last_error(None)


def test_linear_create_reports_a_missing_device_or_succeeds():
    lib = _native.load()
    h = ctypes.c_void_p()
    a = (ctypes.c_double * 2)(1.0, 0.5)
    rc = lib.hgg_create_linear_structured(b"structured 1 2\n4 4\n0 0\n1 1\nrectangular\ntrue true\n",
                                          2, 0, a, b"RK4_4", 0, ctypes.byref(h))
    if rc == 0:
        assert lib.hgg_kernel_kind(h) == 2
        lib.hgg_destroy(h)
    else:
        assert rc == -6 and b"device" in lib.hgg_last_error(None)


def test_python_class_takes_the_linear_applications_only():
    with pytest.raises(ValueError):
        hpgem_b200.HpgemAPILinear(2, 2, "euler")
    # the upwind wave folds the same way as the reference's central one
    assert hpgem_b200.HpgemAPILinear(2, 2, "wave_upwind").numberOfVariables == 3


def test_linear_mesh_file_reports_a_missing_device_or_succeeds():
    import os
    lib = _native.load()
    h = ctypes.c_void_p()
    a = (ctypes.c_double * 3)(1.0, 0.7, 0.3)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mesh_files", "unitCubeN4Per.hpgem")
    rc = lib.hgg_create_linear_mesh_file(path.encode(), 2, 0, a, b"RK4_4", 0, ctypes.byref(h))
    if rc == 0:
        assert lib.hgg_kernel_kind(h) == 2
        lib.hgg_destroy(h)
    else:
        assert rc == -6 and b"device" in lib.hgg_last_error(None)
    # a missing file and an unknown physics are rejected before any device is touched
    assert lib.hgg_create_linear_mesh_file(b"/nonexistent.hpgem", 2, 0, a, b"RK4_4", 0, ctypes.byref(h)) == -1
    assert lib.hgg_create_linear_mesh_file(path.encode(), 2, 7, a, b"RK4_4", 0, ctypes.byref(h)) == -2
