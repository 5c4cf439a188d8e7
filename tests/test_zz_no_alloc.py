"""GPU: hgg_time_derivative_static, the right-hand side of caller-owned device
vectors for callers that cannot allocate device memory while they step, against
the existing hgg_time_derivative on the same state and against the oracle's
time derivative, on two calls in a row (different inputs, shared scratch).

Handles covered: the slice kernel (tiled layout, scratch needed), the pipelined
sum-factorised kernel (scratch needed), the dense kernel of advection and of the
wave, and the stored-matrix kernel of HpgemAPILinear (these three read hpGEM
order and need no scratch).

Collected last (file name) so that it runs after the other GPU tests as well
as alone in a fresh process."""
import ctypes

import numpy as np
import pytest
import torch

import hpgem_b200
from hpgem_b200 import _native
from oracle.dg import ADVECTION, WAVE, Problem
from oracle.linear import LinearOracle, assemble
from oracle.mesh import mesh_from_description

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the solution tolerance of the parity tests
EPS = np.finfo(float).eps


def rel_err(a, b):
    return float(np.abs(np.asarray(a).reshape(-1) - np.asarray(b).reshape(-1)).max() / np.abs(b).max())


def stage_rtol(prob):
    """Tolerance of a stage derivative k = M^{-1} R against the oracle: the oracle
    solves with the element mass matrix by LU in every stage, the library applies
    the inverse folded into its operators; both carry a forward error of
    cond(M) times a small multiple of the round-off."""
    M = np.einsum("q,qi,qj->ij", prob.rule.weights, prob.phi, prob.phi)
    return max(RTOL, 4.0 * np.linalg.cond(M) * EPS)


def description(n, triangular=False):
    dim = len(n)
    return hpgem_b200.structured_description(n, [0.0] * dim, [1.0] * dim, triangular, True)


# (name, cells, triangular, order, physics, params, stored matrices)
CASES = [
    ("hexahedra p=3 slice", [6, 5, 4], False, 3, "advection", [1.0, -0.7, 0.3], False),
    ("hexahedra p=2 pipelined", [5, 4, 3], False, 2, "advection", [0.4, 0.9, -0.2], False),
    ("triangles p=2 dense", [8, 6], True, 2, "advection", [1.0, 0.5], False),
    ("tetrahedra p=2 wave", [2, 3, 2], True, 2, "wave", [1.0], False),
    ("hexahedra p=2 stored matrices", [3, 4, 3], False, 2, "advection", [1.0, 0.7, 0.3], True),
]


def make_solver(cells, triangular, order, physics, params, linear):
    dim = len(cells)
    if linear:
        solver = hpgem_b200.HpgemAPILinear(dim, order, physics, advection=params, tableau="RK4_4")
    elif physics == "wave":
        solver = hpgem_b200.AcousticWave(dim, order, c_inv=params[0], tableau="RK4_4")
    else:
        solver = hpgem_b200.Advection(dim, order, params, tableau="RK4_4")
    return solver.readMesh(description(cells, triangular))


def oracle_derivative(cells, triangular, order, physics, params, linear):
    mesh = mesh_from_description(description(cells, triangular))
    if physics == "wave":
        prob = Problem(mesh, order, WAVE, cinv=params[0])
    else:
        prob = Problem(mesh, order, ADVECTION, a=params)
    if linear:
        lin = LinearOracle(*assemble(prob))
        return prob, lin.time_derivative
    return prob, lambda u: prob.time_derivative(u.reshape(mesh.n_elements, -1)).reshape(-1)


def existing_entry_point(handle, u):
    handle.set_state(0, u)
    handle.time_derivative(0, 1)
    return handle.get_state(1)


@pytest.mark.parametrize("name,cells,triangular,order,physics,params,linear", CASES, ids=[c[0] for c in CASES])
def test_static_scratch_rhs_matches_time_derivative(name, cells, triangular, order, physics, params, linear):
    solver = make_solver(cells, triangular, order, physics, params, linear)
    h = solver.handle
    if linear:
        assert h.kernel_kind == "linear"
    prob, oracle_k = oracle_derivative(cells, triangular, order, physics, params, linear)
    lib = _native.load()
    n = h.vector_length
    rng = np.random.default_rng(7)
    for call in range(2):  # two calls in a row, different inputs, shared scratch
        u = rng.standard_normal(n)
        ref = existing_entry_point(h, u)
        u_dev = torch.from_numpy(u).cuda()
        k_dev = torch.full_like(u_dev, float("nan"))
        torch.cuda.synchronize()  # the library runs on its own stream
        rc = lib.hgg_time_derivative_static(h._raw, ctypes.c_void_p(u_dev.data_ptr()),
                                            ctypes.c_void_p(k_dev.data_ptr()))
        _native.check(rc, h._raw)
        got = k_dev.cpu().numpy()
        assert np.isfinite(got).all()
        assert rel_err(got, ref) < RTOL, (name, call)
        assert rel_err(got, oracle_k(u)) < stage_rtol(prob), (name, call)


def test_static_scratch_rejects_problems_beyond_its_size():
    # 33^3 hexahedra at p = 3: 35968 padded elements x 64 > 2^21 doubles per vector
    solver = hpgem_b200.Advection(3, 3, [1.0, 0.7, 0.3]).readMesh(description([33, 33, 33]))
    h = solver.handle
    lib = _native.load()
    u_dev = torch.zeros(h.vector_length, dtype=torch.float64, device="cuda")
    k_dev = torch.zeros_like(u_dev)
    torch.cuda.synchronize()
    rc = lib.hgg_time_derivative_static(h._raw, ctypes.c_void_p(u_dev.data_ptr()),
                                        ctypes.c_void_p(k_dev.data_ptr()))
    assert rc == -2  # HGG_ERR_UNSUPPORTED
    assert b"static scratch" in lib.hgg_last_error(h._raw)
