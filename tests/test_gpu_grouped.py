"""GPU: the grouped dense kernel of the wave (tiles of 32 elements with the
same operator signature, 16 above 24 basis functions; lane = element, warp =
basis row; FP64 contractions) against the per-element-row kernel it replaces (kernel variant
1) and against the oracle.

Meshes are large enough that every group fills whole tiles (the grouped kernel
runs only when the tiles are at least half full)."""
import numpy as np
import pytest

from oracle.dg import WAVE, WAVE_UPWIND, Problem
from oracle.mesh import mesh_from_description

import hpgem_b200
from hpgem_b200 import _native

pytestmark = pytest.mark.gpu

RTOL = 1e-12
EPS = np.finfo(float).eps


def desc(n, triangular):
    d = len(n)
    return hpgem_b200.structured_description(n, [0.0] * d, [1.0] * d, triangular, True)


def rel_err(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


# (name, cells, order, physics, params, dt, steps, triangular)
CASES = [
    ("triangles p1 wave", [16, 16], 1, "wave", [1.0], 1e-3, 10, True),
    ("triangles p2 wave", [8, 8], 2, "wave", [1.0], 1e-3, 10, True),
    ("triangles p5 upwind wave", [8, 8], 5, "wave_upwind", [0.7], 5e-4, 5, True),
    ("quadrilaterals p2 wave", [8, 8], 2, "wave", [1.2], 1e-3, 10, False),
    ("hexahedra p1 upwind wave", [4, 4, 4], 1, "wave_upwind", [1.0], 1e-3, 10, False),
    ("tetrahedra p2 wave", [4, 4, 4], 2, "wave", [1.3], 1e-3, 5, True),
    ("tetrahedra p2 upwind wave", [4, 4, 4], 2, "wave_upwind", [0.8], 1e-3, 5, True),
    ("tetrahedra p3 upwind wave", [4, 4, 4], 3, "wave_upwind", [1.0], 5e-4, 3, True),
    # above 24 basis functions: tiles of 16 elements (a warp covers two basis rows)
    ("tetrahedra p4 upwind wave, 16-element tiles", [4, 4, 4], 4, "wave_upwind", [1.0], 2e-4, 3, True),
    ("quadrilaterals p4 wave, 16-element tiles", [8, 8], 4, "wave", [1.1], 2e-4, 4, False),
]


def solver_for(cells, order, physics, params, tri, precision=_native.PRECISION_FP64):
    s = hpgem_b200.AcousticWave(len(cells), order, c_inv=params[0], tableau="RK4_4", precision=precision,
                                flux="upwind" if physics == "wave_upwind" else "central")
    return s.readMesh(desc(cells, tri))


def oracle_for(cells, order, physics, params, tri):
    mesh = mesh_from_description(desc(cells, tri))
    return Problem(mesh, order, WAVE_UPWIND if physics == "wave_upwind" else WAVE, cinv=params[0])


@pytest.mark.parametrize("name,cells,order,physics,params,dt,steps,tri", CASES, ids=[c[0] for c in CASES])
def test_grouped_kernel_matches_row_kernel_and_oracle(name, cells, order, physics, params, dt, steps, tri):
    prob = oracle_for(cells, order, physics, params, tri)
    u0 = np.random.default_rng(9).standard_normal(prob.n_dof)
    out = {}
    for variant in (2, 1):  # the grouped kernel wherever the mesh forms tiles, the per-row kernel
        s = solver_for(cells, order, physics, params, tri)
        assert s.handle.kernel_kind == "dense"
        h = s.handle
        h.set_kernel_variant(variant)
        h.set_state(0, u0)
        h.time_derivative(0, 1)
        k = h.get_state(1)
        h.set_state(0, u0)
        h.step(0.0, dt, steps)
        out[variant] = (k, h.get_state(0))
    M = np.einsum("q,qi,qj->ij", prob.rule.weights, prob.phi, prob.phi)
    stage_tol = max(RTOL, 4.0 * np.linalg.cond(M) * EPS)
    # the two organisations do the same arithmetic up to the compiler's FMA contraction
    assert rel_err(out[2][0], out[1][0]) < stage_tol, name
    assert rel_err(out[2][1], out[1][1]) < RTOL, name
    assert rel_err(out[2][0], prob.time_derivative(u0).reshape(-1)) < stage_tol, name
    assert rel_err(out[2][1], prob.step(u0, dt, steps).reshape(-1)) < RTOL, name


@pytest.mark.parametrize("name,cells,order,physics,params,dt,steps,tri", [CASES[1], CASES[6]],
                         ids=[CASES[i][0] for i in (1, 6)])
def test_mixed_form_beside_the_grouped_fp64_kernel(name, cells, order, physics, params, dt, steps, tri):
    """The FP32-mixed form (FP32 contractions) stays within 1e-6 (L2) of the grouped
    FP64 solution."""
    u0 = np.random.default_rng(9).standard_normal(oracle_for(cells, order, physics, params, tri).n_dof)
    res = {}
    for prec in (_native.PRECISION_FP64, _native.PRECISION_FP32):
        s = solver_for(cells, order, physics, params, tri, precision=prec)
        s.setTimeIntegrationVector(0, u0)
        s.handle.step(0.0, dt, steps)
        res[prec] = (s, s.getTimeIntegrationVector(0))
    s64, u64 = res[_native.PRECISION_FP64]
    assert s64.l2Distance(res[_native.PRECISION_FP32][1], u64) < 1e-6
