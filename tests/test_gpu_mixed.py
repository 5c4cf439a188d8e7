"""GPU: the FP32-mixed form (stage vectors and contractions in FP32; solution,
geometry and the Runge-Kutta accumulation in FP64) against the FP64 form and
the oracle.

Tolerances (FP32 unit round-off 6e-8):
* stage derivatives: 1e-5 relative to the largest entry.  Each output sums
  about 40 FP32 products of operator entries (|D| <= 5) scaled by the
  geometry (|ahat| = 2|a|/h) with values up to the largest stage input.
* solution after N steps: 5e-7 relative, and the L2 distance to the FP64
  solution at most 1e-6 (the accuracy target of the mixed form); dt damps the
  stage-derivative rounding in the FP64 accumulation.
"""
import numpy as np
import pytest

from oracle.dg import ADVECTION, Problem
from oracle.mesh import mesh_from_description

import hpgem_b200
from hpgem_b200 import _native

pytestmark = pytest.mark.gpu


def desc(n):
    return hpgem_b200.structured_description(n, [0.0] * len(n), [1.0] * len(n), False, True)


def rel_err(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def l2_distance(prob, a, b):
    """sqrt(sum_e |J_e| d_e^T Mhat d_e): exact L2 norm of the difference on affine elements."""
    M = np.einsum("q,qi,qj->ij", prob.rule.weights, prob.phi, prob.phi)
    d = (np.asarray(a) - np.asarray(b)).reshape(len(prob.absdet), -1)
    return float(np.sqrt(np.einsum("ei,ij,ej,e->", d, M, d, prob.absdet)))


def bump(x):
    return np.exp(-((x - 0.5) ** 2).sum(axis=1) / 0.01)


@pytest.mark.parametrize("cells,tableau,steps", [([6, 5, 4], "RK4_4", 10), ([9, 7, 5], "DormandPrince", 4)])
def test_hex_p3_mixed_against_fp64_and_oracle(cells, tableau, steps):
    a = [1.0, 0.7, 0.3]
    dt = 1e-3
    description = desc(cells)
    prob = Problem(mesh_from_description(description), 3, ADVECTION, a=a)
    u0 = prob.project(lambda x: bump(x)[:, None])
    ref, ref_k = prob.step(u0, dt, steps, tableau, return_stages=True)
    res = {}
    for name, prec in (("fp64", _native.PRECISION_FP64), ("fp32", _native.PRECISION_FP32)):
        s = hpgem_b200.Advection(3, 3, a, tableau=tableau, precision=prec).readMesh(description)
        s.setTimeIntegrationVector(0, u0)
        s.computeTimeSteps(0.0, dt, steps)
        res[name] = (s.getTimeIntegrationVector(0), [s.getTimeIntegrationVector(i + 1) for i in range(len(ref_k))])
    u64, k64 = res["fp64"]
    u32, k32 = res["fp32"]
    assert rel_err(u64, ref) < 1e-12
    for a32, b in zip(k32, ref_k):
        assert rel_err(a32, b) < 1e-5
    assert rel_err(u32, ref) < 5e-7
    assert l2_distance(prob, u32, u64) < 1e-6
    assert rel_err(u32, u64) > 1e-12  # the mixed form really ran in reduced precision


def test_mixed_time_derivative_maps_solution_to_stage_vector():
    s = hpgem_b200.Advection(3, 3, [1.0, 0.7, 0.3], precision=_native.PRECISION_FP32).readMesh(desc([4, 4, 4]))
    s.setInitialSolution(bump)
    s.computeTimeDerivative(0, 1)
    k = s.getTimeIntegrationVector(1)
    f = hpgem_b200.Advection(3, 3, [1.0, 0.7, 0.3]).readMesh(desc([4, 4, 4]))
    f.setInitialSolution(bump)
    f.computeTimeDerivative(0, 1)
    assert rel_err(k, f.getTimeIntegrationVector(1)) < 1e-5
    with pytest.raises(_native.NativeError):
        s.computeTimeDerivative(1, 2)  # FP32 stage vector as input
