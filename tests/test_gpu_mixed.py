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

from oracle.dg import ADVECTION, WAVE, WAVE_UPWIND, Problem
from oracle.mesh import mesh_from_description

import hpgem_b200
from hpgem_b200 import _native

pytestmark = pytest.mark.gpu


def desc(n):
    return hpgem_b200.structured_description(n, [0.0] * len(n), [1.0] * len(n), False, True)


def rel_err(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def l2_distance(prob, a, b):
    """sqrt(sum_e |J_e| sum_v d_ev^T Mhat d_ev): exact L2 norm of the difference (all fields)
    on affine elements."""
    M = np.einsum("q,qi,qj->ij", prob.rule.weights, prob.phi, prob.phi)
    nB = M.shape[0]
    d = (np.asarray(a) - np.asarray(b)).reshape(len(prob.absdet), -1, nB)
    return float(np.sqrt(np.einsum("evi,ij,evj,e->", d, M, d, prob.absdet)))


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


MIXED_CASES = [
    # (cells, triangular, order, physics, params, tableau, dt, steps): the one-shot tensor
    # kernel (quads, hexahedra p != 3) and the dense kernel (simplices, the wave)
    ([12, 10], False, 2, "advection", [1.0, 0.5], "RK4_4", 1e-3, 10),
    ([5, 4, 4], False, 2, "advection", [0.6, -0.7, 0.3], "RK4_4", 1e-3, 6),
    ([8, 6], True, 3, "advection", [0.3, -0.8], "RK4_4", 1e-3, 10),
    ([2, 2, 2], True, 2, "wave", [1.0], "RK4_4", 1e-3, 8),
    ([6, 6], True, 2, "wave", [1.0], "DormandPrince", 1e-3, 5),
    ([16], False, 3, "wave", [2.0], "RK4_4", 1e-3, 10),
    ([2, 2, 2], True, 2, "wave_upwind", [1.0], "RK4_4", 1e-3, 8),
    # above 20 basis functions the mixed form contracts in FP64 (FP32 stage vectors):
    # triangles at p = 5, 100 steps at the batched set's CFL dt = 0.2 h / (2p + 1)
    ([16, 16], True, 5, "advection", [0.6, 0.8], "RK4_4", 0.2 / 16 / 11, 100),
]


@pytest.mark.parametrize("case", MIXED_CASES, ids=lambda c: "%dD-%s-%s-p%d" % (len(c[0]), "tri" if c[1] else "box", c[3], c[2]))
def test_mixed_form_on_tensor_and_dense_kernels(case):
    cells, tri, p, physics, params, tableau, dt, steps = case
    d = len(cells)
    description = hpgem_b200.structured_description(cells, [0.0] * d, [1.0] * d, tri, True)
    if physics == "advection":
        prob = Problem(mesh_from_description(description), p, ADVECTION, a=params)
        u0 = prob.project(lambda x: np.sin(2 * np.pi * x).prod(axis=1)[:, None])
    else:
        prob = Problem(mesh_from_description(description), p, WAVE_UPWIND if physics == "wave_upwind" else WAVE,
                       cinv=params[0])
        u0 = prob.project(lambda x: np.concatenate([np.sin(2 * np.pi * x[:, :1]), 0.3 * np.cos(2 * np.pi * x)], axis=1))
    ref = prob.step(u0, dt, steps, tableau)
    res = {}
    for name, prec in (("fp64", _native.PRECISION_FP64), ("fp32", _native.PRECISION_FP32)):
        if physics == "advection":
            s = hpgem_b200.Advection(d, p, params, tableau=tableau, precision=prec)
        else:
            s = hpgem_b200.AcousticWave(d, p, c_inv=params[0], tableau=tableau, precision=prec,
                                        flux="upwind" if physics == "wave_upwind" else "central")
        s.readMesh(description)
        s.setTimeIntegrationVector(0, u0)
        s.computeTimeSteps(0.0, dt, steps)
        res[name] = s.getTimeIntegrationVector(0)
    assert rel_err(res["fp64"], ref) < 1e-12
    assert rel_err(res["fp32"], ref) < 5e-7
    assert l2_distance(prob, res["fp32"], res["fp64"]) < 1e-6
    assert rel_err(res["fp32"], res["fp64"]) > 1e-12  # the mixed form really ran in reduced precision


def test_mixed_batch_equals_mixed_alone():
    """A batch of mixed-form problems (three kernel organisations) gives each problem's
    mixed result alone.  The grouped launch runs the same per-block code as the single
    launch, but the compiler may contract multiply-adds differently in the two kernels,
    which in FP32 moves stage derivatives by a few units of 6e-8; damped by dt in the FP64
    accumulation that leaves the solution within 1e-8 relative (observed 7.5e-10)."""
    specs = [([12, 10], False, 2, [1.0, 0.5]), ([8, 6], True, 3, [0.3, -0.8]), ([5, 4, 3], False, 3, [1.0, 0.7, 0.3])]
    batch = hpgem_b200.Batch(8)
    solvers, alone = [], []
    for cells, tri, p, a in specs:
        d = len(cells)
        description = hpgem_b200.structured_description(cells, [0.0] * d, [1.0] * d, tri, True)
        f = lambda x: np.sin(2 * np.pi * x).prod(axis=1)
        s = hpgem_b200.Advection(d, p, a, tableau="RK4_4", precision=_native.PRECISION_FP32).readMesh(description)
        s.setInitialSolution(f)
        t = hpgem_b200.Advection(d, p, a, tableau="RK4_4", precision=_native.PRECISION_FP32).readMesh(description)
        t.setInitialSolution(f)
        t.computeTimeSteps(0.0, 1e-3, 6)
        alone.append(t.getTimeIntegrationVector(0))
        solvers.append(s)
        batch.add(s, 1e-3, 6)
    batch.step(8)
    batch.synchronize()
    for s, ref in zip(solvers, alone):
        assert rel_err(s.getTimeIntegrationVector(0), ref) < 1e-8
    batch.close()


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
