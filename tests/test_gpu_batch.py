"""GPU: many problems advanced together by hgg_batch_* give, problem by
problem, the same coefficients as each problem stepped alone (and the oracle
for a sample), including problems that join late, leave early and take
different step counts with different dt."""
import numpy as np
import pytest

from oracle.dg import ADVECTION, WAVE, Problem
from oracle.mesh import mesh_from_description

import hpgem_b200
from hpgem_b200 import _native

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def desc(n, triangular=False):
    dim = len(n)
    return hpgem_b200.structured_description(n, [0.0] * dim, [1.0] * dim, triangular, True)


def rel_err(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def sine(x):
    return np.prod(np.sin(2 * np.pi * x), axis=1)


# (cells, triangular, order, physics, params, tableau, dt, steps)
PROBLEMS = [
    ([8, 6], False, 2, "advection", [1.0, 0.5], "RK4_4", 2e-3, 7),     # tensor, 2D
    ([10, 10], False, 2, "advection", [-0.3, 0.9], "RK4_4", 1e-3, 5),  # same class, other dt
    ([6, 4], True, 3, "advection", [0.2, -0.8], "RK4_4", 1e-3, 6),     # dense, triangles
    ([4, 6], True, 3, "advection", [0.6, 0.6], "RK4_4", 5e-4, 9),
    ([5, 4, 3], False, 3, "advection", [1.0, 0.7, 0.3], "RK4_4", 1e-3, 4),  # slice kernel
    ([4, 3, 5], False, 3, "advection", [-0.5, 0.2, 0.9], "RK4_4", 2e-3, 8),
    ([4, 4, 2], False, 2, "advection", [0.3, 0.3, -0.6], "RK4_4", 1e-3, 3),  # tensor, 3D
    ([2, 2, 2], True, 2, "wave", [1.0], "RK4_4", 1e-3, 5),              # dense, tets, wave
    ([6, 6], False, 1, "wave", [2.0], "RK4_4", 1e-3, 4),                # wave tiles, squares
    ([4, 4, 4], True, 2, "wave", [1.0], "RK4_4", 1e-3, 5),              # wave tiles, tets
    ([4, 4, 4], True, 4, "wave", [0.9], "RK4_4", 2e-4, 3),              # 16-element tiles in the batch
    ([8, 8], False, 2, "advection", [1.0, 0.5], "DormandPrince", 1e-3, 3),  # other tableau
    ([32, 32], True, 4, "advection", [0.8, -0.6], "RK4_4", 2e-4, 4),  # folded operator, tiles
    ([32, 32], True, 5, "advection", [-0.6, 0.8], "RK4_4", 1e-4, 6),
]


def make(problem):
    cells, tri, p, phys, params, tableau, dt, steps = problem
    d = len(cells)
    if phys == "advection":
        s = hpgem_b200.Advection(d, p, params, tableau=tableau)
    else:
        s = hpgem_b200.AcousticWave(d, p, c_inv=params[0], tableau=tableau)
    s.readMesh(desc(cells, tri))
    rng = np.random.default_rng(len(cells) * 100 + p)
    u0 = rng.standard_normal(s.handle.vector_length)
    s.setTimeIntegrationVector(0, u0)
    return s, u0


def alone(problem, u0):
    s, _ = make(problem)
    s.setTimeIntegrationVector(0, u0)
    s.computeTimeSteps(0.0, problem[6], problem[7])
    return s.getTimeIntegrationVector(0)


@pytest.mark.parametrize("autotune", [True, False])
def test_batch_matches_each_problem_alone(autotune):
    batch = hpgem_b200.Batch(64)
    batch.set_autotune(autotune)
    solvers, u0s, slots = [], [], []
    for pr in PROBLEMS:
        s, u0 = make(pr)
        solvers.append(s)
        u0s.append(u0)
        slots.append(batch.add(s, pr[6], pr[7]))
    assert batch.num_classes == 10
    assert solvers[-1].handle.kernel_kind == "linear"
    batch.step(max(pr[7] for pr in PROBLEMS) + 2)  # extra steps: finished problems stay put
    batch.synchronize()
    for pr, s, u0, slot in zip(PROBLEMS, solvers, u0s, slots):
        assert batch.remaining(slot) == 0
        got = s.getTimeIntegrationVector(0)
        ref = alone(pr, u0)
        assert rel_err(got, ref) < RTOL, pr
    batch.close()


def test_batch_members_join_late_and_leave_early():
    batch = hpgem_b200.Batch(8)
    a_pr, b_pr, c_pr = PROBLEMS[0], PROBLEMS[4], PROBLEMS[2]
    a, ua = make(a_pr)
    b, ub = make(b_pr)
    sa = batch.add(a, a_pr[6], a_pr[7])
    sb = batch.add(b, b_pr[6], b_pr[7])
    batch.step(2)
    batch.synchronize()
    assert batch.remaining(sa) == a_pr[7] - 2
    # a third problem joins after two steps; the first one leaves after three more
    c, uc = make(c_pr)
    sc = batch.add(c, c_pr[6], c_pr[7])
    batch.step(3)
    batch.synchronize()
    batch.remove(sa)
    # the removed problem took exactly 5 of its steps
    ref_a5 = alone((a_pr[0], a_pr[1], a_pr[2], a_pr[3], a_pr[4], a_pr[5], a_pr[6], 5), ua)
    assert rel_err(a.getTimeIntegrationVector(0), ref_a5) < RTOL
    batch.step(20)
    batch.synchronize()
    assert batch.remaining(sb) == 0 and batch.remaining(sc) == 0
    assert rel_err(b.getTimeIntegrationVector(0), alone(b_pr, ub)) < RTOL
    assert rel_err(c.getTimeIntegrationVector(0), alone(c_pr, uc)) < RTOL
    batch.close()


def test_batch_sample_against_oracle():
    pr = PROBLEMS[2]
    cells, tri, p, phys, params, tableau, dt, steps = pr
    batch = hpgem_b200.Batch(4)
    s, _ = make(pr)
    prob = Problem(mesh_from_description(desc(cells, tri)), p, ADVECTION, a=params)
    u0 = prob.project(lambda x: sine(x)[:, None])
    s.setTimeIntegrationVector(0, u0)
    slot = batch.add(s, dt, steps)
    batch.step(steps)
    batch.synchronize()
    assert rel_err(s.getTimeIntegrationVector(0), prob.step(u0, dt, steps, tableau)) < RTOL
    batch.remove(slot)
    batch.close()


def test_batch_rejects_bad_arguments():
    batch = hpgem_b200.Batch(1)
    s, _ = make(PROBLEMS[0])
    with pytest.raises(_native.NativeError):
        batch.add(s, -1.0, 3)
    batch.add(s, 1e-3, 3)
    t, _ = make(PROBLEMS[1])
    with pytest.raises(_native.NativeError):
        batch.add(t, 1e-3, 3)  # full
    with pytest.raises(_native.NativeError):
        batch.remove(5)
    batch.close()


def test_batch_steps_stored_matrix_handles():
    """HpgemAPILinear handles (grouped tile kernel) in a batch beside a matrix-free
    handle give the same coefficients as stepped alone."""
    specs = [(hpgem_b200.HpgemAPILinear, [6, 6, 6], 2, 1e-3, 5), (hpgem_b200.HpgemAPILinear, [4, 4, 4], 3, 5e-4, 3),
             (hpgem_b200.HpgemAPISimplified, [6, 6, 6], 2, 1e-3, 4)]
    a = [1.0, 0.7, 0.3]

    def build(cls, cells, p):
        s = cls(3, p, "advection", advection=a, tableau="RK4_4").readMesh(desc(cells))
        return s

    batch = hpgem_b200.Batch(8)
    runs = []
    for cls, cells, p, dt, steps in specs:
        s = build(cls, cells, p)
        u0 = np.random.default_rng(p).standard_normal(s.handle.vector_length)
        s.setTimeIntegrationVector(0, u0)
        runs.append((s, u0, batch.add(s, dt, steps)))
    assert runs[0][0].handle.kernel_kind == "linear"
    batch.step(6)
    batch.synchronize()
    for (cls, cells, p, dt, steps), (s, u0, slot) in zip(specs, runs):
        assert batch.remaining(slot) == 0
        ref = build(cls, cells, p)
        ref.setTimeIntegrationVector(0, u0)
        ref.computeTimeSteps(0.0, dt, steps)
        assert rel_err(s.getTimeIntegrationVector(0), ref.getTimeIntegrationVector(0)) < RTOL
    batch.close()
