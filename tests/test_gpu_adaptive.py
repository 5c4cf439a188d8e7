"""GPU: adaptive time steps of embedded tableaux (computeOneTimeStep(time,
maximumRelativeError, dtMax), HpgemAPISimplified_Impl.h:822-861) against the
oracle's restatement of the same control loop: the accepted dt, the number of
rejected tries, the next estimate and the solution.

Tolerances: the error estimate sum_i dt (b_i - b*_i) k_i is a small difference
of stage derivatives (about 1e-3 of their size), so their agreement (a small
multiple of cond(Mhat) eps relative to their size, from the reference's LU
solves) becomes ~1e-10 relative in the estimate, and dt ~ estimate^(-1/order)
carries 1/order of that: dt, time and the next estimate agree to 1e-9
relative.  The number of rejected tries agrees exactly.  The solution's bound
follows from that: a step whose accepted dt differs by a relative delta moves
the solution by delta times the step's update |u_new - u_old|, so after n
steps the bound is sum_steps 2 delta |u_new - u_old| / |u| plus the 1e-12 parity
bar per step (the rewind of a rejected try rounds like one more update); with
fixed dt the 1e-12 bar of the other tests holds alone."""
import math

import numpy as np
import pytest

from oracle.dg import ADVECTION, WAVE, Problem
from oracle.mesh import mesh_from_description

import hpgem_b200
from hpgem_b200 import _native

pytestmark = pytest.mark.gpu

RTOL = 1e-12
DT_RTOL = 1e-9


def rel_err(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def desc(n, triangular=False):
    d = len(n)
    return hpgem_b200.structured_description(n, [0.0] * d, [1.0] * d, triangular, True)


CASES = [
    # cells, triangular, order, physics, params, tableau, tolerance, first dt estimate
    ([8, 6], False, 2, "advection", [1.0, 0.5], "DormandPrince", 1e-6, 0.2),
    ([6, 6], True, 2, "advection", [0.3, -0.8], "DormandPrince", 1e-7, 0.5),
    ([4, 3, 3], False, 3, "advection", [1.0, 0.7, 0.3], "DormandPrince", 1e-6, 0.3),
    ([4, 4], True, 1, "wave", [1.0], "BogackiShampine", 1e-5, 0.4),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "%dD-%s-%s-p%d-%s" % (
    len(c[0]), "tri" if c[1] else "box", c[3], c[2], c[5]))
def test_adaptive_steps_against_oracle(case):
    cells, tri, p, physics, params, tableau, tol, dt0 = case
    d = len(cells)
    description = desc(cells, tri)
    if physics == "advection":
        prob = Problem(mesh_from_description(description), p, ADVECTION, a=params)
        u0 = prob.project(lambda x: np.sin(2 * np.pi * x).prod(axis=1)[:, None])
        s = hpgem_b200.Advection(d, p, params, tableau=tableau)
    else:
        prob = Problem(mesh_from_description(description), p, WAVE, cinv=params[0])
        u0 = prob.project(lambda x: np.concatenate([np.sin(2 * np.pi * x[:, :1])] + [0 * x[:, :1]] * d, axis=1))
        s = hpgem_b200.AcousticWave(d, p, c_inv=params[0], tableau=tableau)
    s.readMesh(description)
    s.setTimeIntegrationVector(0, u0)
    s.dtEstimate = dt0
    u, t, est = u0, 0.0, dt0
    total_rej = 0
    bound = 0.0
    for step in range(5):
        dt_max = 0.25
        u_prev = u
        u, t, est, dt, rej = prob.step_adaptive(u, t, tol, dt_max, est, tableau)
        tg = s.computeOneTimeStepAdaptive(t - dt, tol, dt_max)
        assert s.lastRejections == rej, step
        assert math.isclose(s.lastDt, dt, rel_tol=DT_RTOL), (step, s.lastDt, dt)
        assert math.isclose(tg, t, rel_tol=DT_RTOL)
        assert math.isclose(s.dtEstimate, est, rel_tol=DT_RTOL)
        delta = abs(s.lastDt - dt) / dt
        bound += RTOL * (1 + rej) + 2 * delta * np.abs(u - u_prev).max() / np.abs(u).max()
        assert rel_err(s.getTimeIntegrationVector(0), u) < bound, (step, bound)
        total_rej += rej
    assert total_rej >= 1  # the first estimate is too large: the control rejected a try


def test_adaptive_solve_reaches_the_final_time_and_tableaux_without_estimate_refuse():
    s = hpgem_b200.Advection(2, 2, [1.0, 0.5], tableau="DormandPrince").readMesh(desc([8, 8]))
    s.setInitialSolution(lambda x: np.sin(2 * np.pi * x).prod(axis=1))
    t, n = s.solveAdaptive(0.0, 0.05, 1e-6, numberOfOutputFrames=2)
    assert abs(t - 0.05) < 1e-12 and n >= 2
    r = hpgem_b200.Advection(2, 2, [1.0, 0.5], tableau="RK4_4").readMesh(desc([4, 4]))
    with pytest.raises(_native.NativeError):
        r.computeOneTimeStepAdaptive(0.0, 1e-6, 0.1)


def test_adaptive_steps_on_stored_matrix_handles():
    """The adaptive control on HpgemAPILinear handles (row kernel and tile kernel)
    takes the steps of the matrix-free handle of the same physics."""
    for cells, p in (([8, 8], 2), ([4, 4, 4], 3)):
        d = len(cells)
        a = [1.0, 0.5, 0.3][:d]
        out = []
        for cls in (hpgem_b200.HpgemAPILinear, hpgem_b200.HpgemAPISimplified):
            s = cls(d, p, "advection", advection=a, tableau="DormandPrince").readMesh(desc(cells, False))
            s.setInitialSolution(lambda x: np.sin(2 * np.pi * x).prod(axis=1))
            s.dtEstimate = 0.05
            steps = []
            t = 0.0
            for _ in range(4):
                t = s.computeOneTimeStepAdaptive(t, 1e-7, 0.25)
                steps.append((s.lastDt, s.lastRejections))
            out.append((steps, s.getTimeIntegrationVector(0)))
        (lin_steps, u_lin), (free_steps, u_free) = out
        assert [r for _, r in lin_steps] == [r for _, r in free_steps]
        for (x, _), (y, _) in zip(lin_steps, free_steps):
            assert math.isclose(x, y, rel_tol=DT_RTOL)
        assert rel_err(u_lin, u_free) < 1e-9
