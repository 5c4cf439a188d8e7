"""CPU: the oracle's upwind acoustic-wave flux, which the reference does not
have (its wave uses the central flux), so no reference golden pins it.  Its
restatement is pinned by the properties the flux must have: a plane wave
converges at order about p + 1 in L2 under refinement, and the discrete energy
int v^2 + c_inv |s|^2 decays (the central flux keeps it up to the time
integrator's own damping)."""
import math

import numpy as np

from oracle.dg import WAVE, WAVE_UPWIND, Problem
from oracle.mesh import mesh_from_description

import hpgem_b200

K = 2 * math.pi * np.array([1.0, 1.0])  # periodic on the unit square
CINV = 1.0
OMEGA = math.sqrt(K @ K / CINV)


def plane_wave(x, t):
    phase = OMEGA * t - x @ K
    v = np.cos(phase)
    s = -(K[None, :] / (CINV * OMEGA)) * np.cos(phase)[:, None]
    return np.concatenate([v[:, None], s], axis=1)


def solve(n, p, physics, T, dt):
    d = hpgem_b200.structured_description([n, n], [0.0, 0.0], [1.0, 1.0], True, True)
    prob = Problem(mesh_from_description(d), p, physics, cinv=CINV)
    u = prob.project(lambda x: plane_wave(x, 0.0))
    steps = int(round(T / dt))
    u = prob.step(u, T / steps, steps, "RK4_4")
    return prob, u


def test_upwind_plane_wave_converges_at_order_p_plus_one():
    p, T = 2, 0.2
    errs = []
    for n in (4, 8):
        prob, u = solve(n, p, WAVE_UPWIND, T, 0.02 / n)
        errs.append(prob.l2_error(u, plane_wave, T))
    rate = math.log2(errs[0] / errs[1])
    assert rate > p + 0.5, (errs, rate)


def energy(prob, u):
    M = np.einsum("q,qi,qj->ij", prob.rule.weights, prob.phi, prob.phi)
    uu = np.asarray(u).reshape(len(prob.absdet), 3, -1)
    w = np.array([1.0, CINV, CINV])
    return float(np.einsum("evi,ij,evj,e,v->", uu, M, uu, prob.absdet, w))


def test_upwind_flux_dissipates_energy_and_central_keeps_it():
    d = hpgem_b200.structured_description([6, 6], [0.0, 0.0], [1.0, 1.0], True, True)
    res = {}
    for name, phys in (("central", WAVE), ("upwind", WAVE_UPWIND)):
        prob = Problem(mesh_from_description(d), 2, phys, cinv=CINV)
        u = prob.project(lambda x: np.concatenate(
            [np.exp(-((x - 0.5) ** 2).sum(1, keepdims=True) / 0.02), np.zeros((len(x), 2))], axis=1))
        e = [energy(prob, u)]
        for _ in range(10):
            u = prob.step(u, 2e-3, 5, "RK4_4")
            e.append(energy(prob, u))
        res[name] = np.array(e)
    up = res["upwind"]
    assert np.all(np.diff(up) < 0)
    assert up[-1] < 0.999 * up[0]
    ce = res["central"]
    assert abs(ce[-1] - ce[0]) < 1e-4 * ce[0]
