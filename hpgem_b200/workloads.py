"""Seeded synthetic workloads of many problems: the batched set (512 independent
2D advection problems) and the served request stream (Poisson arrivals of 2D/3D
advection and acoustic-wave solves).  Both stand in for the reference's
single-mesh runs scaled out; every draw is reproducible from its seed."""
import math

import numpy as np

from .solver import AcousticWave, Advection, structured_description


def _sine_modes(rng, dim, modes=2):
    """u0 = sum_m A_m sin(2 pi k_m . x + phi_m), k_m integer (periodic), 1 <= |k|_inf <= 3."""
    ks, amps, phases = [], [], []
    for _ in range(modes):
        while True:
            k = rng.integers(-3, 4, size=dim)
            if np.abs(k).max() >= 1:
                break
        ks.append(k)
        amps.append(rng.uniform(0.5, 1.0))
        phases.append(rng.uniform(0.0, 2 * math.pi))
    ks = np.array(ks, dtype=float)
    amps = np.array(amps)
    phases = np.array(phases)

    def u0(x):
        return (amps[None, :] * np.sin(2 * math.pi * x @ ks.T + phases[None, :])).sum(axis=1)

    return u0


def batched_problems(n=512, seed=4, steps=100):
    """512 2D advection problems: mesh size N ~ round(exp(U(ln 8, ln 128))) per direction
    (even for triangles, which periodic simplex meshes need), quads or triangles 50/50,
    p ~ U{1..5}, a = (cos t, sin t) with t ~ U(0, 2 pi), a 2-mode sine initial condition,
    RK4 with dt = 0.2 h / (|a| (2p + 1)) (h = 1/N), `steps` steps each."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        N = int(round(math.exp(rng.uniform(math.log(8), math.log(128)))))
        tri = bool(rng.integers(0, 2))
        if tri and N % 2:
            N += 1
        p = int(rng.integers(1, 6))
        th = rng.uniform(0, 2 * math.pi)
        a = [math.cos(th), math.sin(th)]
        dt = 0.2 * (1.0 / N) / (2 * p + 1)
        out.append(dict(cells=[N, N], triangular=tri, order=p, physics="advection", params=a,
                        dt=dt, steps=steps, u0=_sine_modes(rng, 2)))
    return out


def _cells_for_dof(rng, dim, tri, nb_v, target_dof):
    per_cell = (2 if dim == 2 else 5) if tri else 1
    n = max(2, int(round((target_dof / (nb_v * per_cell)) ** (1.0 / dim))))
    if tri and n % 2:
        n += 1
    return [n] * dim


def served_requests(n=2000, seed=5, rate=200.0, dof_range=(1e3, 2e6), steps_range=(50, 2000)):
    """Poisson arrivals (rate per second) of advection / acoustic-wave solves, 50/50, 2D/3D
    50/50, DoF ~ log-uniform over dof_range (the mesh size solved from the DoF per element),
    p ~ U{1..4}, steps ~ U{steps_range}.  2D: quads for advection, triangles for the wave;
    3D: hexahedra for advection, tetrahedra for the wave (the wave's dense kernel holds at
    most 256 coefficients per element, which rules out hexahedra above p = 2)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        wave = bool(rng.integers(0, 2))
        dim = 2 + int(rng.integers(0, 2))
        p = int(rng.integers(1, 5))
        target = math.exp(rng.uniform(math.log(dof_range[0]), math.log(dof_range[1])))
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        tri = wave
        if dim == 2:
            nb = (p + 1) * (p + 2) // 2 if tri else (p + 1) ** 2
        else:
            nb = (p + 1) * (p + 2) * (p + 3) // 6 if tri else (p + 1) ** 3
        V = dim + 1 if wave else 1
        cells = _cells_for_dof(rng, dim, tri, nb * V, target)
        h = 1.0 / cells[0]
        if wave:
            params = [1.0]
            dt = 0.1 * h / (2 * p + 1)
        else:
            v = rng.normal(size=dim)
            v /= np.linalg.norm(v)
            params = list(v)
            dt = 0.2 * h / (2 * p + 1)
        out.append(dict(id=i, arrival=t, cells=cells, triangular=tri, order=p,
                        physics="wave" if wave else "advection", params=params, dt=dt, steps=steps,
                        u0=_sine_modes(rng, dim)))
    return out


def make_solver(spec, precision=0, tableau="RK4_4"):
    """A solver with its mesh read and its initial condition projected."""
    dim = len(spec["cells"])
    if spec["physics"] == "advection":
        s = Advection(dim, spec["order"], spec["params"], tableau=tableau, precision=precision)
    else:
        s = AcousticWave(dim, spec["order"], c_inv=spec["params"][0], tableau=tableau, precision=precision,
                         flux="upwind" if spec["physics"] == "wave_upwind" else "central")
    s.readMesh(structured_description(spec["cells"], [0.0] * dim, [1.0] * dim, spec["triangular"], True))
    if spec["physics"] == "advection":
        s.setInitialSolution(spec["u0"])
    else:
        u0 = spec["u0"]
        s.setInitialSolution(lambda x: np.concatenate([u0(x)[:, None], np.zeros((len(x), dim))], axis=1))
    return s


def dof(spec):
    dim = len(spec["cells"])
    p = spec["order"]
    tri = spec["triangular"]
    cells = int(np.prod(spec["cells"])) * ((2 if dim == 2 else 5) if tri else 1)
    if dim == 2:
        nb = (p + 1) * (p + 2) // 2 if tri else (p + 1) ** 2
    else:
        nb = (p + 1) * (p + 2) * (p + 3) // 6 if tri else (p + 1) ** 3
    V = 1 if spec["physics"] == "advection" else dim + 1
    return cells * nb * V
