"""GPU: hgg_time_derivative_static (right-hand side of caller-owned device
vectors, scratch from a static device array, no allocation) against the
existing hgg_time_derivative on the same state, on two calls in a row.

Collected last (file name) so that it runs after the other GPU tests as well
as alone in a fresh process."""
import ctypes

import numpy as np
import pytest
import torch

import hpgem_b200
from hpgem_b200 import _native

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the solution tolerance of the parity tests


def rel_err(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def description(n, triangular=False):
    dim = len(n)
    return hpgem_b200.structured_description(n, [0.0] * dim, [1.0] * dim, triangular, True)


CASES = [
    # (name, cells, order, velocity, triangular): the slice kernel (tiled layout),
    # the pipelined sum-factorised kernel, the dense kernel (no scratch needed)
    ("hexahedra p=3", [6, 5, 4], 3, [1.0, -0.7, 0.3], False),
    ("hexahedra p=2", [5, 4, 3], 2, [0.4, 0.9, -0.2], False),
    ("triangles p=2", [8, 6], 2, [1.0, 0.5], True),
]


def existing_entry_point(handle, u):
    handle.set_state(0, u)
    handle.time_derivative(0, 1)
    return handle.get_state(1)


@pytest.mark.parametrize("name,cells,order,velocity,triangular", CASES, ids=[c[0] for c in CASES])
def test_static_scratch_rhs_matches_time_derivative(name, cells, order, velocity, triangular):
    solver = hpgem_b200.Advection(len(cells), order, velocity).readMesh(description(cells, triangular))
    h = solver.handle
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
