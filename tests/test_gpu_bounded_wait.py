"""GPU: the device-side failure path of the pipelined kernel.

Every mbarrier wait of the pipelined sum-factorised kernel is bounded.  The
test hook hgg_test_arm_without_copy makes the next launch arm the mbarrier of
each block's first tile with the tile's byte count while issuing no copy for
it (nothing is in flight for that tile), with a small poll limit: the wait
runs out, every block waits for the copies it did issue, sets bit 1 of the
status word and returns.  The host sees HGG_ERR_DEVICE with the bit named;
the CUDA context stays usable (a new handle then computes the right-hand side
the oracle gives).  No copy is left in flight, nothing faults or hangs."""
import numpy as np
import pytest

import hpgem_b200
from hpgem_b200 import _native
from oracle.dg import ADVECTION, Problem
from oracle.mesh import mesh_from_description

pytestmark = pytest.mark.gpu


def description():
    # 300^2 quadrilaterals at p = 2: 1072 tiles of 84 elements, several per block of the
    # persistent grid, so every block also has real tile loads in flight when it gives up
    return hpgem_b200.structured_description([300, 300], [0.0, 0.0], [1.0, 1.0])


def pipelined_solver():
    solver = hpgem_b200.Advection(2, 2, [1.0, 0.5], tableau="RK4_4").readMesh(description())
    solver.handle.set_kernel_variant(2)
    return solver


def test_wait_that_runs_out_sets_status_bit_1():
    solver = pipelined_solver()
    h = solver.handle
    lib = _native.load()
    u = np.random.default_rng(2).standard_normal(h.vector_length)
    h.set_state(0, u)
    assert lib.hgg_test_arm_without_copy(h._raw, 256) == 0
    rc = lib.hgg_time_derivative(h._raw, 0, 1)
    assert rc == -5  # HGG_ERR_DEVICE
    msg = lib.hgg_last_error(h._raw)
    assert b"bounded wait ran out (bit 1)" in msg, msg
    assert b"neighbour" not in msg and b"matrix" not in msg
    assert lib.hgg_synchronize(h._raw) == -5  # the status word stays set
    h.close()

    # the context is intact: a fresh handle on the same kernel gives the oracle's result
    solver = pipelined_solver()
    h = solver.handle
    h.set_state(0, u)
    h.time_derivative(0, 1)
    got = h.get_state(1)
    prob = Problem(mesh_from_description(description()), 2, ADVECTION, a=[1.0, 0.5])
    ref = prob.time_derivative(u.reshape(prob.mesh.n_elements, -1)).reshape(-1)
    assert np.abs(got.reshape(-1) - ref).max() / np.abs(ref).max() < 1e-12


def test_hook_only_on_the_pipelined_kernel():
    lib = _native.load()
    solver = hpgem_b200.Advection(2, 2, [1.0, 0.5], tableau="RK4_4").readMesh(description())
    h = solver.handle
    h.set_kernel_variant(1)  # one-shot kernel: no mbarrier
    assert lib.hgg_test_arm_without_copy(h._raw, 256) == -2
    assert lib.hgg_test_arm_without_copy(h._raw, 0) == -1
