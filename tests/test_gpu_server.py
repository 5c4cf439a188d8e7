"""GPU: the serving loop.  Each solve's result is the same served in a mix of
requests (admitted while others run, co-batched per RK stage) as solved alone
through its own handle: 1e-12 relative, the FP64 tolerance of the parity
tests.  Admission keeps the reserved device bytes within the budget."""
import time

import numpy as np
import pytest

import hpgem_b200
from hpgem_b200 import _native, workloads

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def rel_err(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def description(spec):
    dim = len(spec["cells"])
    return hpgem_b200.structured_description(spec["cells"], [0.0] * dim, [1.0] * dim, spec["triangular"], True)


def alone(spec):
    s = workloads.make_solver(spec)
    s.computeTimeSteps(0.0, spec["dt"], spec["steps"])
    return s.getTimeIntegrationVector(0).reshape(-1)


def initial(spec):
    dim = len(spec["cells"])
    u0 = spec["u0"]
    if spec["physics"] == "advection":
        return u0, 1
    return (lambda x: np.concatenate([u0(x)[:, None], np.zeros((len(x), dim))], axis=1)), dim + 1


def submit(server, spec):
    fn, nv = initial(spec)
    return server.submit(description(spec), spec["order"], spec["physics"], spec["params"], spec["dt"],
                         spec["steps"], initial=fn, n_vars=nv)


def small_stream(n, seed):
    return workloads.served_requests(n=n, seed=seed, rate=1000.0, dof_range=(500, 3e4), steps_range=(3, 40))


def test_served_results_equal_solves_alone():
    specs = small_stream(16, seed=11)
    server = hpgem_b200.Server(budget_bytes=2 << 30, max_chunk=7, setup_threads=3)
    ids = []
    for i, spec in enumerate(specs):
        ids.append(submit(server, spec))
        if i % 5 == 4:
            time.sleep(0.05)  # later requests arrive while earlier ones run
    results = [server.poll(rid, wait=True) for rid in ids]
    stats = server.stats()
    server.stop()
    assert stats["completed"] == len(specs)
    assert stats["dof_updates"] == sum(workloads.dof(s) * s["steps"] for s in specs)
    kinds = {(len(s["cells"]), s["physics"], s["order"]) for s in specs}
    assert len(kinds) > 4  # a real mix of kernel classes
    for spec, (done, u, lat) in zip(specs, results):
        assert done and lat > 0
        assert rel_err(u, alone(spec)) < RTOL, spec["id"]


def test_admission_by_footprint_with_a_tight_budget():
    specs = small_stream(8, seed=12)
    # room for about two of these solves at a time
    server = hpgem_b200.Server(budget_bytes=24 << 20, max_chunk=5, setup_threads=4)
    ids = [submit(server, s) for s in specs]
    peak = 0
    while True:
        st = server.stats()
        peak = max(peak, st["reserved_bytes"])
        if st["completed"] == len(specs):
            break
        time.sleep(0.002)
    results = [server.poll(rid, wait=True) for rid in ids]
    server.stop()
    assert peak <= 24 << 20
    for spec, (done, u, _) in zip(specs, results):
        assert rel_err(u, alone(spec)) < RTOL


def test_request_larger_than_the_budget_fails_cleanly():
    server = hpgem_b200.Server(budget_bytes=1 << 20, max_chunk=5, setup_threads=1)
    spec = small_stream(1, seed=13)[0]
    rid = submit(server, spec)
    with pytest.raises(_native.NativeError) as ex:
        server.poll(rid, wait=True)
    assert ex.value.code == -4  # HGG_ERR_NOMEM
    server.stop()


def test_more_requests_than_slots_wait_for_a_slot_and_mixed_form():
    """A server with 3 slots and 10 requests: the requests beyond the slots wait until
    members leave (none fails); FP32-mixed solves equal the same solves alone in the
    mixed form to the FP32 accumulation error."""
    specs = small_stream(10, seed=14)
    server = hpgem_b200.Server(budget_bytes=2 << 30, max_chunk=4, setup_threads=2, capacity=3)
    ids = []
    for spec in specs:
        fn, nv = initial(spec)
        ids.append(server.submit(description(spec), spec["order"], spec["physics"], spec["params"], spec["dt"],
                                 spec["steps"], initial=fn, n_vars=nv, precision=_native.PRECISION_FP32))
    results = [server.poll(rid, wait=True) for rid in ids]
    stats = server.stats()
    server.stop()
    assert stats["completed"] == len(specs)
    assert stats["device_chunk_s"] > 0 and stats["retire_thread_s"] > 0
    for spec, (done, u, _) in zip(specs, results):
        s = workloads.make_solver(spec, precision=_native.PRECISION_FP32)
        s.computeTimeSteps(0.0, spec["dt"], spec["steps"])
        assert done and rel_err(u, s.getTimeIntegrationVector(0).reshape(-1)) < 1e-5, spec["id"]
