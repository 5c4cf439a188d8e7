"""CPU: the seeded synthetic workloads of the batched and served legs have the shape
the benchmark states: the served stream is 2000 Poisson arrivals at 200 per second
(mean gap 5 ms), advection / wave and 2D / 3D about half each, orders 1..4, DoF
log-uniform in 1e3..2e6 and steps in 50..2000; the same requests at a lower rate
are the same draws with stretched arrival times; the batched set is 512 2D advection
problems on 8^2..128^2 cells at orders 1..5.  All reproducible from their seeds."""
import math

import numpy as np

from hpgem_b200 import workloads


def test_served_stream_shape():
    specs = workloads.served_requests()
    assert len(specs) == 2000
    gaps = np.diff([0.0] + [s["arrival"] for s in specs])
    assert abs(gaps.mean() - 1 / 200) < 0.1 / 200
    wave = np.mean([s["physics"] == "wave" for s in specs])
    three_d = np.mean([len(s["cells"]) == 3 for s in specs])
    assert 0.45 < wave < 0.55 and 0.45 < three_d < 0.55
    assert {s["order"] for s in specs} == {1, 2, 3, 4}
    steps = np.array([s["steps"] for s in specs])
    assert steps.min() >= 50 and steps.max() <= 2000
    dofs = np.array([workloads.dof(s) for s in specs], dtype=float)
    # the mesh is solved from the target DoF, so sizes land near the log-uniform range
    assert dofs.min() > 1e2 and dofs.max() < 4e6
    lg = np.log(dofs)
    assert abs(lg.mean() - 0.5 * (math.log(1e3) + math.log(2e6))) < 0.5


def test_lower_rate_stretches_the_same_requests():
    a = workloads.served_requests(n=50)
    b = workloads.served_requests(n=50, rate=20.0)
    for x, y in zip(a, b):
        assert x["cells"] == y["cells"] and x["order"] == y["order"] and x["steps"] == y["steps"]
        assert abs(y["arrival"] - 10.0 * x["arrival"]) < 1e-9 * max(1.0, y["arrival"])


def test_batched_set_shape_and_seed():
    a, b = workloads.batched_problems(), workloads.batched_problems()
    assert len(a) == 512
    assert all(len(s["cells"]) == 2 and 8 <= s["cells"][0] <= 128 for s in a)
    assert all(not s["triangular"] or s["cells"][0] % 2 == 0 for s in a)  # periodic simplices
    assert {s["order"] for s in a} == {1, 2, 3, 4, 5}
    assert [s["cells"] for s in a] == [s["cells"] for s in b]
