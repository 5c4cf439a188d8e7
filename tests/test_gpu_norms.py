"""GPU: error norms evaluated on the device (computeTotalError, L2 with the rule
of order 2p+2; computeMaxError, max at the element quadrature points) against
the oracle's L2 error and a numpy evaluation of the max error, on every device
layout (tensor order, tiled tensor order, element-major, FP32 stage vectors).
Tolerance 1e-12 relative: the same sums, the elements' partial sums added in a
different order."""
import numpy as np
import pytest

from oracle.dg import ADVECTION, WAVE, Problem
from oracle.mesh import mesh_from_description

import hpgem_b200
from hpgem_b200 import _native

pytestmark = pytest.mark.gpu


def desc(n, tri=False):
    d = len(n)
    return hpgem_b200.structured_description(n, [0.0] * d, [1.0] * d, tri, True)


def exact_adv(x, t):
    return np.sin(2 * np.pi * (x[:, 0] - t)) * np.cos(2 * np.pi * x[:, -1])


def exact_wave(x, t):
    d = x.shape[1]
    return np.concatenate([np.sin(2 * np.pi * (x[:, :1] + t))] + [0.5 * np.cos(2 * np.pi * x[:, i:i + 1])
                                                                 for i in range(d)], axis=1)


CASES = [([6, 5], False, 2, "advection"), ([4, 4], True, 3, "advection"), ([4, 3, 3], False, 3, "advection"),
         ([2, 2, 2], True, 2, "wave"), ([5, 4], False, 1, "wave")]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "%dD-%s-p%d-%s" % (len(c[0]), "tri" if c[1] else "box", c[2], c[3]))
@pytest.mark.parametrize("precision", [_native.PRECISION_FP64, _native.PRECISION_FP32])
def test_device_error_norms(case, precision):
    cells, tri, p, physics = case
    d = len(cells)
    description = desc(cells, tri)
    if physics == "advection":
        prob = Problem(mesh_from_description(description), p, ADVECTION, a=[1.0] * d)
        s = hpgem_b200.Advection(d, p, [1.0] * d, tableau="RK4_4", precision=precision)
        exact = lambda x, t: exact_adv(x, t)[:, None]
    else:
        prob = Problem(mesh_from_description(description), p, WAVE, cinv=1.0)
        s = hpgem_b200.AcousticWave(d, p, c_inv=1.0, tableau="RK4_4", precision=precision)
        exact = exact_wave
    s.readMesh(description)
    rng = np.random.default_rng(3)
    u = rng.standard_normal(s.handle.vector_length)
    # the solution vector (FP64) and a stage vector (FP32 in the mixed form)
    for vec in (0, 1):
        s.setTimeIntegrationVector(vec, u)
        stored = s.getTimeIntegrationVector(vec).reshape(-1)
        ref = prob.l2_error(stored, exact, 0.3)
        got = s.computeTotalError(exact, 0.3, vec=vec)
        assert abs(got - ref) < 1e-12 * ref, (vec, got, ref)
        # max error at the element rule's points
        x = s.quadraturePoints().reshape(-1, d)
        ex = np.asarray(exact(x, 0.3)).reshape(len(prob.absdet), len(prob.rule.weights), -1)
        uh = np.einsum("qj,evj->eqv", prob.phi, stored.reshape(len(prob.absdet), ex.shape[2], -1))
        ref_max = np.abs(uh - ex).max(axis=(0, 1))
        got_max = s.computeMaxError(exact, 0.3, vec=vec)
        assert np.allclose(got_max, ref_max, rtol=1e-12, atol=0), (vec, got_max, ref_max)
