"""CPU-side checks of the native library: it loads, exports the C ABI, and its
host set-up (what hpGEM computes before the time loop) agrees with the oracle.
No kernel runs here."""
import ctypes
import re
import os

import numpy as np
import pytest

from oracle.dg import ADVECTION, WAVE, Problem
from oracle.mesh import mesh_from_description

import hpgem_b200
from hpgem_b200 import _native
from hpgem_b200.descriptor import structured_descriptor

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    header = open(os.path.join(ROOT, "include", "hpgem_b200.h")).read()
    declared = set(re.findall(r"\b(hgg_\w+)\s*\(", header))
    assert declared == set(_native.EXPORTED)
    for name in declared:
        assert hasattr(lib, name), name


def test_descriptor_struct_matches_header_layout():
    # the ctypes mirror must have the same field order as the C struct
    header = open(os.path.join(ROOT, "include", "hpgem_b200.h")).read()
    body = header[header.index("typedef struct hgg_problem_desc"):header.index("} hgg_problem_desc;")]
    names = re.findall(r"\*?\s*(\w+)(?:\[\d+\])?;", body)
    assert names == [f[0] for f in _native.ProblemDesc._fields_]


CASES = [
    ("structured 1 2\n4 4\n0 0\n1 1\nrectangular\ntrue true\n", 2, 0, [1.0, 0.5]),
    ("structured 1 2\n4 6\n0 0\n1 2\ntriangular\ntrue true\n", 3, 0, [0.3, -0.7]),
    ("structured 1 3\n3 3 3\n0 0 0\n1 1 1\nrectangular\ntrue true true\n", 3, 0, [1.0, 0.7, 0.3]),
    ("structured 1 3\n2 2 2\n0 0 0\n1 1 1\ntriangular\ntrue true true\n", 2, 1, [1.0]),
    ("structured 1 1\n6\n0\n1\nrectangular\ntrue\n", 4, 0, [0.7]),
]


@pytest.mark.parametrize("description,p,physics,params", CASES)
def test_host_setup_matches_oracle(description, p, physics, params):
    D = structured_descriptor(description, p, physics, params)
    mesh = mesh_from_description(description)
    prob = Problem(mesh, p, ADVECTION if physics == 0 else WAVE,
                   a=params if physics == 0 else (0, 0, 0), cinv=params[0] if physics else 1.0)
    assert D["n_elements"] == mesh.n_elements and D["n_basis"] == prob.nB
    assert np.array_equal(D["face_elements"], mesh.faces["table"][:, :2])
    assert np.array_equal(D["face_local"], mesh.faces["table"][:, 2:].astype(np.int32))
    assert np.allclose(D["quad_weights"], prob.rule.weights, rtol=0, atol=1e-15)
    assert np.allclose(D["basis_values"], prob.phi, rtol=0, atol=1e-14)
    assert np.allclose(D["basis_grads"], prob.dphi, rtol=0, atol=1e-13)
    assert np.allclose(D["face_weights"], prob.face_rule.weights, rtol=0, atol=1e-15)
    assert np.allclose(D["jacobians"], prob.J, rtol=0, atol=1e-15)
    assert np.allclose(D["face_normals"], prob.normals, rtol=0, atol=1e-14)
    # both sides of every face tabulate the same physical points
    tabs = D["face_tabs"]
    for f in range(0, len(D["face_elements"]), 7):
        tl, tr = D["face_tab_index"][f]
        fl = mesh.faces["table"][f, 2]
        assert np.allclose(tabs[tl], prob.phiF[fl], atol=1e-14)
        combo = prob.faces_c[f, 3]
        assert np.allclose(tabs[tr], prob.phiR[combo], atol=1e-14)


def test_invalid_descriptions_are_rejected():
    lib = _native.load()
    desc = _native.ProblemDesc()
    owner = ctypes.c_void_p()
    a = (ctypes.c_double * 3)(1.0, 0.5, 0.0)
    for text in ("structured 1 2\n4 4\n0 0\n1 1\nhexagonal\ntrue true\n",
                 "unstructured 1 2\n",
                 "structured 1 2\n0 4\n0 0\n1 1\nrectangular\ntrue true\n",
                 "structured 1 2\n4 4\n0 0\n1 1\nrectangular\nfalse true\n"):  # boundary faces
        rc = lib.hgg_structured_descriptor(text.encode(), 2, 0, a, b"RK4_4", 0,
                                           ctypes.byref(desc), ctypes.byref(owner))
        assert rc == -1, text
        assert lib.hgg_last_error(None)
    rc = lib.hgg_structured_descriptor(b"structured 1 2\n4 4\n0 0\n1 1\nrectangular\ntrue true\n",
                                       2, 0, a, b"NoSuchTableau", 0, ctypes.byref(desc),
                                       ctypes.byref(owner))
    assert rc == -1


def test_create_reports_a_missing_device_or_succeeds():
    lib = _native.load()
    h = ctypes.c_void_p()
    a = (ctypes.c_double * 2)(1.0, 0.5)
    rc = lib.hgg_create_structured(b"structured 1 2\n4 4\n0 0\n1 1\nrectangular\ntrue true\n",
                                   2, 0, a, b"RK4_4", 0, ctypes.byref(h))
    if rc == 0:
        lib.hgg_destroy(h)
    else:
        assert rc == -6 and b"device" in lib.hgg_last_error(None)


def test_precision_forms_are_checked_before_the_device():
    """An unknown precision is invalid (decided before looking for a device); both
    forms exist for every shape, so they get as far as the device check."""
    lib = _native.load()
    h = ctypes.c_void_p()
    a = (ctypes.c_double * 3)(1.0, 0.5, 0.3)
    quads = b"structured 1 2\n4 4\n0 0\n1 1\nrectangular\ntrue true\n"
    assert lib.hgg_create_structured(quads, 2, 0, a, b"RK4_4", 7, ctypes.byref(h)) == -1
    for text in (quads, b"structured 1 2\n4 4\n0 0\n1 1\ntriangular\ntrue true\n",
                 b"structured 1 3\n4 4 4\n0 0 0\n1 1 1\nrectangular\ntrue true true\n"):
        for prec in (_native.PRECISION_FP64, _native.PRECISION_FP32):
            rc = lib.hgg_create_structured(text, 3, 0, a, b"RK4_4", prec, ctypes.byref(h))
            if rc == 0:
                lib.hgg_destroy(h)
            else:
                assert rc == -6, (text, prec, rc)


def test_solve_step_count_rule():
    # HpgemAPISimplified::solve rounds the step count up to a multiple of the frames
    s = hpgem_b200.HpgemAPISimplified(2, 1)
    T, dt, frames = 1.0, 0.3, 3
    steps = int(np.ceil(T / dt))
    steps += (frames - steps % frames) % frames
    assert steps == 6
