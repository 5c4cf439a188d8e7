"""The "mesh 2" file reader (hgg_mesh_file_descriptor / hgg_create_mesh_file;
hpGEM's readMesh(fileName), kernel/Base/MeshManipulator.cpp:readMesh) against
the structured generator on the same mesh.

The three files are Preprocessor outputs of the reference's test suite
(tests/files/unitLineN4Per, unitSquareTrianglesN4Per, unitCubeN4Per); the
structured description each one was generated from is the ``source`` entry of
tests/golden/meshes.json. Read from the file or generated from the
description, the library must build the same problem: the same element order,
Jacobians, face table, face tabulations and normals, and (on the GPU) the same
time steps."""
import ctypes
import json
import os

import numpy as np
import pytest

import hpgem_b200
from hpgem_b200 import _native
from hpgem_b200.descriptor import mesh_file_descriptor, structured_descriptor

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = os.path.join(HERE, "golden", "mesh_files")
MESHES = json.load(open(os.path.join(HERE, "golden", "meshes.json")))

# (file stem, order, physics, params)
CASES = [
    ("unitLineN4Per", 3, 0, [0.7]),
    ("unitSquareTrianglesN4Per", 2, 0, [1.0, -0.5]),
    ("unitSquareTrianglesN4Per", 3, 1, [1.3]),
    ("unitCubeN4Per", 2, 0, [1.0, 0.7, 0.3]),
    ("unitCubeN4Per", 3, 2, [1.0]),
]


def source_description(stem):
    src = MESHES[stem]["source"]
    return hpgem_b200.structured_description(src["n"], src["lower"], src["upper"],
                                             src["triangular"], src["periodic"])


def path_of(stem):
    return os.path.join(FILES, stem + ".hpgem")


@pytest.mark.parametrize("stem,order,physics,params", CASES)
def test_file_and_structured_descriptors_agree(stem, order, physics, params):
    F = mesh_file_descriptor(path_of(stem), order, physics, params)
    S = structured_descriptor(source_description(stem), order, physics, params)
    assert F.keys() == S.keys()
    for key in F:
        a, b = F[key], S[key]
        if isinstance(a, np.ndarray):
            assert a.shape == b.shape, key
            if a.dtype.kind in "iu":
                assert np.array_equal(a, b), key
            else:
                # coordinates differ only in their last bits (hex floats in the file,
                # lower + i * h in the generator)
                assert np.allclose(a, b, rtol=0, atol=1e-14), key
        else:
            assert a == b, key


def test_file_element_count_matches_its_header():
    for stem in ("unitLineN4Per", "unitSquareTrianglesN4Per", "unitCubeN4Per"):
        header = open(path_of(stem)).read().split("\n")[1].split()
        D = mesh_file_descriptor(path_of(stem), 1, 0, [1.0, 0.0, 0.0])
        assert D["n_elements"] == int(header[1])
        assert D["n_elements"] == len(MESHES[stem]["element_nodes"])


def test_malformed_files_are_rejected(tmp_path):
    lib = _native.load()
    desc = _native.ProblemDesc()
    owner = ctypes.c_void_p()
    a = (ctypes.c_double * 3)(1.0, 0.5, 0.0)
    good = open(path_of("unitSquareTrianglesN4Per")).read()
    cut = good[:good.index("elements") + 40]
    bad = {
        "missing.hpgem": None,
        "version1.hpgem": good.replace("mesh 2", "mesh 1", 1),
        "truncated.hpgem": cut,
        "notamesh.hpgem": "structured 1 2\n4 4\n0 0\n1 1\nrectangular\ntrue true\n",
    }
    for name, text in bad.items():
        p = tmp_path / name
        if text is not None:
            p.write_text(text)
        rc = lib.hgg_mesh_file_descriptor(str(p).encode(), 2, 0, a, b"RK4_4", 0,
                                          ctypes.byref(desc), ctypes.byref(owner))
        assert rc == -1, name
        assert lib.hgg_last_error(None), name


@pytest.mark.gpu
@pytest.mark.parametrize("stem,order,physics,params", CASES)
def test_file_and_structured_handles_step_alike(stem, order, physics, params):
    """Same initial vector, ten RK4 steps through each handle: the solutions
    agree to rounding (the geometry differs only in the last bits of the node
    coordinates)."""
    F = hpgem_b200.Handle.mesh_file(path_of(stem), order, physics, params)
    S = hpgem_b200.Handle.structured(source_description(stem), order, physics, params)
    assert F.vector_length == S.vector_length
    rng = np.random.default_rng(3)
    u0 = rng.standard_normal(F.vector_length)
    for h in (F, S):
        h.set_state(0, u0)
        h.step(0.0, 1e-3, 10)
    a, b = F.get_state(0), S.get_state(0)
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


@pytest.mark.gpu
def test_read_mesh_file_solves_like_read_mesh():
    """The solver-level route (readMeshFile, then the 090Advection self test's
    projection, time loop and L2 error) gives the L2 error of the structured
    route on the same mesh."""
    a = [1.0, 0.7, 0.3]

    def exact(x, t):
        return np.sin(2 * np.pi * (x - t * np.asarray(a)).sum(axis=1))

    errors = []
    for route in ("file", "structured"):
        s = hpgem_b200.Advection(3, 2, a)
        if route == "file":
            s.readMeshFile(path_of("unitCubeN4Per"))
        else:
            s.readMesh(source_description("unitCubeN4Per"))
        s.setInitialSolution(lambda x: exact(x, 0.0))
        s.handle.step(0.0, 0.01, 20)
        errors.append(s.computeTotalError(exact, 0.2))
    assert abs(errors[0] - errors[1]) <= 1e-12 * errors[1]
    assert errors[0] < 0.2  # p = 2 on 4^3 hexahedra: the solution is resolved


@pytest.mark.gpu
def test_linear_read_mesh_file_steps_like_structured():
    """HpgemAPILinear from the file steps like HpgemAPILinear from its structured source."""
    out = []
    for route in ("file", "structured"):
        s = hpgem_b200.HpgemAPILinear(3, 2, "wave", c_inv=1.0, tableau="RK4_4")
        if route == "file":
            s.readMeshFile(path_of("unitCubeN4Per"))
        else:
            s.readMesh(source_description("unitCubeN4Per"))
        assert s.handle.kernel_kind == "linear"
        u0 = np.random.default_rng(4).standard_normal(s.handle.vector_length)
        s.setTimeIntegrationVector(0, u0)
        s.handle.step(0.0, 1e-3, 5)
        out.append(s.getTimeIntegrationVector(0))
    assert np.abs(out[0] - out[1]).max() <= 1e-12 * np.abs(out[1]).max()
