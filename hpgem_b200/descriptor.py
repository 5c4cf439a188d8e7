"""Reads the host-built hgg_problem_desc of a structured mesh into numpy arrays
(hgg_structured_descriptor: the tabulations, geometry and face table the
library builds from a Preprocessor structured description)."""
import ctypes

import numpy as np

from . import _native


def _arr(ptr, shape, dtype):
    n = int(np.prod(shape))
    ctype = {np.float64: ctypes.c_double, np.int64: ctypes.c_int64, np.int32: ctypes.c_int32}[dtype]
    if n == 0:
        return np.zeros(shape, dtype=dtype)
    buf = (ctype * n).from_address(ptr)
    return np.ctypeslib.as_array(buf).reshape(shape).astype(dtype).copy()


def structured_descriptor(description, order, physics, params, tableau="RK4_4"):
    return _descriptor("hgg_structured_descriptor", description, order, physics, params, tableau)


def mesh_file_descriptor(path, order, physics, params, tableau="RK4_4"):
    """The descriptor of a Preprocessor "mesh 2" file (hgg_mesh_file_descriptor)."""
    return _descriptor("hgg_mesh_file_descriptor", path, order, physics, params, tableau)


def _descriptor(entry, source, order, physics, params, tableau):
    lib = _native.load()
    desc = _native.ProblemDesc()
    owner = ctypes.c_void_p()
    p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
    _native.check(getattr(lib, entry)(source.encode(), order, physics,
                                      ctypes.c_void_p(p.ctypes.data), tableau.encode(), 0,
                                      ctypes.byref(desc), ctypes.byref(owner)))
    try:
        d, nB, nQ, nQf = desc.dim, desc.n_basis, desc.n_quad, desc.n_face_quad
        E, F, S = desc.n_elements, desc.n_faces, desc.n_stages
        out = dict(
            dim=d, shape=desc.shape, order=desc.order, n_vars=desc.n_vars, physics=desc.physics,
            advection=np.array(desc.advection[:3]), c_inv=desc.c_inv, n_elements=E, n_basis=nB,
            quad_weights=_arr(desc.quad_weights, (nQ,), np.float64),
            basis_values=_arr(desc.basis_values, (nQ, nB), np.float64),
            basis_grads=_arr(desc.basis_grads, (nQ, nB, d), np.float64),
            face_weights=_arr(desc.face_weights, (nQf,), np.float64),
            face_tabs=_arr(desc.face_tabs, (desc.n_face_tabs, nQf, nB), np.float64),
            jacobians=_arr(desc.jacobians, (E, d, d), np.float64),
            face_elements=_arr(desc.face_elements, (F, 2), np.int64),
            face_local=_arr(desc.face_local, (F, 2), np.int32),
            face_tab_index=_arr(desc.face_tab_index, (F, 2), np.int32),
            face_normals=_arr(desc.face_normals, (F, d), np.float64),
            rk_a=_arr(desc.rk_a, (S, S), np.float64), rk_b=_arr(desc.rk_b, (S,), np.float64),
            rk_c=_arr(desc.rk_c, (S,), np.float64))
    finally:
        lib.hgg_free_descriptor(owner)
    return out


def linear_descriptor(description, order, physics, params, tableau="RK4_4"):
    """The stored matrices hgg_linear_descriptor assembles (HpgemAPILinear's
    createMassMatrices / createStiffnessMatrices for the reference's linear
    advection and wave applications) as numpy arrays."""
    lib = _native.load()
    desc = _native.LinearDesc()
    owner = ctypes.c_void_p()
    p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
    _native.check(lib.hgg_linear_descriptor(description.encode(), order, physics,
                                            ctypes.c_void_p(p.ctypes.data), tableau.encode(), 0,
                                            ctypes.byref(desc), ctypes.byref(owner)))
    try:
        R, E, F, S = desc.n_rows, desc.n_elements, desc.n_faces, desc.n_stages
        out = dict(
            n_rows=R, n_elements=E, n_faces=F,
            mass=_arr(desc.mass, (E, R, R), np.float64),
            element_stiffness=_arr(desc.element_stiffness, (E, R, R), np.float64),
            face_elements=_arr(desc.face_elements, (F, 2), np.int64),
            face_stiffness=_arr(desc.face_stiffness, (F, 4, R, R), np.float64),
            rk_a=_arr(desc.rk_a, (S, S), np.float64), rk_b=_arr(desc.rk_b, (S,), np.float64),
            rk_c=_arr(desc.rk_c, (S,), np.float64))
    finally:
        lib.hgg_free_linear_descriptor(owner)
    return out
