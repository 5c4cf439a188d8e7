"""Oracle driver: set-up in numpy, time stepping in C (test infrastructure only).

``Problem`` gathers what hpGEM's PhysicalElement / PhysicalFace provide at
quadrature points and hands it to oracle/dg_oracle.c:
* element rule of order 2p+1 (Element::setDefaultBasisFunctionSet,
  kernel/Base/Element.cpp:89-98, orderCoeff_ = 2 in Element.h:575) and the face
  rule of the same requested order 2p+1 (Element::setQuadratureRulesWithOrder
  hands it to the element's faces, kernel/Base/Element.cpp:144-175);
* basis values and reference gradients at the element points;
* the element Jacobian of the vertex map (MappingToPhysSimplexLinear,
  MappingToPhysHypercubeLinear), constant on the affine elements of
  structured meshes;
* per face, the left side's basis values at the face points mapped into the
  left element through the local face, the right side's through the
  face-to-face vertex correspondence (FaceGeometry::mapRefFaceToRefElemR /
  mapRefFaceToRefFace, kernel/Geometry/FaceGeometry.h:372-395);
* the normal from the left element, outward, with length equal to the ratio
  of physical to reference face measure (FaceGeometry::getNormalVector,
  FaceGeometry.h:412-459).
Butcher tableaux restate kernel/Base/TimeIntegration/{RK4Methods,DormandPrince,
ForwardEuler,MidPoint,RK2TVD,RK3TVD,BogackiShampine}.cpp.
"""
import ctypes
import math

import numpy as np

from . import build as _build
from .basis import tabulate
from .mesh import Mesh
from .quadrature import get_rule
from .refgeom import SHAPES, vertex_shape_functions

ADVECTION = 0
WAVE = 1
WAVE_UPWIND = 2  # the wave with the upwind flux (restated; the reference has the central flux)

TABLEAUX = {
    # RK4Methods.cpp:45-63
    "RK4_4": dict(order=4, A=[[0, 0, 0, 0], [0.5, 0, 0, 0], [0.0, 0.5, 0, 0], [0.0, 0.0, 1.0, 0]],
                  b=[1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6], c=[0.0, 0.5, 0.5, 1.0]),
    # DormandPrince.cpp:45-78 (fifth-order weights; the published Dormand-Prince 5(4) pair)
    "DormandPrince": dict(order=5, A=[
        [0] * 7,
        [1. / 5.] + [0] * 6,
        [3. / 40., 9. / 40.] + [0] * 5,
        [44. / 45., -56. / 15., 32. / 9.] + [0] * 4,
        [19372. / 6561., -25360. / 2187., 64448. / 6561., -212. / 729.] + [0] * 3,
        [9017. / 3168., -355. / 33., 46732. / 5247., 49. / 176., -5103. / 18656.] + [0] * 2,
        [35. / 384., 0., 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84., 0]],
        b=[35. / 384., 0., 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84., 0.],
        c=[0., 1. / 5., 3. / 10., 4. / 5., 8. / 9., 1., 1.]),
    # ForwardEuler.cpp, MidPoint.cpp, RK2TVD.cpp, RK3TVD.cpp
    "ForwardEuler": dict(order=1, A=[[0]], b=[1.0], c=[0.0]),
    "MidPoint": dict(order=2, A=[[0, 0], [0.5, 0]], b=[0.0, 1.0], c=[0.0, 0.5]),
    "RK2TVD": dict(order=2, A=[[0, 0], [1.0, 0]], b=[0.5, 0.5], c=[0.0, 0.0]),
    "RK3TVD": dict(order=3, A=[[0, 0, 0], [1.0, 0, 0], [0.25, 0.25, 0]],
                   b=[1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0], c=[0.0, 0.0, 0.0]),
    # BogackiShampine.cpp:48-62 (its c_ copies the first Dormand-Prince nodes)
    "BogackiShampine": dict(order=3, A=[[0, 0, 0, 0], [1. / 2., 0, 0, 0], [0., 3. / 4., 0, 0],
                                        [2. / 9., 1. / 3., 4. / 9., 0]],
                            b=[2. / 9., 1. / 3., 4. / 9., 0.], c=[0., 1. / 5., 3. / 10., 4. / 5.]),
}


# error coefficients b_i - b*_i of the embedded pairs (DormandPrince.cpp:75-82,
# BogackiShampine.cpp:61-67); the order used by the step-size control is the tableau's
ERROR_COEFFICIENTS = {
    "DormandPrince": [35. / 384. - 5179. / 57600., 0. - 0., 500. / 1113. - 7571. / 16695.,
                      125. / 192. - 393. / 640., -2187. / 6784. - -92097. / 339200.,
                      11. / 84. - 187. / 2100., 0. - 1. / 40.],
    "BogackiShampine": [2. / 9. - 7. / 24., 1. / 3. - 1. / 4., 4. / 9. - 1. / 3., 0. - 1. / 8.],
}


class _CProblem(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("nB", ctypes.c_int), ("nQ", ctypes.c_int),
                ("nQf", ctypes.c_int), ("V", ctypes.c_int), ("nFL", ctypes.c_int),
                ("physics", ctypes.c_int), ("a", ctypes.c_double * 3), ("cinv", ctypes.c_double),
                ("wq", ctypes.c_void_p), ("phi", ctypes.c_void_p), ("dphi", ctypes.c_void_p),
                ("wqf", ctypes.c_void_p), ("phiF", ctypes.c_void_p), ("phiR", ctypes.c_void_p),
                ("nE", ctypes.c_long), ("nF", ctypes.c_long), ("jac", ctypes.c_void_p),
                ("absdet", ctypes.c_void_p), ("faces", ctypes.c_void_p),
                ("normal", ctypes.c_void_p)]


_lib = None


def _library():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(_build.build())
        for name in ("oracle_step", "oracle_time_derivative", "oracle_project"):
            getattr(_lib, name).restype = ctypes.c_int
    return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def face_map_to_element(shape, local_face_vertices, xi):
    """Reference-face points -> element reference points through the face's vertices."""
    fshape = SHAPES[shape]["face_shape"]
    N = vertex_shape_functions(fshape, xi)
    verts = SHAPES[shape]["vertices"][local_face_vertices]
    return N @ verts


def element_jacobians(shape, coords):
    """Jacobian dx/dxi of the vertex map, evaluated at the reference centroid."""
    d = SHAPES[shape]["dim"]
    centre = SHAPES[shape]["vertices"].mean(axis=0)
    h = 1e-30
    J = np.empty((len(coords), d, d))
    for c in range(d):
        xc = centre.astype(complex)
        xc[c] += 1j * h
        N = vertex_shape_functions(shape, xc[None, :])[0]
        J[:, :, c] = np.imag(np.einsum("k,ekr->er", N, coords)) / h
    return J


class Problem:
    """One mesh + order + physics, laid out for the C oracle."""

    def __init__(self, mesh: Mesh, p: int, physics: int, a=(0.0, 0.0, 0.0), cinv=1.0):
        shape = mesh.shape
        d = SHAPES[shape]["dim"]
        self.mesh, self.p, self.physics, self.shape, self.dim = mesh, p, physics, shape, d
        self.V = 1 if physics == ADVECTION else d + 1
        self.a = np.zeros(3)
        self.a[:d] = np.asarray(a, dtype=float)[:d]
        self.cinv = float(cinv)
        self.rule = get_rule(shape, 2 * p + 1)
        fshape = SHAPES[shape]["face_shape"]
        # faces get the rule of the requested order 2p+1 when the element's rule is set
        # (Element::setQuadratureRulesWithOrder, kernel/Base/Element.cpp:144-175; the
        # faces were created under the empty basis's rule, Element.h:583, Face.cpp:149-168)
        self.face_rule = get_rule(fshape, 2 * p + 1)
        self.phi, self.dphi = tabulate(shape, p, self.rule.points)
        self.nB = self.phi.shape[1]
        self.J = element_jacobians(shape, mesh.element_coords)
        self.absdet = np.abs(np.linalg.det(self.J)) if d > 0 else np.ones(len(self.J))
        fl = SHAPES[shape]["faces"]
        xi = self.face_rule.points
        self.phiF = np.stack([tabulate(shape, p, face_map_to_element(shape, loc, xi))[0]
                              for loc in fl])
        table = mesh.faces["table"]
        perms = mesh.faces["perm"]
        combos = {}
        right = np.empty(len(table), dtype=np.int64)
        for i, row in enumerate(table):
            if row[1] < 0:
                right[i] = 0
                continue
            key = (int(row[3]), tuple(perms[i]))
            if key not in combos:
                combos[key] = len(combos)
            right[i] = combos[key]
        self.combos = list(combos.keys())
        phiR = []
        for fR, perm in self.combos:
            loc = [fl[fR][k] for k in perm]
            phiR.append(tabulate(shape, p, face_map_to_element(shape, loc, xi))[0])
        if not phiR:
            phiR = [np.zeros_like(self.phiF[0])]
        self.phiR = np.stack(phiR)
        self.faces_c = np.ascontiguousarray(
            np.stack([table[:, 0], table[:, 1], table[:, 2], right], axis=1).astype(np.int64))
        self.normals = self._normals()
        self._c = None

    def _normals(self):
        shape, d = self.shape, self.dim
        table = self.mesh.faces["table"]
        coords = self.mesh.element_coords
        fl = SHAPES[shape]["faces"]
        fshape = SHAPES[shape]["face_shape"]
        out = np.zeros((len(table), d))
        fverts = SHAPES[fshape]["vertices"]
        fcentre = fverts.mean(axis=0) if len(fverts) else np.zeros(0)
        for i, (L, _, fL, _) in enumerate(table):
            J = self.J[L]
            loc = fl[fL]
            ec = coords[L].mean(axis=0)
            fc = coords[L][loc].mean(axis=0)
            if d == 1:
                n = np.array([1.0])
            else:
                h = 1e-30
                T = np.empty((d, d - 1))
                for c in range(d - 1):
                    xc = fcentre.astype(complex)
                    xc[c] += 1j * h
                    pr = face_map_to_element(shape, loc, xc[None, :])[0]
                    T[:, c] = J @ (np.imag(pr) / h)
                n = np.array([T[1, 0], -T[0, 0]]) if d == 2 else np.cross(T[:, 0], T[:, 1])
            if np.dot(n, fc - ec) < 0:
                n = -n
            out[i] = n
        return out

    # -- C view -----------------------------------------------------------------
    def _cstruct(self):
        if self._c is None:
            keep = dict(
                wq=np.ascontiguousarray(self.rule.weights, dtype=float),
                phi=np.ascontiguousarray(self.phi), dphi=np.ascontiguousarray(self.dphi),
                wqf=np.ascontiguousarray(self.face_rule.weights, dtype=float),
                phiF=np.ascontiguousarray(self.phiF), phiR=np.ascontiguousarray(self.phiR),
                jac=np.ascontiguousarray(self.J), absdet=np.ascontiguousarray(self.absdet),
                faces=self.faces_c, normal=np.ascontiguousarray(self.normals))
            s = _CProblem()
            s.dim, s.nB, s.nQ, s.nQf = self.dim, self.nB, len(self.rule), len(self.face_rule)
            s.V, s.nFL, s.physics = self.V, len(SHAPES[self.shape]["faces"]), self.physics
            for k in range(3):
                s.a[k] = self.a[k]
            s.cinv = self.cinv
            for k, v in keep.items():
                setattr(s, k, _ptr(v))
            s.nE, s.nF = self.mesh.n_elements, len(self.faces_c)
            self._c = (s, keep)
        return self._c[0]

    @property
    def n_dof(self):
        return self.mesh.n_elements * self.V * self.nB

    def quadrature_points(self):
        """Physical coordinates of every element quadrature point, [nE][nQ][dim]."""
        N = vertex_shape_functions(self.shape, self.rule.points)
        return np.einsum("qk,ekr->eqr", N, self.mesh.element_coords)

    def project(self, u0):
        """setInitialSolution: L2 projection of u0(x[n, dim]) -> [n, V]."""
        x = self.quadrature_points()
        vals = np.asarray(u0(x.reshape(-1, self.dim)), dtype=float).reshape(
            self.mesh.n_elements, len(self.rule), self.V)
        out = np.empty((self.mesh.n_elements, self.V * self.nB))
        rc = _library().oracle_project(ctypes.byref(self._cstruct()), _ptr(np.ascontiguousarray(vals)),
                                       _ptr(out))
        if rc:
            raise RuntimeError("oracle_project failed: %d" % rc)
        return out

    def time_derivative(self, u):
        u = np.ascontiguousarray(u, dtype=float)
        out = np.empty_like(u)
        rc = _library().oracle_time_derivative(ctypes.byref(self._cstruct()), _ptr(u), _ptr(out))
        if rc:
            raise RuntimeError("oracle_time_derivative failed: %d" % rc)
        return out

    def step(self, u, dt, nsteps, tableau="RK4_4", return_stages=False):
        """computeOneTimeStep ``nsteps`` times; returns the new solution."""
        tab = TABLEAUX[tableau]
        S = len(tab["b"])
        vec = np.zeros((S + 1,) + np.shape(u))
        vec[0] = u
        A = np.ascontiguousarray(np.asarray(tab["A"], dtype=float).reshape(S, S))
        b = np.ascontiguousarray(tab["b"], dtype=float)
        rc = _library().oracle_step(ctypes.byref(self._cstruct()), _ptr(vec), ctypes.c_int(S),
                                    _ptr(A), _ptr(b), ctypes.c_double(dt), ctypes.c_int(nsteps))
        if rc:
            raise RuntimeError("oracle_step failed: %d" % rc)
        return (vec[0].copy(), vec[1:].copy()) if return_stages else vec[0].copy()

    def error_and_norm(self, u, stages, dt, tableau):
        """computeErrorAndNormOfUpdate (HpgemAPISimplified_Impl.h:719-749): per element the
        deviation sum_i (k_i dt) err_i and its squared Euclidean norm, summed, square root;
        and the sum over elements of the Euclidean norms of u."""
        err = ERROR_COEFFICIENTS[tableau]
        nE = len(self.absdet)
        uu = np.asarray(u).reshape(nE, -1)
        error = 0.0
        norm = 0.0
        for e in range(nE):
            norm += math.sqrt(float(np.dot(uu[e], uu[e])))
            dev = np.zeros(uu.shape[1])
            for i in range(len(err)):
                dev += (np.asarray(stages[i]).reshape(nE, -1)[e] * dt) * err[i]
            error += float(np.dot(dev, dev))
        return math.sqrt(error), norm

    def step_adaptive(self, u, time, max_relative_error, dt_max, dt_estimate, tableau="DormandPrince"):
        """computeOneTimeStep(time, maximumRelativeError, dtMax) (HpgemAPISimplified_Impl.h:822-861):
        returns (u, time, next dt estimate, accepted dt, rejected tries)."""
        tab = TABLEAUX[tableau]
        order = tab["order"]
        dt = min(dt_estimate, dt_max)
        error, norm = math.inf, 0.0
        rejections = 0
        while max_relative_error * norm < error or math.isinf(error):
            u_new, stages = self.step(u, dt, 1, tableau, return_stages=True)
            error, norm = self.error_and_norm(u_new, stages, dt, tableau)
            if max_relative_error * norm < error or math.isinf(error):
                for j in range(len(tab["b"])):  # the reference rewinds by subtraction
                    u_new = u_new + (-dt * tab["b"][j]) * stages[j]
                u = u_new
                dt = 0.8 * dt * (max_relative_error / error * norm) ** (1.0 / order)
                rejections += 1
            else:
                u = u_new
        estimate = 0.9 * dt * (max_relative_error / error * norm) ** (1.0 / order)
        return u, time + dt, estimate, dt, rejections

    def l2_error(self, u, exact, t):
        """computeTotalError (HpgemAPISimplified_Impl.h:326-401): rule of order 2p+2."""
        rule = get_rule(self.shape, 2 * self.p + 2)
        phi, _ = tabulate(self.shape, self.p, rule.points)
        N = vertex_shape_functions(self.shape, rule.points)
        x = np.einsum("qk,ekr->eqr", N, self.mesh.element_coords)
        ex = np.asarray(exact(x.reshape(-1, self.dim), t)).reshape(len(x), len(rule), self.V)
        uq = np.einsum("qj,evj->eqv", phi, np.asarray(u).reshape(len(x), self.V, self.nB))
        err2 = ((ex - uq) ** 2).sum(axis=2)
        total = np.einsum("q,eq,e->", rule.weights, err2, self.absdet)
        return float(np.sqrt(abs(total)))
