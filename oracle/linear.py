"""Oracle for HpgemAPILinear's stored-matrix time stepping (test infrastructure only).

Restates kernel/Base/HpgemAPILinear_Impl.h:
* createMassMatrices (:131-139) and createStiffnessMatrices (:250-288): per
  element a mass and a stiffness matrix, per face the four blocks
  (LEFT,LEFT), (LEFT,RIGHT), (RIGHT,LEFT), (RIGHT,RIGHT) of the face matrix;
  ``assemble`` builds them in numpy from an oracle ``Problem`` with the
  integrands of the reference's two linear applications:
  - advection, tests/self/Basic/080AdvectionLinear_SelfTest.cpp:108-168
    (element: phi_i (a . grad phi_j) in row j, column i; face: the upwind
    side's trial functions, -(a . n_j) phi_j phi_i with n_j the unit normal
    out of the test function's side, halved for flow parallel to the face,
    integrated with the face weight times |n|);
  - wave, applications/ExampleMultipleVariableProblem/AcousticWaveLinear_Impl.h:
    98-284 (mass c_inv on the s variables; element grad_d phi_j phi_i in the
    (p, s_d) and (s_d, p) blocks; face -0.5 n_d phi_j phi_i with the scaled
    normal out of the basis function's side, no |n| factor);
* multiplyStiffnessMatrices (:360-434) + solveMassMatrixEquations (:143-156):
  ``time_derivative`` multiplies the element matrix, then adds both sides of
  every face, then solves with the element's mass matrix;
* the Runge-Kutta loop of HpgemAPISimplified::computeOneTimeStep
  (HpgemAPISimplified_Impl.h:788-820), which HpgemAPILinear inherits, with the
  stage time t + c_i dt handed to the right-hand side;
* the source terms of computeRightHandSide (:471-506): after the multiply,
  addSourceTerm (:437-450) adds per element the integral of phi_i g_v(x, t)
  (computeIntegrandSourceTermAtElement, :201-229, ElementIntegral: weights
  times |J|) and addSourceTermAtBoundary (:452-469) adds, for every boundary
  face to its left element, the integral of phi_i g_v(x, n, t) (the face
  integrand of the application, FaceIntegral: weights times |n|), both before
  the mass solve.  ``source_lifts`` restates the integration weights, and
  g is the application's function: for 080AdvectionLinear_SelfTest.cpp:72-88
  g = -u_exact(x, t) (a . n) on inflow faces (a . n < 0), 0 elsewhere.
"""
import numpy as np

from .dg import ADVECTION, TABLEAUX, WAVE, face_map_to_element
from .refgeom import SHAPES, vertex_shape_functions


def assemble(prob):
    """(mass [E][R][R], stiffness [E][R][R], face_elements [F][2], faces [F][4][R][R])."""
    if prob.physics not in (ADVECTION, WAVE):
        raise ValueError("the reference's linear applications are advection and the central-flux wave")
    d, nB, E = prob.dim, prob.nB, prob.mesh.n_elements
    wave = prob.physics == WAVE
    V = d + 1 if wave else 1
    R = V * nB
    w = np.asarray(prob.rule.weights, dtype=float)
    phi = prob.phi                                   # [nQ][nB]
    Jinv = np.linalg.inv(prob.J)                     # [E][d][d]
    grad = np.einsum("ecr,qbc->eqbr", Jinv, prob.dphi)  # J^{-T} grad_ref: [E][nQ][nB][d]
    wq = w[None, :] * prob.absdet[:, None]           # [E][nQ]
    mass1 = np.einsum("eq,qi,qj->eij", wq, phi, phi)
    mass = np.zeros((E, R, R))
    K = np.zeros((E, R, R))
    a = prob.a[:d]
    if not wave:
        mass[:] = mass1
        ag = np.einsum("eqjr,r->eqj", grad, a)
        K[:] = np.einsum("eq,qi,eqj->eji", wq, phi, ag)
    else:
        for v in range(V):
            mass[:, v * nB:(v + 1) * nB, v * nB:(v + 1) * nB] = mass1 * (prob.cinv if v > 0 else 1.0)
        for c in range(d):
            blk = np.einsum("eq,eqj,qi->eij", wq, grad[..., c], phi)  # [E][test i][basis j]
            K[:, 0:nB, (c + 1) * nB:(c + 2) * nB] = blk
            K[:, (c + 1) * nB:(c + 2) * nB, 0:nB] = blk
    table = prob.faces_c
    F = len(table)
    faces = np.zeros((F, 4, R, R))
    wf = np.asarray(prob.face_rule.weights, dtype=float)
    for f in range(F):
        L, Rt, fL, combo = (int(x) for x in table[f])
        ph = (prob.phiF[fL], prob.phiR[combo])      # [nQf][nB] per side
        n = prob.normals[f]
        area = float(np.sqrt(np.dot(n, n)))
        for ts in range(2):
            for tr in range(2):
                pp = np.einsum("q,qa,qb->ab", wf, ph[ts], ph[tr])  # [test function][trial function]
                blk = faces[f, 2 * ts + tr]
                if not wave:
                    A = float(np.dot(a, n / area))
                    if A > 1e-12:
                        factor = 1.0 if tr == 0 else 0.0
                    elif A < -1e-12:
                        factor = 1.0 if tr == 1 else 0.0
                    else:
                        factor = 0.5
                    an = A if ts == 0 else -A
                    blk[:] = -an * area * factor * pp
                elif Rt < 0:
                    # boundary face (AcousticWaveLinear_Impl.h:254-258, 271-272): -n_d in
                    # the (p, s_d) block, nothing in (s_d, p); only (LEFT, LEFT) is used
                    for c in range(d):
                        blk[0:nB, (c + 1) * nB:(c + 2) * nB] = -n[c] * pp
                else:
                    sgn = -1.0 if tr == 1 else 1.0
                    for c in range(d):
                        t = -0.5 * sgn * n[c] * pp
                        blk[0:nB, (c + 1) * nB:(c + 2) * nB] = t
                        blk[(c + 1) * nB:(c + 2) * nB, 0:nB] = t
    return mass, K, table[:, :2].astype(np.int64), faces


def source_lifts(prob):
    """Integration data of the two source terms of one mesh.

    Returns a dict with, for the element source: ``elem_x`` [E][nQ][dim] (the
    element rule's points) and ``elem_w`` [E][nQ][nB] (w_q |J_e| phi_i(q)); for
    the boundary source: ``bface`` (boundary face ids), ``bleft`` (their left
    elements), ``bface_x`` [Fb][nQf][dim], ``bface_n`` [Fb][dim] (unit normals)
    and ``bface_w`` [Fb][nQf][nB] (w_q |n_f| phi_i(q) on the left side)."""
    shape, d = prob.shape, prob.dim
    coords = prob.mesh.element_coords
    N = vertex_shape_functions(shape, prob.rule.points)
    elem_x = np.einsum("qk,ekr->eqr", N, coords)
    elem_w = np.einsum("q,e,qi->eqi", np.asarray(prob.rule.weights, dtype=float), prob.absdet, prob.phi)
    table = prob.faces_c
    bface = np.nonzero(table[:, 1] < 0)[0]
    fl = SHAPES[shape]["faces"]
    wf = np.asarray(prob.face_rule.weights, dtype=float)
    bx, bn, bw = [], [], []
    for f in bface:
        L, fL = int(table[f, 0]), int(table[f, 2])
        xi = face_map_to_element(shape, fl[fL], prob.face_rule.points)
        bx.append(vertex_shape_functions(shape, xi) @ coords[L])
        n = prob.normals[f]
        area = float(np.sqrt(np.dot(n, n)))
        bn.append(n / area)
        bw.append(wf[:, None] * area * prob.phiF[fL])
    z = np.zeros((0, len(wf), d))
    return {"elem_x": elem_x, "elem_w": elem_w, "bface": bface, "bleft": table[bface, 0].astype(np.int64),
            "bface_x": np.array(bx) if bx else z, "bface_n": np.array(bn).reshape(-1, d),
            "bface_w": np.array(bw) if bw else np.zeros((0, len(wf), prob.nB))}


class LinearOracle:
    """Stored matrices of one mesh; faces with right element -1 are boundary faces
    (only their (LEFT, LEFT) block is used, HpgemAPILinear_Impl.h:410-430)."""

    def __init__(self, mass, stiffness, face_elements, faces):
        self.mass = np.asarray(mass, dtype=float)
        self.K = np.asarray(stiffness, dtype=float)
        self.fe = np.asarray(face_elements, dtype=np.int64).reshape(-1, 2)
        self.faces = np.asarray(faces, dtype=float)
        self.E, self.R = self.mass.shape[0], self.mass.shape[1]
        self.lifts = None
        self.element_source = None   # g(x [n][dim], t) -> [n][V]   (useSourceTerm)
        self.boundary_source = None  # g(x [n][dim], unit normal [n][dim], t) -> [n][V]  (useSourceTermAtBoundary)

    def set_sources(self, prob, element_source=None, boundary_source=None):
        """HpgemAPILinear's useSourceTerm / useSourceTermAtBoundary with the integrand
        phi_i g_v; ``prob`` is the oracle Problem the matrices were assembled from."""
        self.lifts = source_lifts(prob)
        self.element_source, self.boundary_source = element_source, boundary_source
        return self

    def _add_sources(self, r, t):
        lf = self.lifts
        if self.element_source is not None:  # addSourceTerm: every element
            x = lf["elem_x"]
            g = np.asarray(self.element_source(x.reshape(-1, x.shape[2]), t), dtype=float)
            g = g.reshape(x.shape[0], x.shape[1], -1)
            r += np.einsum("eqi,eqv->evi", lf["elem_w"], g).reshape(r.shape)
        if self.boundary_source is not None and len(lf["bface"]):  # addSourceTermAtBoundary
            x = lf["bface_x"]
            n = np.repeat(lf["bface_n"][:, None, :], x.shape[1], axis=1)
            g = np.asarray(self.boundary_source(x.reshape(-1, x.shape[2]), n.reshape(-1, x.shape[2]), t),
                           dtype=float).reshape(x.shape[0], x.shape[1], -1)
            add = np.einsum("fqi,fqv->fvi", lf["bface_w"], g).reshape(len(lf["bface"]), -1)
            for f in range(len(lf["bface"])):  # face by face, as the reference adds them
                r[lf["bleft"][f]] += add[f]

    def time_derivative(self, u, t=0.0):
        u = np.asarray(u, dtype=float).reshape(self.E, self.R)
        r = np.einsum("eij,ej->ei", self.K, u)
        # both sides of every face (the reference adds them face by face; the sums
        # here differ from that order by rounding only)
        L, Rt = self.fe[:, 0], self.fe[:, 1]
        inner = Rt >= 0
        uR = u[np.where(inner, Rt, 0)]
        left = np.einsum("fij,fj->fi", self.faces[:, 0], u[L])
        left[inner] += np.einsum("fij,fj->fi", self.faces[inner, 1], uR[inner])
        np.add.at(r, L, left)
        right = (np.einsum("fij,fj->fi", self.faces[inner, 2], u[L[inner]]) +
                 np.einsum("fij,fj->fi", self.faces[inner, 3], uR[inner]))
        np.add.at(r, Rt[inner], right)
        if self.lifts is not None:
            self._add_sources(r, t)
        k = np.linalg.solve(self.mass, r[..., None])[..., 0]   # LU with partial pivoting per element
        return k.reshape(-1)

    def step(self, u, dt, nsteps, tableau="RK4_4", t0=0.0):
        tab = TABLEAUX[tableau]
        A, b = np.asarray(tab["A"], dtype=float), np.asarray(tab["b"], dtype=float)
        c = np.asarray(tab["c"], dtype=float)
        S = len(b)
        u = np.asarray(u, dtype=float).reshape(-1).copy()
        t = t0
        for _ in range(nsteps):
            ks = []
            for i in range(S):
                w = u.copy()
                for j in range(i):
                    if A[i][j] != 0.0:
                        w += dt * A[i][j] * ks[j]
                ks.append(self.time_derivative(w, t + c[i] * dt))
            for j in range(S):
                if b[j] != 0.0:
                    u += dt * b[j] * ks[j]
            t += dt
        return u
