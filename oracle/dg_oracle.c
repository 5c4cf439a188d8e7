/*
 * CPU oracle: hpGEM's explicit DG time step, restated in plain C.
 *
 * TEST INFRASTRUCTURE ONLY: built by oracle/build.py into oracle/_build/ and
 * called through ctypes by the tests, the smoke check and the CPU-baseline
 * leg of bench.py.  The hpgem_b200 library never links or calls it.
 *
 * It follows, loop for loop, what hpGEM does on the CPU for one mesh:
 *   computeOneTimeStep          kernel/Base/HpgemAPISimplified_Impl.h:788-820
 *   computeTimeDerivative       :777-786  (= computeRightHandSide + solveMassMatrixEquations)
 *   computeRightHandSide        :625-695  (element loop overwrites, then every internal
 *                                          face adds its LEFT and RIGHT integrals)
 *   getLinearCombinationOfVectors :599-620 (copy * coeff[0], then axpy per extra vector,
 *                                          recomputed for every element and both face sides)
 *   solveMassMatrixEquations    :205-225  (mass matrix rebuilt by quadrature, then solved by
 *                                          LU with partial pivoting, as LAPACK dgesv does via
 *                                          MiddleSizeMatrix::solve, kernel/LinearAlgebra/
 *                                          MiddleSizeMatrix.cpp:723-745)
 *   scaleAndAddVector           :707-717
 *   ElementIntegral::integrate  kernel/Integration/ElementIntegral_Impl.h:96-151
 *                               (first point assigns, later points axpy; scale |J| unless
 *                                the application switched Jacobian scaling off)
 *   FaceIntegral::integrate     kernel/Integration/FaceIntegral_Impl.h:68-127 (scale |n|)
 * Physics:
 *   ADVECTION (weak form, upwind)  tests/self/Basic/090Advection_SelfTest.cpp:92-220
 *   WAVE (strong form, central)    applications/ExampleMultipleVariableProblem/
 *                                  AcousticWave_Impl.h:102-129, 169-226, 289-373
 *                                  (Jacobian scaling off, AcousticWave.h:223-233)
 *   WAVE_UPWIND                    the same with the upwind (Riemann) flux, restated:
 *                                  the reference has the central flux only
 * Gradients are mapped as hpGEM's H1ConformingTransformation::transformDeriv
 * (kernel/Base/H1ConformingTransformation.h:64-69): solve J^T g = g_ref.
 * The textbook LU (Golub & Van Loan, Algorithm 3.4.1) stands in for dgesv;
 * it differs from an optimised LAPACK only by rounding.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { ORACLE_ADVECTION = 0, ORACLE_WAVE = 1, ORACLE_WAVE_UPWIND = 2 };

typedef struct {
    int dim, nB, nQ, nQf, V, nFL, physics;
    double a[3];
    double cinv;
    const double *wq, *phi, *dphi;  /* element rule [nQ], [nQ][nB], [nQ][nB][dim] */
    const double *wqf;              /* face rule [nQf] */
    const double *phiF;             /* left-side tabulation [nFL][nQf][nB] */
    const double *phiR;             /* right-side tabulation per combination [nC][nQf][nB] */
    long nE, nF;
    const double *jac;              /* [nE][dim][dim], J[r][c] = dx_r/dxi_c */
    const double *absdet;           /* [nE] */
    const long *faces;              /* [nF][4]: left, right, left local face, right combination */
    const double *normal;           /* [nF][dim]: outward from left, length = area ratio */
} oracle_problem;

/* solve A x = b in place for a small dense n x n system (A copied), partial pivoting */
static int small_solve(int n, const double *Ain, double *b) {
    double A[9];
    memcpy(A, Ain, sizeof(double) * n * n);
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (fabs(A[i * n + k]) > fabs(A[p * n + k])) p = i;
        if (A[p * n + k] == 0.0) return -1;
        if (p != k) {
            for (int j = 0; j < n; ++j) {
                double t = A[k * n + j]; A[k * n + j] = A[p * n + j]; A[p * n + j] = t;
            }
            double t = b[k]; b[k] = b[p]; b[p] = t;
        }
        for (int i = k + 1; i < n; ++i) {
            double l = A[i * n + k] / A[k * n + k];
            for (int j = k; j < n; ++j) A[i * n + j] -= l * A[k * n + j];
            b[i] -= l * b[k];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = b[i];
        for (int j = i + 1; j < n; ++j) s -= A[i * n + j] * b[j];
        b[i] = s / A[i * n + i];
    }
    return 0;
}

/* LU with partial pivoting (GvL 3.4.1) and the two triangular solves: dgesv semantics */
static int lu_solve(int n, double *A, double *b, int *piv) {
    for (int k = 0; k < n; ++k) {
        int p = k;
        double best = fabs(A[k * n + k]);
        for (int i = k + 1; i < n; ++i) {
            double v = fabs(A[i * n + k]);
            if (v > best) { best = v; p = i; }
        }
        piv[k] = p;
        if (A[p * n + k] == 0.0) return -1;
        if (p != k)
            for (int j = 0; j < n; ++j) {
                double t = A[k * n + j]; A[k * n + j] = A[p * n + j]; A[p * n + j] = t;
            }
        double inv = 1.0 / A[k * n + k];
        for (int i = k + 1; i < n; ++i) A[i * n + k] *= inv;
        for (int i = k + 1; i < n; ++i) {
            double l = A[i * n + k];
            if (l != 0.0)
                for (int j = k + 1; j < n; ++j) A[i * n + j] -= l * A[k * n + j];
        }
    }
    for (int k = 0; k < n; ++k)
        if (piv[k] != k) { double t = b[k]; b[k] = b[piv[k]]; b[piv[k]] = t; }
    for (int i = 0; i < n; ++i) {
        double s = b[i];
        for (int j = 0; j < i; ++j) s -= A[i * n + j] * b[j];
        b[i] = s;
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = b[i];
        for (int j = i + 1; j < n; ++j) s -= A[i * n + j] * b[j];
        b[i] = s / A[i * n + i];
    }
    return 0;
}

/* physical gradients of all basis functions at element quadrature point q */
static void phys_grads(const oracle_problem *P, long e, int q, double *g) {
    int d = P->dim;
    double JT[9];
    const double *J = P->jac + e * d * d;
    for (int r = 0; r < d; ++r)
        for (int c = 0; c < d; ++c) JT[r * d + c] = J[c * d + r];
    for (int j = 0; j < P->nB; ++j) {
        double *gj = g + j * d;
        for (int k = 0; k < d; ++k) gj[k] = P->dphi[((long)q * P->nB + j) * d + k];
        small_solve(d, JT, gj);
    }
}

static void accumulate(double *res, const double *val, int n, double scale, int first) {
    if (first)
        for (int i = 0; i < n; ++i) res[i] = val[i] * scale;
    else
        for (int i = 0; i < n; ++i) res[i] += scale * val[i];
}

/* computeRightHandSideAtElement: result overwritten */
static void element_rhs(const oracle_problem *P, long e, const double *w, double *res,
                        double *work) {
    int nB = P->nB, d = P->dim, V = P->V;
    double *g = work;                 /* nB*dim */
    double *integrand = work + nB * 3; /* V*nB */
    double absJ = P->absdet[e];
    for (int q = 0; q < P->nQ; ++q) {
        const double *ph = P->phi + (long)q * nB;
        phys_grads(P, e, q, g);
        if (P->physics == ORACLE_ADVECTION) {
            double u = 0.0;
            for (int j = 0; j < nB; ++j) u += w[j] * ph[j];
            for (int i = 0; i < nB; ++i) {
                double adg = 0.0;
                for (int k = 0; k < d; ++k) adg += P->a[k] * g[i * d + k];
                integrand[i] = u * adg;
            }
            accumulate(res, integrand, nB, P->wq[q] * absJ, q == 0);
        } else {
            double gs[3] = {0, 0, 0}, div = 0.0;
            for (int j = 0; j < nB; ++j)
                for (int k = 0; k < d; ++k) {
                    gs[k] += g[j * d + k] * w[0 * nB + j];
                    div += g[j * d + k] * w[(k + 1) * nB + j];
                }
            for (int i = 0; i < nB; ++i) {
                integrand[0 * nB + i] = ph[i] * div;
                for (int k = 0; k < d; ++k) integrand[(k + 1) * nB + i] = ph[i] * gs[k];
            }
            for (int i = 0; i < V * nB; ++i) integrand[i] *= absJ;
            accumulate(res, integrand, V * nB, P->wq[q], q == 0);
        }
    }
}

/* computeRightHandSideAtFace(face, side, left, right): returns the side's integral */
static void face_rhs(const oracle_problem *P, long f, int side, const double *wL,
                     const double *wR, double *res, double *work) {
    int nB = P->nB, d = P->dim, V = P->V;
    const long *fr = P->faces + f * 4;
    const double *n = P->normal + f * d;
    double nn = 0.0;
    for (int k = 0; k < d; ++k) nn += n[k] * n[k];
    double area = sqrt(nn);
    double *integrand = work;
    for (int q = 0; q < P->nQf; ++q) {
        const double *pl = P->phiF + ((long)fr[2] * P->nQf + q) * nB;
        const double *pr = P->phiR + ((long)fr[3] * P->nQf + q) * nB;
        const double *ps = side == 0 ? pl : pr;
        if (P->physics == ORACLE_ADVECTION) {
            double A = 0.0;
            for (int k = 0; k < d; ++k) A += P->a[k] * (n[k] / area);
            int sign = side == 0 ? 1 : -1;
            double jump = 0.0;
            if (A > 1e-12) {
                for (int j = 0; j < nB; ++j) jump += wL[j] * pl[j];
                jump *= A * sign;
            } else if (A < -1e-12) {
                for (int j = 0; j < nB; ++j) jump += wR[j] * pr[j];
                jump *= A * sign;
            } else if (fabs(A) < 1e-12) {
                for (int j = 0; j < nB; ++j) jump += wL[j] * pl[j];
                for (int j = 0; j < nB; ++j) jump += wR[j] * pr[j];
                jump *= A * sign / 2;
            }
            for (int i = 0; i < nB; ++i) integrand[i] = -jump * ps[i];
            accumulate(res, integrand, nB, P->wqf[q] * area, q == 0);
        } else {
            double uL[4], uR[4];
            for (int v = 0; v < V; ++v) {
                uL[v] = 0.0; uR[v] = 0.0;
                for (int j = 0; j < nB; ++j) uL[v] += pl[j] * wL[v * nB + j];
                for (int j = 0; j < nB; ++j) uR[v] += pr[j] * wR[v * nB + j];
            }
            double js[3], jv = 0.0;
            for (int k = 0; k < d; ++k) {
                js[k] = n[k] * (uL[0] - uR[0]);
                jv += n[k] * (uL[k + 1] - uR[k + 1]);
            }
            /* upwind flux (ORACLE_WAVE_UPWIND): the central terms plus (1/2) |A_n| [[U]],
             * c |n| [[v]] / 2 and c cinv n (n . [[s]]) / (2 |n|), c = 1 / sqrt(cinv), with the
             * jump of this side minus the other (the sign flips on the right side) */
            double upv = 0.0, ups[3] = {0.0, 0.0, 0.0};
            if (P->physics == ORACLE_WAVE_UPWIND) {
                double c = 1.0 / sqrt(P->cinv), sg = side == 0 ? 1.0 : -1.0;
                upv = 0.5 * c * area * (uL[0] - uR[0]) * sg;
                for (int k = 0; k < d; ++k) ups[k] = 0.5 * c * P->cinv * (n[k] / area) * jv * sg;
            }
            for (int i = 0; i < nB; ++i) {
                integrand[0 * nB + i] = -0.5 * ps[i] * jv - ps[i] * upv;
                for (int k = 0; k < d; ++k) integrand[(k + 1) * nB + i] = -0.5 * ps[i] * js[k] - ps[i] * ups[k];
            }
            accumulate(res, integrand, V * nB, P->wqf[q], q == 0);
        }
    }
}

/* solveMassMatrixEquationsAtElement: M rebuilt by quadrature, then LU solve */
static int mass_solve(const oracle_problem *P, long e, double *x, double *M, int *piv) {
    int nB = P->nB, V = P->V, N = V * nB;
    double absJ = P->absdet[e];
    for (int q = 0; q < P->nQ; ++q) {
        const double *ph = P->phi + (long)q * nB;
        double s = P->wq[q] * absJ;
        for (int iv = 0; iv < V; ++iv) {
            double c = (P->physics != ORACLE_ADVECTION && iv > 0) ? P->cinv : 1.0;
            for (int ib = 0; ib < nB; ++ib)
                for (int jb = 0; jb < nB; ++jb) {
                    double val = ph[ib] * ph[jb] * c;
                    long idx = (long)(iv * nB + ib) * N + iv * nB + jb;
                    if (q == 0) M[idx] = val * s; else M[idx] += s * val;
                }
        }
        if (q == 0)  /* zero the off-diagonal variable blocks (integrand entries are 0) */
            for (int iv = 0; iv < V; ++iv)
                for (int jv = 0; jv < V; ++jv)
                    if (iv != jv)
                        for (int ib = 0; ib < nB; ++ib)
                            for (int jb = 0; jb < nB; ++jb)
                                M[(long)(iv * nB + ib) * N + jv * nB + jb] = 0.0;
    }
    return lu_solve(N, M, x, piv);
}

typedef struct {
    double *w, *wL, *wR, *tmp, *work, *M;
    int *piv;
} scratch;

static int scratch_alloc(const oracle_problem *P, scratch *s) {
    int N = P->V * P->nB;
    s->w = malloc(sizeof(double) * N);
    s->wL = malloc(sizeof(double) * N);
    s->wR = malloc(sizeof(double) * N);
    s->tmp = malloc(sizeof(double) * N);
    s->work = malloc(sizeof(double) * (N + 3 * P->nB + 16));
    s->M = malloc(sizeof(double) * N * N);
    s->piv = malloc(sizeof(int) * N);
    return (s->w && s->wL && s->wR && s->tmp && s->work && s->M && s->piv) ? 0 : -1;
}

static void scratch_free(scratch *s) {
    free(s->w); free(s->wL); free(s->wR); free(s->tmp); free(s->work); free(s->M); free(s->piv);
}

static void lincomb(long e, int N, double *const *vec, const int *ids, const double *coef,
                    int n, double *out) {
    const double *v0 = vec[ids[0]] + e * N;
    for (int i = 0; i < N; ++i) out[i] = v0[i] * coef[0];
    for (int k = 1; k < n; ++k) {
        const double *vk = vec[ids[k]] + e * N;
        for (int i = 0; i < N; ++i) out[i] += coef[k] * vk[i];
    }
}

/* computeTimeDerivative(inputVectorIds, coefficients, resultVectorId) */
static int time_derivative(const oracle_problem *P, double *const *vec, const int *ids,
                           const double *coef, int n, int out, scratch *s) {
    int N = P->V * P->nB;
    for (long e = 0; e < P->nE; ++e) {
        lincomb(e, N, vec, ids, coef, n, s->w);
        element_rhs(P, e, s->w, vec[out] + e * N, s->work);
    }
    for (long f = 0; f < P->nF; ++f) {
        const long *fr = P->faces + f * 4;
        if (fr[1] < 0) return -2;  /* boundary faces are outside this restatement */
        lincomb(fr[0], N, vec, ids, coef, n, s->wL);
        lincomb(fr[1], N, vec, ids, coef, n, s->wR);
        face_rhs(P, f, 0, s->wL, s->wR, s->tmp, s->work);
        double *rl = vec[out] + fr[0] * N;
        for (int i = 0; i < N; ++i) rl[i] += s->tmp[i];
        face_rhs(P, f, 1, s->wL, s->wR, s->tmp, s->work);
        double *rr = vec[out] + fr[1] * N;
        for (int i = 0; i < N; ++i) rr[i] += s->tmp[i];
    }
    for (long e = 0; e < P->nE; ++e)
        if (mass_solve(P, e, vec[out] + e * N, s->M, s->piv)) return -3;
    return 0;
}

/* vectors: [nVec][nE][V*nB]; vector 0 = solution, 1..S = stage derivatives */
int oracle_step(const oracle_problem *P, double *vectors, int S, const double *A,
                const double *b, double dt, int nsteps) {
    int N = P->V * P->nB;
    double *vec[32];
    if (S + 1 > 32) return -1;
    for (int i = 0; i <= S; ++i) vec[i] = vectors + (long)i * P->nE * N;
    scratch s;
    if (scratch_alloc(P, &s)) return -4;
    int ids[32];
    double coef[32];
    int rc = 0;
    for (int step = 0; step < nsteps && rc == 0; ++step) {
        for (int i = 0; i < S && rc == 0; ++i) {
            ids[0] = 0;
            coef[0] = 1.0;
            for (int j = 0; j < i; ++j) {
                ids[j + 1] = 1 + j;
                coef[j + 1] = dt * A[i * S + j];
            }
            rc = time_derivative(P, vec, ids, coef, i + 1, 1 + i, &s);
        }
        for (int j = 0; j < S && rc == 0; ++j) {
            double sc = dt * b[j];
            for (long e = 0; e < P->nE; ++e) {
                double *u = vec[0] + e * N;
                const double *k = vec[1 + j] + e * N;
                for (int i = 0; i < N; ++i) u[i] += sc * k[i];
            }
        }
    }
    scratch_free(&s);
    return rc;
}

/* computeTimeDerivative(inputVectorId, resultVectorId): out = M^-1 R(in) */
int oracle_time_derivative(const oracle_problem *P, double *in, double *out) {
    double *vec[2] = {in, out};
    int ids[1] = {0};
    double coef[1] = {1.0};
    scratch s;
    if (scratch_alloc(P, &s)) return -4;
    int rc = time_derivative(P, vec, ids, coef, 1, 1, &s);
    scratch_free(&s);
    return rc;
}

/* setInitialSolution (HpgemAPISimplified_Impl.h:751-758 with :239-291):
 * values: the initial solution at every element quadrature point [nE][nQ][V] */
int oracle_project(const oracle_problem *P, const double *values, double *out) {
    int nB = P->nB, V = P->V, N = V * nB;
    scratch s;
    if (scratch_alloc(P, &s)) return -4;
    for (long e = 0; e < P->nE; ++e) {
        double *r = out + e * N;
        double absJ = P->absdet[e];
        for (int q = 0; q < P->nQ; ++q) {
            const double *ph = P->phi + (long)q * nB;
            const double *u0 = values + (e * P->nQ + q) * V;
            for (int v = 0; v < V; ++v)
                for (int i = 0; i < nB; ++i) {
                    double c = (P->physics != ORACLE_ADVECTION && v > 0) ? P->cinv : 1.0;
                    double val = ph[i] * u0[v] * c;
                    if (P->physics != ORACLE_ADVECTION) val *= absJ;
                    s.tmp[v * nB + i] = val;
                }
            accumulate(r, s.tmp, N, P->wq[q] * (P->physics != ORACLE_ADVECTION ? 1.0 : absJ), q == 0);
        }
        if (mass_solve(P, e, r, s.M, s.piv)) { scratch_free(&s); return -3; }
    }
    scratch_free(&s);
    return 0;
}
