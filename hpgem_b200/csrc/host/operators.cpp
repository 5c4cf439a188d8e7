// Reference-element operators and per-element geometry (see operators.h).
#include "operators.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>
#include <utility>

#include "refshapes.h"

namespace hgg {

void invert_matrix(int n, const double *A, double *Ainv) {
    // Gauss-Jordan with partial pivoting on [A | I]
    std::vector<double> M((size_t)n * 2 * n, 0.0);
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) M[i * 2 * n + j] = A[i * n + j];
        M[i * 2 * n + n + i] = 1.0;
    }
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(M[i * 2 * n + k]) > std::fabs(M[p * 2 * n + k])) p = i;
        if (M[p * 2 * n + k] == 0.0) throw std::runtime_error("singular reference mass matrix");
        if (p != k)
            for (int j = 0; j < 2 * n; ++j) std::swap(M[k * 2 * n + j], M[p * 2 * n + j]);
        double inv = 1.0 / M[k * 2 * n + k];
        for (int j = 0; j < 2 * n; ++j) M[k * 2 * n + j] *= inv;
        for (int i = 0; i < n; ++i) {
            if (i == k) continue;
            double l = M[i * 2 * n + k];
            if (l != 0.0)
                for (int j = 0; j < 2 * n; ++j) M[i * 2 * n + j] -= l * M[k * 2 * n + j];
        }
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) Ainv[i * n + j] = M[i * 2 * n + n + j];
}

namespace {

void matmul(int n, const double *A, const double *B, double *C) {
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int k = 0; k < n; ++k) s += A[i * n + k] * B[k * n + j];
            C[i * n + j] = s;
        }
}

double det(int d, const double *J) {
    if (d == 1) return J[0];
    if (d == 2) return J[0] * J[3] - J[1] * J[2];
    return J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
           J[2] * (J[3] * J[7] - J[4] * J[6]);
}

void inverse_small(int d, const double *J, double *Ji) { invert_matrix(d, J, Ji); }

// 1D hierarchical basis psi_0 = (1-x)/2, psi_1 = (1+x)/2, psi_{k+2} = (1-x^2) L_k(x) / 4
void psi1d(int np, double x, double *v, double *dv) {
    for (int a = 0; a < np; ++a) {
        Dual X = dconst(x);
        X.g[0] = 1.0;
        Dual r = a == 0 ? (1.0 - X) / 2. : (a == 1 ? (1.0 + X) / 2. : (1.0 - X) * (1.0 + X) * lobatto(a - 2, X) / 4.);
        v[a] = r.v;
        if (dv) dv[a] = r.g[0];
    }
}

// Tries to express the operators in sum-factorised form; fills the tensor fields
// of `op` and returns true when every check passes.
bool try_tensor(const hgg_problem_desc &desc, HostOperators &op) {
    const int d = op.dim, nB = op.nB, p = op.order, np = p + 1;
    if (!is_hypercube(op.shape) || op.dim < 2) { op.tensor_reason = "not a square or cube"; return false; }
    if (op.physics != HGG_PHYSICS_ADVECTION) { op.tensor_reason = "wave uses the dense form"; return false; }
    // The tensor form is derived from hpGEM's default H1 set; it is only taken
    // when the dense operators built from the caller's own tabulations agree
    // with it entry by entry (checked below), so a caller with another basis
    // simply keeps the dense form.
    std::vector<Dual> vals;
    int total = 1;
    for (int i = 0; i < d; ++i) total *= np;
    if (total != nB) { op.tensor_reason = "basis size"; return false; }
    // factorise each hpGEM basis function on a tensor grid of p+2 points per axis
    const int ng = p + 2;
    std::vector<double> gx(ng);
    for (int i = 0; i < ng; ++i) gx[i] = -0.9 + 1.8 * i / (ng - 1) + 0.013 * i;  // generic points
    int ngrid = 1;
    for (int i = 0; i < d; ++i) ngrid *= ng;
    std::vector<double> hv((size_t)ngrid * nB), pv((size_t)ng * np);
    for (int g = 0; g < ngrid; ++g) {
        double x[3] = {0, 0, 0};
        int r = g;
        for (int i = 0; i < d; ++i) { x[i] = gx[r % ng]; r /= ng; }
        eval_basis(op.shape, p, x, vals);
        for (int j = 0; j < nB; ++j) hv[(size_t)g * nB + j] = vals[j].v;
    }
    for (int i = 0; i < ng; ++i) psi1d(np, gx[i], &pv[i * np], nullptr);
    op.tpos.assign(nB, -1);
    op.tsign.assign(nB, 0.0);
    std::vector<int> used(nB, 0);
    for (int j = 0; j < nB; ++j) {
        for (int t = 0; t < nB && op.tpos[j] < 0; ++t) {
            int a[3] = {0, 0, 0}, r = t;
            for (int i = 0; i < d; ++i) { a[i] = r % np; r /= np; }
            for (double s : {1.0, -1.0}) {
                bool ok = true;
                for (int g = 0; g < ngrid && ok; ++g) {
                    int gi[3] = {0, 0, 0}, rr = g;
                    for (int i = 0; i < d; ++i) { gi[i] = rr % ng; rr /= ng; }
                    double prod = s;
                    for (int i = 0; i < d; ++i) prod *= pv[gi[i] * np + a[i]];
                    ok = std::fabs(prod - hv[(size_t)g * nB + j]) <= 1e-13 * (1.0 + std::fabs(prod));
                }
                if (ok && !used[t]) {
                    op.tpos[j] = t;
                    op.tsign[j] = s;
                    used[t] = 1;
                    break;
                }
            }
        }
        if (op.tpos[j] < 0) { op.tensor_reason = "basis is not a tensor product"; return false; }
    }
    // 1D operators with a Gauss rule of np points (exact for degree 2p)
    std::vector<double> M1(np * np, 0.0), S1(np * np, 0.0), M1i(np * np);
    {
        // Gauss-Legendre nodes via the same Newton construction as the element rules
        std::vector<double> x(np), w(np);
        const double pi = 3.14159265358979323846;
        for (int i = 0; i < np; ++i) {
            double z = std::cos(pi * (i + 0.75) / (np + 0.5)), dp = 1.0;
            for (int it = 0; it < 100; ++it) {
                double p0 = 1.0, p1 = z;
                for (int k = 2; k <= np; ++k) {
                    double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                    p0 = p1;
                    p1 = pk;
                }
                double pn = np == 1 ? z : p1, pm = np == 1 ? 1.0 : p0;
                dp = np * (z * pn - pm) / (z * z - 1.0);
                double dz = pn / dp;
                z -= dz;
                if (std::fabs(dz) < 1e-17 && it > 3) break;
            }
            x[i] = z;
            w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
        }
        std::vector<double> v(np), dv(np);
        for (int q = 0; q < np; ++q) {
            psi1d(np, x[q], v.data(), dv.data());
            for (int a = 0; a < np; ++a)
                for (int b = 0; b < np; ++b) {
                    M1[a * np + b] += w[q] * v[a] * v[b];
                    S1[a * np + b] += w[q] * dv[a] * v[b];
                }
        }
    }
    invert_matrix(np, M1.data(), M1i.data());
    op.np = np;
    op.D1.assign(np * np, 0.0);
    for (int a = 0; a < np; ++a)
        for (int b = 0; b < np; ++b)
            for (int k = 0; k < np; ++k) op.D1[a * np + b] += M1i[a * np + k] * S1[k * np + b];
    op.lift.assign(2 * np, 0.0);
    std::vector<double> pm(np), pp(np);
    psi1d(np, -1.0, pm.data(), nullptr);
    psi1d(np, 1.0, pp.data(), nullptr);
    for (int side = 0; side < 2; ++side) {
        const double *t = side ? pp.data() : pm.data();
        int pos = -1;
        for (int a = 0; a < np; ++a) {
            if (t[a] == 1.0 && pos < 0) pos = a;
            else if (t[a] != 0.0) { op.tensor_reason = "trace is not a single mode"; return false; }
        }
        op.trace_pos[side] = pos;
        for (int a = 0; a < np; ++a)
            for (int k = 0; k < np; ++k) op.lift[side * np + a] += M1i[a * np + k] * t[k];
    }
    // tensor form of a dense operator: entry (i, j) for hpGEM indices i, j
    auto unpack = [&](int t, int *a) { for (int i = 0; i < d; ++i) { a[i] = t % np; t /= np; } };
    // volume: vol[c] must equal I (x) .. D1 (axis c) .. (x) I.  The dense operators
    // carry the rounding of the reference mass-matrix inverse (condition number
    // grows quickly with p on hexahedra), so compare relative to the largest entry.
    double vmax = 1.0, pmax = 1.0;
    for (double v : op.vol) vmax = std::max(vmax, std::fabs(v));
    for (double v : op.pairs) pmax = std::max(pmax, std::fabs(v));
    const double tol_vol = 1e-9 * vmax, tol_pair = 1e-9 * pmax;
    for (int c = 0; c < d; ++c)
        for (int i = 0; i < nB; ++i)
            for (int j = 0; j < nB; ++j) {
                int ai[3], aj[3];
                unpack(op.tpos[i], ai);
                unpack(op.tpos[j], aj);
                double pred = op.D1[ai[c] * np + aj[c]];
                for (int k = 0; k < d; ++k)
                    if (k != c && ai[k] != aj[k]) pred = 0.0;
                pred *= op.tsign[i] * op.tsign[j];
                double have = op.vol[((size_t)c * nB + i) * nB + j];
                if (std::fabs(pred - have) > tol_vol) {
                    op.tensor_reason = "volume operator is not sum-factorisable";
                    return false;
                }
            }
    // faces: local face -> (axis, side); the operators of every element slot must be
    // lift(side) trace(side') (x) identity on the tangential axes, with the
    // neighbour's trace taken on the opposite side
    const ShapeInfo &si = shape_info(op.shape);
    std::vector<int> face_axis(si.n_faces), face_side(si.n_faces);
    for (int f = 0; f < si.n_faces; ++f) {
        int fvn = d == 1 ? 1 : si.face_vertices;
        face_axis[f] = -1;
        for (int c = 0; c < d; ++c) {
            double v0 = si.vertices[si.faces[f][0]][c];
            bool same = true;
            for (int k = 1; k < fvn; ++k) same &= si.vertices[si.faces[f][k]][c] == v0;
            if (same) { face_axis[f] = c; face_side[f] = v0 > 0 ? 1 : 0; }
        }
    }
    auto check_pair = [&](int pid, int axis, int side_test, int side_trial) {
        const double *P = &op.pairs[(size_t)pid * nB * nB];
        for (int i = 0; i < nB; ++i)
            for (int j = 0; j < nB; ++j) {
                int ai[3], aj[3];
                unpack(op.tpos[i], ai);
                unpack(op.tpos[j], aj);
                double pred = op.lift[side_test * np + ai[axis]] *
                              (aj[axis] == op.trace_pos[side_trial] ? 1.0 : 0.0);
                for (int k = 0; k < d; ++k)
                    if (k != axis && ai[k] != aj[k]) pred = 0.0;
                pred *= op.tsign[i] * op.tsign[j];
                double have = P[i * nB + j];
                if (std::fabs(pred - have) > tol_pair) return false;
            }
        return true;
    };
    std::map<std::pair<int, int>, bool> checked;
    auto check_cached = [&](int pid, int axis, int st, int sn) {
        auto key = std::make_pair(pid, axis * 4 + st * 2 + sn);
        auto it = checked.find(key);
        if (it != checked.end()) return it->second;
        bool ok = check_pair(pid, axis, st, sn);
        checked[key] = ok;
        return ok;
    };
    const int ns = 2 * d;
    op.t_nbr.assign((size_t)op.nE * ns, 0);
    op.t_mode.assign((size_t)op.nE * ns, MODE_NONE);
    op.t_sigma.assign((size_t)op.nE * ns, 0.0);
    for (int64_t e = 0; e < op.nE; ++e)
        for (int f = 0; f < op.nfl; ++f) {
            int axis = face_axis[f], side = face_side[f];
            if (axis < 0) { op.tensor_reason = "face not axis aligned"; return false; }
            size_t s = (size_t)e * op.nfl + f;
            if (!check_cached(op.self_pair[s], axis, side, side) ||
                !check_cached(op.nbr_pair[s], axis, side, 1 - side)) {
                op.tensor_reason = "neighbour orientation is not aligned";
                return false;
            }
            size_t ts = (size_t)e * ns + 2 * axis + side;
            op.t_nbr[ts] = op.nbr[s];
            op.t_mode[ts] = op.mode[s];
            op.t_sigma[ts] = op.face_geo[s];
        }
    return true;
}

}  // namespace

HostOperators build_operators(const hgg_problem_desc &desc, bool faces) {
    HostOperators op;
    const int d = desc.dim;
    if (d < 1 || d > 3) throw std::invalid_argument("dim must be 1, 2 or 3");
    if (desc.shape < HGG_SHAPE_LINE || desc.shape > HGG_SHAPE_TETRAHEDRON)
        throw std::invalid_argument("unknown shape");
    if (shape_info(desc.shape).dim != d) throw std::invalid_argument("shape does not match dim");
    if (desc.physics != HGG_PHYSICS_ADVECTION && desc.physics != HGG_PHYSICS_WAVE &&
        desc.physics != HGG_PHYSICS_WAVE_UPWIND)
        throw std::invalid_argument("unknown physics");
    const int V = desc.physics == HGG_PHYSICS_ADVECTION ? 1 : d + 1;
    if (desc.n_vars != V) throw std::invalid_argument("n_vars must be 1 (advection) or dim+1 (wave)");
    if (desc.n_elements <= 0 || desc.n_basis <= 0 || desc.n_quad <= 0 || desc.n_face_quad <= 0)
        throw std::invalid_argument("empty mesh or rule");
    if (desc.n_elements > (int64_t)1 << 31) throw std::invalid_argument("too many elements");
    if (!desc.quad_weights || !desc.basis_values || !desc.basis_grads || !desc.face_weights ||
        !desc.face_tabs || !desc.jacobians || !desc.face_elements || !desc.face_local ||
        !desc.face_tab_index || !desc.face_normals)
        throw std::invalid_argument("missing descriptor array");
    if (desc.physics != HGG_PHYSICS_ADVECTION && !(desc.c_inv > 0.0))
        throw std::invalid_argument("c_inv must be positive");
    op.shape = desc.shape;
    op.dim = d;
    op.order = desc.order;
    op.nB = desc.n_basis;
    op.V = V;
    op.physics = desc.physics;
    op.c_inv = desc.c_inv;
    op.nE = desc.n_elements;
    op.nfl = shape_info(desc.shape).n_faces;
    const int nB = op.nB, nQ = desc.n_quad, nQf = desc.n_face_quad;

    // reference mass matrix and its inverse
    std::vector<double> M((size_t)nB * nB, 0.0);
    for (int q = 0; q < nQ; ++q)
        for (int i = 0; i < nB; ++i)
            for (int j = 0; j < nB; ++j)
                M[i * nB + j] += desc.quad_weights[q] * desc.basis_values[q * nB + i] *
                                 desc.basis_values[q * nB + j];
    op.mass_inv.resize((size_t)nB * nB);
    invert_matrix(nB, M.data(), op.mass_inv.data());

    // volume operators
    op.vol.assign((size_t)d * nB * nB, 0.0);
    std::vector<double> K((size_t)nB * nB);
    for (int c = 0; c < d; ++c) {
        std::fill(K.begin(), K.end(), 0.0);
        for (int q = 0; q < nQ; ++q)
            for (int i = 0; i < nB; ++i)
                for (int j = 0; j < nB; ++j) {
                    double gi = desc.basis_grads[((size_t)q * nB + i) * d + c];
                    double gj = desc.basis_grads[((size_t)q * nB + j) * d + c];
                    double pi = desc.basis_values[q * nB + i], pj = desc.basis_values[q * nB + j];
                    K[i * nB + j] += desc.quad_weights[q] *
                                     (desc.physics == HGG_PHYSICS_ADVECTION ? gi * pj : pi * gj);
                }
        matmul(nB, op.mass_inv.data(), K.data(), &op.vol[(size_t)c * nB * nB]);
    }

    // element geometry
    op.abs_det.resize(op.nE);
    op.elem_geo.assign((size_t)op.nE * (desc.physics == HGG_PHYSICS_ADVECTION ? d : d * d), 0.0);
    for (int64_t e = 0; e < op.nE; ++e) {
        const double *J = desc.jacobians + e * d * d;
        double dt = det(d, J);
        if (!(std::fabs(dt) > 0.0)) throw std::invalid_argument("degenerate element");
        op.abs_det[e] = std::fabs(dt);
        double Ji[9];
        inverse_small(d, J, Ji);
        if (desc.physics == HGG_PHYSICS_ADVECTION) {
            for (int c = 0; c < d; ++c) {
                double s = 0.0;
                for (int r = 0; r < d; ++r) s += Ji[c * d + r] * desc.advection[r];
                op.elem_geo[e * d + c] = s;
            }
        } else {  // G[r][c] = (J^{-T})[r][c] = Ji[c][r]
            for (int r = 0; r < d; ++r)
                for (int c = 0; c < d; ++c) op.elem_geo[(e * d + r) * d + c] = Ji[c * d + r];
        }
    }

    if (!faces) {
        op.tensor = false;
        return op;
    }

    // face operators per (test tabulation, trial tabulation) pair
    std::map<std::pair<int, int>, int> pair_id;
    auto get_pair = [&](int s, int n) {
        auto key = std::make_pair(s, n);
        auto it = pair_id.find(key);
        if (it != pair_id.end()) return it->second;
        int id = (int)pair_id.size();
        pair_id.emplace(key, id);
        std::vector<double> E((size_t)nB * nB, 0.0);
        const double *ps = desc.face_tabs + (size_t)s * nQf * nB;
        const double *pn = desc.face_tabs + (size_t)n * nQf * nB;
        for (int q = 0; q < nQf; ++q)
            for (int i = 0; i < nB; ++i)
                for (int j = 0; j < nB; ++j) E[i * nB + j] += desc.face_weights[q] * ps[q * nB + i] * pn[q * nB + j];
        size_t off = op.pairs.size();
        op.pairs.resize(off + (size_t)nB * nB);
        matmul(nB, op.mass_inv.data(), E.data(), &op.pairs[off]);
        return id;
    };
    const size_t slots = (size_t)op.nE * op.nfl;
    op.nbr.assign(slots, -1);
    op.self_pair.assign(slots, 0);
    op.nbr_pair.assign(slots, 0);
    op.mode.assign(slots, MODE_NONE);
    op.face_geo.assign(slots * (desc.physics == HGG_PHYSICS_ADVECTION ? 1 : d), 0.0);
    for (int64_t f = 0; f < desc.n_faces; ++f) {
        int64_t L = desc.face_elements[2 * f], R = desc.face_elements[2 * f + 1];
        int fL = desc.face_local[2 * f], fR = desc.face_local[2 * f + 1];
        int tL = desc.face_tab_index[2 * f], tR = desc.face_tab_index[2 * f + 1];
        if (L < 0 || L >= op.nE || fL < 0 || fL >= op.nfl)
            throw std::invalid_argument("bad face table");
        if (R < 0) throw std::invalid_argument("boundary faces are not supported (periodic meshes only)");
        if (R >= op.nE || fR < 0 || fR >= op.nfl || tL < 0 || tR < 0 || tL >= desc.n_face_tabs ||
            tR >= desc.n_face_tabs)
            throw std::invalid_argument("bad face table");
        size_t sL = (size_t)L * op.nfl + fL, sR = (size_t)R * op.nfl + fR;
        if (op.nbr[sL] >= 0 || op.nbr[sR] >= 0) throw std::invalid_argument("element face used twice");
        op.nbr[sL] = (int32_t)R;
        op.nbr[sR] = (int32_t)L;
        op.self_pair[sL] = get_pair(tL, tL);
        op.nbr_pair[sL] = get_pair(tL, tR);
        op.self_pair[sR] = get_pair(tR, tR);
        op.nbr_pair[sR] = get_pair(tR, tL);
        const double *n = desc.face_normals + f * d;
        double nn = 0.0;
        for (int c = 0; c < d; ++c) nn += n[c] * n[c];
        double area = std::sqrt(nn);
        if (desc.physics == HGG_PHYSICS_ADVECTION) {
            // 090Advection_SelfTest.cpp:160-191, evaluated once with the left unit normal
            double A = 0.0;
            for (int c = 0; c < d; ++c) A += desc.advection[c] * (n[c] / area);
            int8_t mL = MODE_NONE, mR = MODE_NONE;
            if (A > 1e-12) { mL = MODE_SELF; mR = MODE_NBR; }
            else if (A < -1e-12) { mL = MODE_NBR; mR = MODE_SELF; }
            else if (std::fabs(A) < 1e-12) { mL = MODE_AVG; mR = MODE_AVG; }
            op.mode[sL] = mL;
            op.mode[sR] = mR;
            op.face_geo[sL] = A * area / op.abs_det[L];
            op.face_geo[sR] = -A * area / op.abs_det[R];
        } else {
            for (int c = 0; c < d; ++c) {
                op.face_geo[sL * d + c] = 0.5 * n[c] / op.abs_det[L];
                op.face_geo[sR * d + c] = -0.5 * n[c] / op.abs_det[R];
            }
        }
    }
    for (size_t s = 0; s < slots; ++s)
        if (op.nbr[s] < 0) throw std::invalid_argument("element face without a neighbour");
    op.n_pairs = (int)pair_id.size();
    op.tensor = try_tensor(desc, op);
    return op;
}

}  // namespace hgg
