// HpgemAPILinear's stored matrices (kernel/Base/HpgemAPILinear_Impl.h) and
// their folded device form; see linear.h.
#include "linear.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <map>
#include <utility>
#include <stdexcept>
#include <string>
#include <thread>

#include "operators.h"

namespace hgg {

namespace {

uint64_t fnv1a(const double *m, size_t n) {
    const unsigned char *p = reinterpret_cast<const unsigned char *>(m);
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < n * sizeof(double); ++i) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

// determinant of a small (d <= 3) matrix
double small_det(int d, const double *J) {
    if (d == 1) return J[0];
    if (d == 2) return J[0] * J[3] - J[1] * J[2];
    return J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
           J[2] * (J[3] * J[7] - J[4] * J[6]);
}

// runs f(i) for i in [0, n) on the host's cores; rethrows the first exception
template <typename F>
void parallel_for(int64_t n, F &&f) {
    const int64_t hw = std::max(1u, std::thread::hardware_concurrency());
    const int64_t nt = std::min<int64_t>(hw, n);
    if (nt <= 1) {
        for (int64_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::vector<std::exception_ptr> errors(nt);
    std::vector<std::thread> pool;
    for (int64_t t = 0; t < nt; ++t)
        pool.emplace_back([&, t] {
            try {
                for (int64_t i = t; i < n; i += nt) f(i);
            } catch (...) {
                errors[t] = std::current_exception();
            }
        });
    for (auto &th : pool) th.join();
    for (auto &e : errors)
        if (e) std::rethrow_exception(e);
}

// Key of a small geometry record (a Jacobian, a normal): every value rounded to
// 2^-40 of the record's largest magnitude, so that records which differ only by
// the rounding of the mesh coordinates (cells of width 1/6, say, whose
// Jacobians carry entries of 1e-17 where a zero belongs) share their matrices;
// the matrices of such records differ by ~1e-16 relative.
std::string geometry_key(const double *v, int n, const int32_t *ints = nullptr, int ni = 0) {
    std::string key;
    for (int i = 0; i < ni; ++i) key.append(reinterpret_cast<const char *>(&ints[i]), sizeof(int32_t));
    double big = 0.0;
    for (int i = 0; i < n; ++i) big = std::max(big, std::fabs(v[i]));
    int e = 0;
    std::frexp(big, &e);
    key.append(reinterpret_cast<const char *>(&e), sizeof(e));
    for (int i = 0; i < n; ++i) {
        const int64_t q = big == 0.0 ? 0 : (int64_t)std::nearbyint(std::ldexp(v[i], 40 - e));
        key.append(reinterpret_cast<const char *>(&q), sizeof(q));
    }
    return key;
}

}  // namespace

int MatrixPool::add(const double *m) {
    const size_t n = (size_t)R_ * R_;
    const uint64_t h = fnv1a(m, n);
    auto range = index_.equal_range(h);
    for (auto it = range.first; it != range.second; ++it)
        if (std::memcmp(get(it->second), m, n * sizeof(double)) == 0) return it->second;
    const int id = size();
    data_.insert(data_.end(), m, m + n);
    index_.emplace(h, id);
    return id;
}

LinearSystem linear_from_desc(const hgg_linear_desc &d) {
    if (d.n_rows < 1 || d.n_rows > 256) throw std::invalid_argument("n_rows must be 1..256");
    if (d.n_elements < 1 || d.n_faces < 0) throw std::invalid_argument("need at least one element");
    if (d.n_elements > INT32_MAX) throw std::invalid_argument("too many elements");
    if (!d.mass || !d.element_stiffness || (d.n_faces > 0 && (!d.face_elements || !d.face_stiffness)))
        throw std::invalid_argument("null matrix array");
    LinearSystem s;
    const int R = d.n_rows;
    const size_t RR = (size_t)R * R;
    s.R = R;
    s.E = d.n_elements;
    s.F = d.n_faces;
    s.pool = MatrixPool(R);
    s.mass_id.resize(s.E);
    s.stiffness_id.resize(s.E);
    for (int64_t e = 0; e < s.E; ++e) {
        s.mass_id[e] = s.pool.add(d.mass + e * RR);
        s.stiffness_id[e] = s.pool.add(d.element_stiffness + e * RR);
    }
    s.face_elements.assign(d.face_elements, d.face_elements + 2 * s.F);
    s.face_id.assign(4 * s.F, -1);
    for (int64_t f = 0; f < s.F; ++f) {
        const int64_t L = s.face_elements[2 * f], Rt = s.face_elements[2 * f + 1];
        if (L < 0 || L >= s.E || Rt < -1 || Rt >= s.E) throw std::invalid_argument("bad face table");
        for (int b = 0; b < (Rt >= 0 ? 4 : 1); ++b)
            s.face_id[4 * f + b] = s.pool.add(d.face_stiffness + (4 * f + b) * RR);
    }
    return s;
}

LinearSystem assemble_linear(const hgg_problem_desc &desc) {
    const bool upwind = desc.physics == HGG_PHYSICS_WAVE_UPWIND;
    const bool wave = desc.physics == HGG_PHYSICS_WAVE || upwind;
    if (desc.physics != HGG_PHYSICS_ADVECTION && !wave)
        throw std::invalid_argument("the stored-matrix form has advection and the wave");
    // the upwind wave's extra face terms (1/2) |A_n| [[U]]: c |n| [[v]] / 2 and
    // c c_inv n (n . [[s]]) / (2 |n|), c = 1 / sqrt(c_inv) (the matrix-free kernels' flux)
    const double c_wave = upwind ? 1.0 / std::sqrt(desc.c_inv) : 0.0;
    const int d = desc.dim, nB = desc.n_basis, nQ = desc.n_quad, nQf = desc.n_face_quad;
    const int V = wave ? d + 1 : 1, R = V * nB;
    if (R > 256) throw std::invalid_argument("the stored-matrix form takes at most 256 rows per element");
    LinearSystem s;
    s.R = R;
    s.E = desc.n_elements;
    s.F = desc.n_faces;
    s.pool = MatrixPool(R);
    s.mass_id.resize(s.E);
    s.stiffness_id.resize(s.E);
    const size_t RR = (size_t)R * R;
    std::vector<double> M(RR), K(RR), grad((size_t)nQ * nB * d), Jinv(9);
    const double *a = desc.advection;
    // the matrices depend on the element only through its Jacobian (affine
    // elements): elements with the same Jacobian (geometry_key) share them
    std::map<std::string, std::pair<int32_t, int32_t>> by_jacobian;
    for (int64_t e = 0; e < s.E; ++e) {
        const double *J = desc.jacobians + e * d * d;
        const std::string jkey = geometry_key(J, d * d);
        auto known = by_jacobian.find(jkey);
        if (known != by_jacobian.end()) {
            s.mass_id[e] = known->second.first;
            s.stiffness_id[e] = known->second.second;
            continue;
        }
        const double absdet = std::fabs(small_det(d, J));
        invert_matrix(d, J, Jinv.data());
        // physical gradients J^{-T} grad_ref (H1ConformingTransformation::transformDeriv)
        for (int q = 0; q < nQ; ++q)
            for (int b = 0; b < nB; ++b)
                for (int r = 0; r < d; ++r) {
                    double g = 0.0;
                    for (int c = 0; c < d; ++c) g += Jinv[c * d + r] * desc.basis_grads[((size_t)q * nB + b) * d + c];
                    grad[((size_t)q * nB + b) * d + r] = g;
                }
        std::fill(M.begin(), M.end(), 0.0);
        std::fill(K.begin(), K.end(), 0.0);
        for (int q = 0; q < nQ; ++q) {
            const double wq = desc.quad_weights[q] * absdet;
            const double *phi = desc.basis_values + (size_t)q * nB;
            const double *gq = grad.data() + (size_t)q * nB * d;
            for (int v = 0; v < V; ++v) {
                // mass: 080 (default hpGEM mass), AcousticWaveLinear_Impl.h:104-129 (c_inv on s)
                const double sv = (wave && v > 0) ? desc.c_inv : 1.0;
                for (int i = 0; i < nB; ++i)
                    for (int j = 0; j < nB; ++j) M[(size_t)(v * nB + i) * R + v * nB + j] += wq * sv * phi[i] * phi[j];
            }
            if (!wave) {
                // 080AdvectionLinear_SelfTest.cpp:108-121: result(j, i) = phi_i (a . grad phi_j)
                for (int j = 0; j < nB; ++j) {
                    double ag = 0.0;
                    for (int r = 0; r < d; ++r) ag += a[r] * gq[j * d + r];
                    for (int i = 0; i < nB; ++i) K[(size_t)j * R + i] += wq * phi[i] * ag;
                }
            } else {
                // AcousticWaveLinear_Impl.h:171-207: test i, basis j
                for (int j = 0; j < nB; ++j)
                    for (int i = 0; i < nB; ++i)
                        for (int c = 0; c < d; ++c) {
                            const double t = wq * gq[j * d + c] * phi[i];
                            K[(size_t)i * R + (c + 1) * nB + j] += t;
                            K[(size_t)((c + 1) * nB + i) * R + j] += t;
                        }
            }
        }
        s.mass_id[e] = s.pool.add(M.data());
        s.stiffness_id[e] = s.pool.add(K.data());
        by_jacobian.emplace(jkey, std::make_pair(s.mass_id[e], s.stiffness_id[e]));
    }
    s.face_elements.assign(desc.face_elements, desc.face_elements + 2 * s.F);
    s.face_id.assign(4 * s.F, -1);
    std::vector<double> B(4 * RR);
    // a face's blocks depend on its two tabulations and its normal only
    std::map<std::string, int64_t> by_face;
    for (int64_t f = 0; f < s.F; ++f) {
        const int64_t L = desc.face_elements[2 * f], Rt = desc.face_elements[2 * f + 1];
        if (L < 0 || L >= s.E || Rt < -1 || Rt >= s.E) throw std::invalid_argument("bad face table");
        // a boundary face (right element -1) has only its (LEFT, LEFT) block
        // (FaceMatrix of one side; Face::isInternal() false)
        const bool boundary = Rt < 0;
        if (boundary && upwind) throw std::invalid_argument("the upwind wave has no boundary faces here");
        const int tab[3] = {desc.face_tab_index[2 * f], boundary ? desc.face_tab_index[2 * f] : desc.face_tab_index[2 * f + 1],
                            boundary ? 1 : 0};
        if (tab[0] < 0 || tab[1] < 0 || tab[0] >= desc.n_face_tabs || tab[1] >= desc.n_face_tabs)
            throw std::invalid_argument("bad face tabulation index");
        const double *n = desc.face_normals + f * d;
        std::string fkey = geometry_key(n, d, tab, 3);
        auto known = by_face.find(fkey);
        if (known != by_face.end()) {
            for (int b = 0; b < 4; ++b) s.face_id[4 * f + b] = s.face_id[4 * known->second + b];
            continue;
        }
        by_face.emplace(std::move(fkey), f);
        double area = 0.0;
        for (int c = 0; c < d; ++c) area += n[c] * n[c];
        area = std::sqrt(area);
        std::fill(B.begin(), B.end(), 0.0);
        for (int q = 0; q < nQf; ++q) {
            const double *ph[2] = {desc.face_tabs + ((size_t)tab[0] * nQf + q) * nB,
                                   desc.face_tabs + ((size_t)tab[1] * nQf + q) * nB};
            if (!wave) {
                // 080AdvectionLinear_SelfTest.cpp:125-168: row j (test), column i (trial) on the
                // upwind side, -(a . n_j) phi_j phi_i with n_j the unit normal out of j's side,
                // halved when the flow is parallel to the face; integrated with w |n|
                double A = 0.0;
                for (int c = 0; c < d; ++c) A += a[c] * (n[c] / area);
                const double wq = desc.face_weights[q] * area;
                for (int ts = 0; ts < (boundary ? 1 : 2); ++ts)
                    for (int tr = 0; tr < (boundary ? 1 : 2); ++tr) {
                        double factor = 0.0;
                        if (A > 1e-12) factor = tr == 0 ? 1.0 : 0.0;
                        else if (A < -1e-12) factor = tr == 1 ? 1.0 : 0.0;
                        else if (std::fabs(A) < 1e-12) factor = 0.5;
                        if (factor == 0.0) continue;
                        const double an = ts == 0 ? A : -A;
                        double *blk = B.data() + (2 * ts + tr) * RR;
                        for (int j = 0; j < nB; ++j)
                            for (int i = 0; i < nB; ++i) blk[(size_t)j * R + i] += wq * (-an * ph[ts][j] * ph[tr][i]) * factor;
                    }
            } else {
                // AcousticWaveLinear_Impl.h:217-282 (internal faces): test side iS, basis side jS,
                // normal out of the left element, negated for a right-side basis function;
                // the normal carries the face scale (no |n| factor)
                const double wq = desc.face_weights[q];
                for (int ts = 0; ts < (boundary ? 1 : 2); ++ts)
                    for (int tr = 0; tr < (boundary ? 1 : 2); ++tr) {
                        const double sgn = tr == 1 ? -1.0 : 1.0;
                        double *blk = B.data() + (2 * ts + tr) * RR;
                        for (int j = 0; j < nB; ++j)
                            for (int i = 0; i < nB; ++i) {
                                const double pp = wq * ph[tr][j] * ph[ts][i];
                                for (int c = 0; c < d; ++c) {
                                    if (boundary) {  // :254-258 and :271-272: -n_d in (p, s_d), 0 in (s_d, p)
                                        blk[(size_t)i * R + (c + 1) * nB + j] += -n[c] * pp;
                                        continue;
                                    }
                                    const double t = -0.5 * sgn * n[c] * pp;
                                    blk[(size_t)i * R + (c + 1) * nB + j] += t;
                                    blk[(size_t)((c + 1) * nB + i) * R + j] += t;
                                }
                                if (upwind) {  // own side: -(1/2) |A_n|; other side: +(1/2) |A_n|
                                    const double side = ts == tr ? -0.5 : 0.5;
                                    blk[(size_t)i * R + j] += side * c_wave * area * pp;
                                    for (int c = 0; c < d; ++c)
                                        for (int m = 0; m < d; ++m)
                                            blk[(size_t)((c + 1) * nB + i) * R + (m + 1) * nB + j] +=
                                                side * c_wave * desc.c_inv * n[c] * n[m] / area * pp;
                                }
                            }
                    }
            }
        }
        for (int b = 0; b < (boundary ? 1 : 4); ++b) s.face_id[4 * f + b] = s.pool.add(B.data() + b * RR);
    }
    return s;
}

LinearOperators fold_linear(const LinearSystem &s) {
    const int R = s.R;
    const size_t RR = (size_t)R * R;
    LinearOperators out;
    out.R = R;
    out.E = s.E;
    // per element: own-side blocks and neighbour blocks in face order
    std::vector<std::vector<int32_t>> own(s.E);
    std::vector<std::vector<std::pair<int32_t, int32_t>>> nb(s.E);  // (neighbour, block)
    for (int64_t f = 0; f < s.F; ++f) {
        const int64_t L = s.face_elements[2 * f], Rt = s.face_elements[2 * f + 1];
        own[L].push_back(s.face_id[4 * f + 0]);
        if (Rt >= 0) {
            nb[L].push_back({(int32_t)Rt, s.face_id[4 * f + 1]});
            nb[Rt].push_back({(int32_t)L, s.face_id[4 * f + 2]});
            own[Rt].push_back(s.face_id[4 * f + 3]);
        }
    }
    for (int64_t e = 0; e < s.E; ++e) out.slots = std::max(out.slots, (int)nb[e].size());

    // distinct products M^{-1} (sum of pool matrices): key = mass id, then the summed ids
    std::map<std::vector<int32_t>, int> products;
    std::vector<std::vector<int32_t>> keys;
    auto product_id = [&](std::vector<int32_t> key) {
        auto it = products.find(key);
        if (it != products.end()) return it->second;
        const int id = (int)keys.size();
        products.emplace(key, id);
        keys.push_back(std::move(key));
        return id;
    };
    out.self_mat.resize(s.E);
    out.nbr.assign((size_t)s.E * out.slots, -1);
    out.nbr_mat.assign((size_t)s.E * out.slots, -1);
    for (int64_t e = 0; e < s.E; ++e) {
        std::vector<int32_t> key{s.mass_id[e], s.stiffness_id[e]};
        std::sort(own[e].begin(), own[e].end());  // the same blocks give the same key in any face order
        key.insert(key.end(), own[e].begin(), own[e].end());
        out.self_mat[e] = product_id(std::move(key));
        // neighbour slots ordered by their matrix: elements whose neighbour blocks
        // are the same matrices get the same tuple whatever the order of their
        // faces in the face list (periodic boundaries list them differently)
        std::vector<std::pair<int32_t, int32_t>> slots_e;  // (matrix, neighbour)
        for (size_t k = 0; k < nb[e].size(); ++k)
            slots_e.push_back({product_id({s.mass_id[e], nb[e][k].second}), nb[e][k].first});
        std::stable_sort(slots_e.begin(), slots_e.end(),
                         [](const std::pair<int32_t, int32_t> &x, const std::pair<int32_t, int32_t> &y) {
                             return x.first < y.first;
                         });
        for (size_t k = 0; k < slots_e.size(); ++k) {
            out.nbr[(size_t)e * out.slots + k] = slots_e[k].second;
            out.nbr_mat[(size_t)e * out.slots + k] = slots_e[k].first;
        }
    }

    // inverse of every distinct mass matrix that is used
    std::map<int32_t, int> inv_index;
    for (const auto &k : keys) inv_index.emplace(k[0], 0);
    std::vector<int32_t> inv_ids;
    for (auto &kv : inv_index) {
        kv.second = (int)inv_ids.size();
        inv_ids.push_back(kv.first);
    }
    std::vector<double> inv(inv_ids.size() * RR);
    parallel_for((int64_t)inv_ids.size(), [&](int64_t i) { invert_matrix(R, s.pool.get(inv_ids[i]), &inv[i * RR]); });

    out.table.assign(keys.size() * RR, 0.0);
    parallel_for((int64_t)keys.size(), [&](int64_t p) {
        const std::vector<int32_t> &k = keys[p];
        std::vector<double> S(s.pool.get(k[1]), s.pool.get(k[1]) + RR);
        for (size_t t = 2; t < k.size(); ++t) {
            const double *m = s.pool.get(k[t]);
            for (size_t x = 0; x < RR; ++x) S[x] += m[x];
        }
        const double *Mi = &inv[(size_t)inv_index.at(k[0]) * RR];
        double *D = &out.table[p * RR];
        for (int i = 0; i < R; ++i)
            for (int l = 0; l < R; ++l) {
                const double mil = Mi[(size_t)i * R + l];
                if (mil == 0.0) continue;
                const double *srow = &S[(size_t)l * R];
                double *drow = D + (size_t)i * R;
                for (int j = 0; j < R; ++j) drow[j] += mil * srow[j];
            }
    });
    return out;
}

}  // namespace hgg
