// Source-term plan of HpgemAPILinear (sources.h).
#include "sources.h"

#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>

#include "operators.h"

namespace hgg {

namespace {

double abs_det(int d, const double *J) {
    if (d == 1) return std::fabs(J[0]);
    if (d == 2) return std::fabs(J[0] * J[3] - J[1] * J[2]);
    return std::fabs(J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
                     J[2] * (J[3] * J[7] - J[4] * J[6]));
}

}  // namespace

SourcePlan plan_sources(const StructuredProblem &P, const std::vector<double> &mass,
                        const std::vector<int32_t> &mass_of, bool element_source, bool boundary_source) {
    const Mesh &m = P.mesh;
    const ShapeInfo &si = shape_info(m.shape);
    SourcePlan sp;
    const int d = m.dim, nB = P.n_basis, V = P.n_vars, R = V * nB;
    const int nQ = P.rule.size(), nQf = P.face_rule.size();
    const int64_t E = m.n_elements, F = m.n_faces();
    sp.R = R;
    sp.V = V;
    sp.nB = nB;
    sp.dim = d;
    sp.nQ = nQ;
    sp.nQf = nQf;
    sp.element = element_source;
    sp.boundary = boundary_source;
    const size_t RR = (size_t)R * R;
    if ((int64_t)mass_of.size() != E || mass.size() % RR != 0)
        throw std::invalid_argument("source terms: mass matrices do not match the mesh");
    const int n_mass = (int)(mass.size() / RR);
    std::vector<double> minv(mass.size());
    for (int i = 0; i < n_mass; ++i) invert_matrix(R, &mass[i * RR], &minv[i * RR]);

    // distinct lifts, keyed by (kind, mass, tabulation, scale)
    std::map<std::string, int> known;
    auto lift_of = [&](int kind, int mid, int tab, double scale) {
        std::string key(reinterpret_cast<const char *>(&kind), sizeof kind);
        key.append(reinterpret_cast<const char *>(&mid), sizeof mid);
        key.append(reinterpret_cast<const char *>(&tab), sizeof tab);
        key.append(reinterpret_cast<const char *>(&scale), sizeof scale);
        auto it = known.find(key);
        if (it != known.end()) return it->second;
        const int np = kind == 0 ? nQ : nQf, cols = np * V;
        const double *phi = kind == 0 ? P.basis_values.data() : P.face_tabs.data() + (size_t)tab * nQf * nB;
        const double *w = kind == 0 ? P.rule.weights.data() : P.face_rule.weights.data();
        const double *Mi = &minv[(size_t)mid * RR];
        const size_t o = sp.table.size();
        sp.table.resize(o + (size_t)cols * R);
        for (int q = 0; q < np; ++q)
            for (int v = 0; v < V; ++v)
                for (int r = 0; r < R; ++r) {
                    double s = 0.0;
                    for (int j = 0; j < nB; ++j) s += Mi[(size_t)r * R + v * nB + j] * (w[q] * scale * phi[q * nB + j]);
                    sp.table[o + (size_t)(q * V + v) * R + r] = s;
                }
        const int id = (int)sp.table_off.size();
        sp.table_off.push_back((int64_t)o);
        sp.table_cols.push_back(cols);
        known.emplace(std::move(key), id);
        return id;
    };

    std::vector<std::vector<std::pair<int32_t, int64_t>>> entries(E);
    if (element_source) {
        sp.n_elem_points = E * nQ;
        sp.elem_xyz.resize((size_t)sp.n_elem_points * d);
        for (int64_t e = 0; e < E; ++e) {
            for (int q = 0; q < nQ; ++q)
                reference_to_physical(m, e, &P.rule.points[(size_t)q * d], &sp.elem_xyz[((size_t)e * nQ + q) * d]);
            const double J = abs_det(d, &P.jacobians[(size_t)e * d * d]);
            entries[e].push_back({lift_of(0, mass_of[e], 0, J), e * nQ * V});
        }
    }
    if (boundary_source) {
        const int64_t base = sp.n_elem_points * V;
        const int fv = d == 1 ? 1 : si.face_vertices;
        int64_t b = 0;
        for (int64_t f = 0; f < F; ++f) {
            if (m.face_elements[2 * f + 1] >= 0) continue;
            const int64_t L = m.face_elements[2 * f];
            const int fL = m.face_local[2 * f];
            const double *n = &P.normals[(size_t)f * d];
            double area = 0.0;
            for (int c = 0; c < d; ++c) area += n[c] * n[c];
            area = std::sqrt(area);
            int verts[4] = {0, 0, 0, 0};
            for (int k = 0; k < fv; ++k) verts[k] = si.faces[fL][k];
            for (int q = 0; q < nQf; ++q) {
                double xi[3] = {0, 0, 0}, x[3] = {0, 0, 0};
                face_to_element(m.shape, verts, P.face_rule.points.data() + (size_t)q * (d - 1), xi);
                reference_to_physical(m, L, xi, x);
                for (int c = 0; c < d; ++c) {
                    sp.face_xyz.push_back(x[c]);
                    sp.face_normals.push_back(n[c] / area);
                }
            }
            entries[L].push_back({lift_of(1, mass_of[L], P.face_tab_index[2 * f], area), base + b * nQf * V});
            ++b;
        }
        sp.n_face_points = b * nQf;
    }
    sp.values = (sp.n_elem_points + sp.n_face_points) * V;
    sp.ptr.push_back(0);
    for (int64_t e = 0; e < E; ++e) {
        if (entries[e].empty()) continue;
        sp.elem.push_back((int32_t)e);
        for (const auto &en : entries[e]) {
            sp.lift.push_back(en.first);
            sp.off.push_back(en.second);
        }
        sp.ptr.push_back((int32_t)sp.lift.size());
    }
    return sp;
}

}  // namespace hgg
