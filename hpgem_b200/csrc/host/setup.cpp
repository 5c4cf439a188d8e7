// Host-side set-up of hpGEM, restated for the stand-alone path (see setup.h).
#include "setup.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <sstream>
#include <stdexcept>
#include <unordered_map>

namespace hgg {

// ---------------------------------------------------------------------------
// quadrature
// ---------------------------------------------------------------------------
namespace {

struct SimplexRuleEntry {
    const char *name;
    int shape, order, n, offset;
};
#include "simplex_rules.inc"

// Gauss-Legendre nodes and weights on [-1, 1] by Newton's method on P_n
// (the classical construction; hpGEM's line rules Cn1_1_1 .. C1_11_6 are these
// rules, GaussQuadratureRulesForLine.cpp).
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    const double pi = 3.14159265358979323846;
    for (int i = 0; i < n; ++i) {
        double z = std::cos(pi * (i + 0.75) / (n + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = pk;
            }
            double pn = n == 1 ? z : p1, pm = n == 1 ? 1.0 : p0;
            dp = n * (z * pn - pm) / (z * z - 1.0);
            double dz = pn / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-17 && it > 3) break;
        }
        // derivative at the converged root
        double p0 = 1.0, p1 = z;
        for (int k = 2; k <= n; ++k) {
            double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = pk;
        }
        double pn = n == 1 ? z : p1, pm = n == 1 ? 1.0 : p0;
        dp = n * (z * pn - pm) / (z * z - 1.0);
        x[n - 1 - i] = z;
        w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
    for (int i = 0; i < n / 2; ++i) {  // exact symmetry
        double s = 0.5 * (x[n - 1 - i] - x[i]);
        x[i] = -s;
        x[n - 1 - i] = s;
        double ws = 0.5 * (w[i] + w[n - 1 - i]);
        w[i] = w[n - 1 - i] = ws;
    }
}

Rule tensor_rule(int shape, int n) {
    std::vector<double> x, w;
    gauss_legendre(n, x, w);
    Rule r;
    r.order = 2 * n - 1;
    if (shape == LINE) {
        r.dim = 1;
        r.name = "C1_" + std::to_string(n);
        for (int i = 0; i < n; ++i) {
            r.points.push_back(x[i]);
            r.weights.push_back(w[i]);
        }
    } else if (shape == SQUARE) {  // x fastest (GaussQuadratureRulesForSquare.cpp:152-182)
        r.dim = 2;
        r.name = "C2_" + std::to_string(n);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                r.points.push_back(x[i]);
                r.points.push_back(x[j]);
                r.weights.push_back(w[i] * w[j]);
            }
    } else {  // cube: z fastest (GaussQuadratureRulesForCube.cpp:282-304)
        r.dim = 3;
        r.name = "C3_" + std::to_string(n);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) {
                    r.points.push_back(x[i]);
                    r.points.push_back(x[j]);
                    r.points.push_back(x[k]);
                    r.weights.push_back(w[i] * w[j] * w[k]);
                }
    }
    return r;
}

}  // namespace

Rule get_rule(int shape, int order) {
    if (shape == 0) {
        Rule r;
        r.name = "Cn0_inf_1";
        r.order = 1 << 30;
        r.dim = 0;
        r.weights = {1.0};
        return r;
    }
    if (is_hypercube(shape)) {
        for (int n = 1; n <= 6; ++n)
            if (2 * n - 1 >= order) return tensor_rule(shape, n);
        throw std::invalid_argument("no quadrature rule of order " + std::to_string(order));
    }
    // the registry keeps rules sorted by order (AllGaussQuadratureRules::addRule, :119-131)
    std::vector<const SimplexRuleEntry *> sorted;
    for (const auto &e : kSimplexRules) {
        if (e.shape != shape) continue;
        auto it = sorted.begin();
        while (it != sorted.end() && (*it)->order < e.order) ++it;
        sorted.insert(it, &e);
    }
    for (const SimplexRuleEntry *e : sorted) {
        if (e->order < order) continue;
        Rule r;
        r.name = e->name;
        r.order = e->order;
        r.dim = shape == TRIANGLE ? 2 : 3;
        const double *d = kSimplexData + e->offset;
        for (int i = 0; i < e->n; ++i) {
            r.weights.push_back(d[0]);
            for (int k = 0; k < r.dim; ++k) r.points.push_back(d[1 + k]);
            d += 1 + r.dim;
        }
        return r;
    }
    throw std::invalid_argument("no quadrature rule of order " + std::to_string(order));
}

// ---------------------------------------------------------------------------
// structured meshes (applications/Preprocessor/lib/hpgem.cpp:55-265)
// ---------------------------------------------------------------------------
StructuredDescription parse_structured(const std::string &text) {
    std::istringstream in(text);
    std::string word;
    int version = 0, dim = 0;
    in >> word >> version >> dim;
    if (word != "structured" || version != 1 || dim < 1 || dim > 3)
        throw std::invalid_argument("not a 'structured 1 <dim>' mesh description");
    StructuredDescription d;
    d.n.resize(dim);
    d.lower.resize(dim);
    d.upper.resize(dim);
    for (auto &v : d.n) in >> v;
    for (auto &v : d.lower) in >> v;
    for (auto &v : d.upper) in >> v;
    std::string kind;
    in >> kind;
    if (kind != "triangular" && kind != "rectangular")
        throw std::invalid_argument("mesh must be either triangular or rectangular");
    d.triangular = kind == "triangular";
    for (int i = 0; i < dim; ++i) {
        std::string b;
        in >> b;
        if (b != "true" && b != "false") throw std::invalid_argument("bad periodicity flag");
        d.periodic.push_back(b == "true");
    }
    if (!in) throw std::invalid_argument("truncated mesh description");
    for (auto v : d.n)
        if (v < 1) throw std::invalid_argument("element counts must be positive");
    if (d.triangular && dim == 1) throw std::invalid_argument("no simplices in one dimension");
    return d;
}

namespace {

struct FaceKey {
    std::array<int64_t, 4> v;
    bool operator==(const FaceKey &o) const { return v == o.v; }
};
struct FaceKeyHash {
    size_t operator()(const FaceKey &k) const {
        uint64_t h = 1469598103934665603ull;
        for (int64_t x : k.v) {
            h ^= (uint64_t)x + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
            h *= 1099511628211ull;
        }
        return (size_t)h;
    }
};

}  // namespace

Mesh structured_mesh(const StructuredDescription &d) {
    const int dim = (int)d.n.size();
    std::vector<int64_t> n_elem(d.n), n_nodes(dim);
    std::vector<double> size(dim);
    for (int i = 0; i < dim; ++i) {
        n_nodes[i] = n_elem[i] + (d.periodic[i] ? 0 : 1);
        size[i] = d.upper[i] - d.lower[i];  // hpgem.cpp:87-89
    }
    Mesh m;
    m.dim = dim;
    m.shape = dim == 1 ? LINE : (dim == 2 ? (d.triangular ? TRIANGLE : SQUARE)
                                          : (d.triangular ? TETRAHEDRON : CUBE));
    const ShapeInfo &si = shape_info(m.shape);
    m.n_vertices = si.n_vertices;

    // coordinate `sub` of node `node` (getNodeCoordinates, hpgem.cpp:100-137): the
    // base position, shifted by the period in the k-th direction in which the node
    // has index 0 when bit k of `sub` is set
    auto node_coordinate = [&](int64_t node, int sub, double *x) {
        int64_t rest = node;
        int k = 0;
        for (int i = 0; i < dim; ++i) {
            int64_t idx = rest % n_nodes[i];
            rest /= n_nodes[i];
            x[i] = d.lower[i] + idx * size[i] / n_elem[i];
            if (d.periodic[i] && idx == 0) {
                if ((sub >> k) & 1) x[i] += size[i];
                ++k;
            }
        }
    };

    std::vector<int> rotate = {2, 0, 3, 1, 6, 4, 7, 5};
    std::vector<std::vector<int>> corners;
    if (dim == 2) corners = {{0, 1, 2}, {1, 3, 2}};
    if (dim == 3) corners = {{1, 2, 4, 7}, {0, 1, 2, 4}, {1, 3, 2, 7}, {1, 4, 5, 7}, {2, 6, 4, 7}};
    std::vector<int64_t> mult(1, 1);
    for (int i = 1; i < dim; ++i) mult.push_back(mult.back() * n_nodes[i - 1]);

    int64_t cells = 1;
    for (int i = 0; i < dim; ++i) cells *= n_elem[i];
    m.n_elements = cells * (d.triangular ? (int64_t)corners.size() : 1);
    m.nodes.resize(m.n_elements * m.n_vertices);
    m.coords.resize(m.n_elements * m.n_vertices * dim);

    std::vector<int64_t> loop(dim, 0);
    size_t tri = 0;
    const int cube_vertices = 1 << dim;
    std::vector<int64_t> ids(cube_vertices);
    std::vector<int> subs(cube_vertices);
    for (int64_t e = 0; e < m.n_elements; ++e) {
        // element vertex list, hpgem.cpp:159-181
        ids.assign(1, 0);
        for (int i = 0; i < dim; ++i) {
            size_t cur = ids.size();
            for (size_t j = 0; j < cur; ++j) {
                ids[j] += loop[i] * mult[i];
                ids.push_back(ids[j] + mult[i]);
            }
        }
        for (int j = 0; j < cube_vertices; ++j) {
            int sub = 0, prev = 0;
            for (int i = 0; i < dim; ++i) {
                if (((j & (1 << i)) != 0) && (loop[i] == n_nodes[i] - 1)) {
                    ids[j] -= n_nodes[i] * mult[i];
                    sub += 1 << prev++;
                }
                if (d.periodic[i] && (loop[i] + (j & (1 << i)) == 0)) prev++;
            }
            subs[j] = sub;
        }
        for (int v = 0; v < m.n_vertices; ++v) {
            int j = d.triangular ? corners[tri][v] : v;
            m.nodes[e * m.n_vertices + v] = ids[j];
            node_coordinate(ids[j], subs[j], &m.coords[(e * m.n_vertices + v) * dim]);
        }
        if (d.triangular && ++tri == corners.size()) tri = 0;
        if (tri == 0) {  // advance, with the alternating rotation of hpgem.cpp:182-221
            for (int i = 0; i < dim; ++i) {
                for (auto &c : corners)
                    for (int &k : c) k = rotate[k];
                if (++loop[i] < n_elem[i]) break;
                for (auto &c : corners)
                    for (int &k : c)
                        if (loop[i] % 2 == 1) k = rotate[k];
                loop[i] = 0;
            }
        }
    }

    pair_faces(m);
    return m;
}

// Pairs the elements' faces by their (global) node sets, in order of first
// appearance; periodic copies of a node share its number, so periodic faces pair.
void pair_faces(Mesh &m) {
    const ShapeInfo &si = shape_info(m.shape);
    const int dim = m.dim;
    const int fv = dim == 1 ? 1 : si.face_vertices;
    std::unordered_map<FaceKey, int64_t, FaceKeyHash> open;
    open.reserve((size_t)(m.n_elements * si.n_faces / 2 + 16));
    for (int64_t e = 0; e < m.n_elements; ++e) {
        for (int f = 0; f < si.n_faces; ++f) {
            FaceKey key{{-1, -1, -1, -1}};
            int64_t g[4];
            for (int k = 0; k < fv; ++k) g[k] = key.v[k] = m.nodes[e * m.n_vertices + si.faces[f][k]];
            std::sort(key.v.begin(), key.v.begin() + fv);
            auto it = open.find(key);
            if (it == open.end()) {
                open.emplace(key, m.n_faces());
                m.face_elements.push_back(e);
                m.face_elements.push_back(-1);
                m.face_local.push_back(f);
                m.face_local.push_back(-1);
                for (int k = 0; k < fv; ++k) m.face_perm.push_back(-1);
            } else {
                int64_t fid = it->second;
                open.erase(it);
                int64_t L = m.face_elements[2 * fid];
                int fL = m.face_local[2 * fid];
                m.face_elements[2 * fid + 1] = e;
                m.face_local[2 * fid + 1] = f;
                for (int k = 0; k < fv; ++k) {
                    int64_t want = m.nodes[L * m.n_vertices + si.faces[fL][k]];
                    int slot = -1;
                    for (int s = 0; s < fv; ++s)
                        if (g[s] == want) slot = s;
                    m.face_perm[fid * fv + k] = slot;
                }
            }
        }
    }
}

// A "mesh 2" file as the Preprocessor writes it and MeshManipulator::readMesh
// reads it: "mesh 2"; "nNodes nElements dim [nFaces [nEdges]]"; a partition
// line; "zones", their count and names; "nodes", then per node a partition line
// and "k x_1 ... x_{k dim}" (k coordinate copies, hexadecimal floating point;
// periodic nodes have several); "elements", then per element
// "n node_1 copy_1 ... node_n copy_n zone ..." and a shadow line.  Faces are
// paired from the element nodes as for the structured generator.
Mesh read_mesh2(const std::string &text) {
    std::vector<std::string> lines;
    {
        std::istringstream in(text);
        std::string ln;
        while (std::getline(in, ln)) {
            const size_t a = ln.find_first_not_of(" \t\r"), b = ln.find_last_not_of(" \t\r");
            lines.push_back(a == std::string::npos ? std::string() : ln.substr(a, b - a + 1));
        }
    }
    auto bad = [](const std::string &what) { return std::invalid_argument("mesh file: " + what); };
    if (lines.size() < 3 || lines[0] != "mesh 2") throw bad("first line is not \"mesh 2\"");
    std::istringstream head(lines[1]);
    int64_t n_nodes = -1, n_elem = -1;
    int dim = -1;
    head >> n_nodes >> n_elem >> dim;
    if (n_nodes <= 0 || n_elem <= 0 || dim < 1 || dim > 3) throw bad("bad header \"" + lines[1] + "\"");
    size_t i = 2;
    while (i < lines.size() && lines[i] != "zones") ++i;
    if (i + 1 >= lines.size()) throw bad("no zones section");
    const int n_zones = std::stoi(lines[i + 1]);
    i += 2 + n_zones;
    if (i >= lines.size() || lines[i] != "nodes") throw bad("no nodes section");
    ++i;
    std::vector<std::vector<double>> node_coords((size_t)n_nodes);
    for (int64_t nd = 0; nd < n_nodes; ++nd) {
        ++i;  // partition line
        if (i >= lines.size()) throw bad("truncated nodes section");
        const char *c = lines[i].c_str();
        char *end = nullptr;
        const long k = std::strtol(c, &end, 10);
        if (k < 1) throw bad("node without coordinates");
        c = end;
        for (long j = 0; j < k * dim; ++j) {
            const double v = std::strtod(c, &end);  // reads hexadecimal floating point
            if (end == c) throw bad("node coordinate");
            node_coords[nd].push_back(v);
            c = end;
        }
        ++i;
    }
    if (i >= lines.size() || lines[i] != "elements") throw bad("no elements section");
    ++i;
    Mesh m;
    m.dim = dim;
    m.n_elements = n_elem;
    for (int64_t e = 0; e < n_elem; ++e, i += 2) {
        if (i >= lines.size()) throw bad("truncated elements section");
        std::istringstream el(lines[i]);
        int nv = 0;
        el >> nv;
        const int shape = dim == 1 ? (nv == 2 ? LINE : -1)
                        : dim == 2 ? (nv == 3 ? TRIANGLE : nv == 4 ? SQUARE : -1)
                                   : (nv == 4 ? TETRAHEDRON : nv == 8 ? CUBE : -1);
        if (shape < 0) throw bad("element with " + std::to_string(nv) + " vertices in " + std::to_string(dim) + "D");
        if (e == 0) {
            m.shape = shape;
            m.n_vertices = nv;
            m.nodes.resize((size_t)n_elem * nv);
            m.coords.resize((size_t)n_elem * nv * dim);
        } else if (shape != m.shape) {
            throw bad("mixed element shapes are not supported");
        }
        for (int v = 0; v < nv; ++v) {
            int64_t nd = -1, copy = -1;
            el >> nd >> copy;
            if (!el || nd < 0 || nd >= n_nodes || copy < 0 || (copy + 1) * dim > (int64_t)node_coords[nd].size())
                throw bad("element vertex out of range");
            m.nodes[e * nv + v] = nd;
            for (int k = 0; k < dim; ++k) m.coords[(e * nv + v) * dim + k] = node_coords[nd][copy * dim + k];
        }
    }
    pair_faces(m);
    return m;
}

void reference_to_physical(const Mesh &m, int64_t e, const double *xi, double *x) {
    double N[8];
    vertex_shape_functions(m.shape, xi, N);
    for (int r = 0; r < m.dim; ++r) {
        double s = 0.0;
        for (int k = 0; k < m.n_vertices; ++k) s += N[k] * m.coords[(e * m.n_vertices + k) * m.dim + r];
        x[r] = s;
    }
}

void face_to_element(int shape, const int *face_vertices, const double *xi_face, double *xi) {
    const ShapeInfo &s = shape_info(shape);
    double N[4];
    int fv = s.dim == 1 ? 1 : s.face_vertices;
    vertex_shape_functions(s.face_shape, xi_face, N);
    for (int c = 0; c < s.dim; ++c) {
        double v = 0.0;
        for (int k = 0; k < fv; ++k) v += N[k] * s.vertices[face_vertices[k]][c];
        xi[c] = v;
    }
}

// ---------------------------------------------------------------------------
// Butcher tableaux (kernel/Base/TimeIntegration/*.cpp)
// ---------------------------------------------------------------------------
bool butcher_tableau(const std::string &name, std::vector<double> &a, std::vector<double> &b,
                     std::vector<double> &c, int &S) {
    std::vector<std::vector<double>> A;
    if (name == "RK4_4") {  // RK4Methods.cpp:45-63
        A = {{}, {0.5}, {0.0, 0.5}, {0.0, 0.0, 1.0}};
        b = {1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6};
        c = {0.0, 0.5, 0.5, 1.0};
    } else if (name == "DormandPrince") {  // DormandPrince.cpp:45-78
        A = {{},
             {1. / 5.},
             {3. / 40., 9. / 40.},
             {44. / 45., -56. / 15., 32. / 9.},
             {19372. / 6561., -25360. / 2187., 64448. / 6561., -212. / 729.},
             {9017. / 3168., -355. / 33., 46732. / 5247., 49. / 176., -5103. / 18656.},
             {35. / 384., 0., 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84.}};
        b = {35. / 384., 0., 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84., 0.};
        c = {0., 1. / 5., 3. / 10., 4. / 5., 8. / 9., 1., 1.};
    } else if (name == "ForwardEuler") {
        A = {{}};
        b = {1.0};
        c = {0.0};
    } else if (name == "MidPoint") {
        A = {{}, {0.5}};
        b = {0.0, 1.0};
        c = {0.0, 0.5};
    } else if (name == "RK2TVD") {
        A = {{}, {1.0}};
        b = {0.5, 0.5};
        c = {0.0, 0.0};
    } else if (name == "RK3TVD") {
        A = {{}, {1.0}, {0.25, 0.25}};
        b = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0};
        c = {0.0, 0.0, 0.0};
    } else if (name == "BogackiShampine") {
        A = {{}, {1. / 2.}, {0., 3. / 4.}, {2. / 9., 1. / 3., 4. / 9.}};
        b = {2. / 9., 1. / 3., 4. / 9., 0.};
        c = {0., 1. / 5., 3. / 10., 4. / 5.};
    } else {
        return false;
    }
    S = (int)b.size();
    a.assign(S * S, 0.0);
    for (int i = 0; i < S; ++i)
        for (size_t j = 0; j < A[i].size(); ++j) a[i * S + j] = A[i][j];
    return true;
}

bool butcher_error_estimate(const std::string &name, std::vector<double> &error, int &order) {
    if (name == "DormandPrince") {  // the fifth-order weights minus the fourth-order ones
        error = {35. / 384. - 5179. / 57600., 0. - 0., 500. / 1113. - 7571. / 16695., 125. / 192. - 393. / 640.,
                 -2187. / 6784. - -92097. / 339200., 11. / 84. - 187. / 2100., 0. - 1. / 40.};
        order = 5;
        return true;
    }
    if (name == "BogackiShampine") {  // the third-order weights minus the second-order ones
        error = {2. / 9. - 7. / 24., 1. / 3. - 1. / 4., 4. / 9. - 1. / 3., 0. - 1. / 8.};
        order = 3;
        return true;
    }
    return false;
}

// ---------------------------------------------------------------------------
// descriptor contents for a structured mesh
// ---------------------------------------------------------------------------
StructuredProblem build_structured(const std::string &description, int order, int physics,
                                   const double *params, const std::string &tableau, bool boundary_faces) {
    return build_problem(structured_mesh(parse_structured(description)), order, physics, params, tableau,
                         boundary_faces);
}

StructuredProblem build_problem(Mesh mesh, int order, int physics, const double *params, const std::string &tableau,
                                bool boundary_faces) {
    StructuredProblem P;
    P.mesh = std::move(mesh);
    const Mesh &m = P.mesh;
    const ShapeInfo &si = shape_info(m.shape);
    const int d = m.dim;
    P.order = order;
    P.physics = physics;
    P.n_vars = physics == 0 ? 1 : d + 1;
    if (physics == 0) {
        for (int i = 0; i < d; ++i) P.advection[i] = params ? params[i] : 0.0;
    } else {
        P.c_inv = params ? params[0] : 1.0;
    }
    for (int64_t f = 0; f < m.n_faces() && !boundary_faces; ++f)
        if (m.face_elements[2 * f + 1] < 0)
            throw std::invalid_argument("boundary faces are not supported: use a fully periodic mesh");
    if (!butcher_tableau(tableau, P.rk_a, P.rk_b, P.rk_c, P.n_stages))
        throw std::invalid_argument("unknown Butcher tableau " + tableau);

    // Element rule of order 2p+1 (Element::setDefaultBasisFunctionSet, Element.cpp:89-98).
    // Face rule of order 2p+1 as well: the faces are created while the elements
    // still hold the rule of their empty basis (Element.h:583, Face.cpp:149-168),
    // and setQuadratureRulesWithOrder(2p+1) then gives every face of the element
    // the face shape's rule for the requested order 2p+1, not for the element
    // rule's actual order (Element.cpp:144-175).  The two differ for triangles at
    // p = 1 (2 against 3 points) and p = 3 (4 against 5); only integrands that are
    // not polynomials (source terms) see the difference.
    P.rule = get_rule(m.shape, 2 * order + 1);
    P.face_rule = get_rule(si.face_shape, 2 * order + 1);
    try {  // the reference has no rule of order 2p+2 for every shape (e.g. p = 5)
        P.error_rule = get_rule(m.shape, 2 * order + 2);
    } catch (const std::invalid_argument &) {
        P.error_rule = Rule();
    }
    P.n_basis = basis_count(m.shape, order);
    const int nB = P.n_basis, nQ = P.rule.size();
    std::vector<Dual> vals;
    P.basis_values.resize((size_t)nQ * nB);
    P.basis_grads.resize((size_t)nQ * nB * d);
    for (int q = 0; q < nQ; ++q) {
        eval_basis(m.shape, order, &P.rule.points[q * d], vals);
        for (int j = 0; j < nB; ++j) {
            P.basis_values[q * nB + j] = vals[j].v;
            for (int k = 0; k < d; ++k) P.basis_grads[(q * nB + j) * d + k] = vals[j].g[k];
        }
    }
    const int nE = P.error_rule.size();
    P.error_basis.resize((size_t)nE * nB);
    for (int q = 0; q < nE; ++q) {
        eval_basis(m.shape, order, &P.error_rule.points[q * d], vals);
        for (int j = 0; j < nB; ++j) P.error_basis[q * nB + j] = vals[j].v;
    }

    // element Jacobians of the vertex map at the reference centroid
    double centre[3] = {0, 0, 0};
    for (int k = 0; k < si.n_vertices; ++k)
        for (int c = 0; c < d; ++c) centre[c] += si.vertices[k][c] / si.n_vertices;
    double N[8], dN[24];
    vertex_shape_functions(m.shape, centre, N, dN);
    P.jacobians.assign((size_t)m.n_elements * d * d, 0.0);
    for (int64_t e = 0; e < m.n_elements; ++e)
        for (int r = 0; r < d; ++r)
            for (int c = 0; c < d; ++c) {
                double s = 0.0;
                for (int k = 0; k < si.n_vertices; ++k)
                    s += m.coords[(e * si.n_vertices + k) * d + r] * dN[k * d + c];
                P.jacobians[(e * d + r) * d + c] = s;
            }

    // face tabulations: one per (local face, vertex order) that occurs
    const int fv = d == 1 ? 1 : si.face_vertices;
    const int nQf = P.face_rule.size();
    std::map<std::vector<int>, int> tabs;
    auto tab_of = [&](const std::vector<int> &verts) {
        auto it = tabs.find(verts);
        if (it != tabs.end()) return it->second;
        int id = (int)tabs.size();
        tabs.emplace(verts, id);
        for (int q = 0; q < nQf; ++q) {
            double xi[3];
            face_to_element(m.shape, verts.data(), &P.face_rule.points[q * (d - 1)], xi);
            eval_basis(m.shape, order, xi, vals);
            for (int j = 0; j < nB; ++j) P.face_tabs.push_back(vals[j].v);
        }
        return id;
    };
    const int64_t F = m.n_faces();
    P.face_tab_index.resize(2 * F);
    P.normals.resize(F * d);
    std::vector<int> verts(fv);
    double fcentre[3] = {0, 0, 0};
    if (d > 1) {
        const ShapeInfo &fs = shape_info(si.face_shape);
        for (int k = 0; k < fs.n_vertices; ++k)
            for (int c = 0; c < d - 1; ++c) fcentre[c] += fs.vertices[k][c] / fs.n_vertices;
    }
    for (int64_t f = 0; f < F; ++f) {
        int64_t L = m.face_elements[2 * f];
        int fL = m.face_local[2 * f], fR = m.face_local[2 * f + 1];
        for (int k = 0; k < fv; ++k) verts[k] = si.faces[fL][k];
        P.face_tab_index[2 * f] = tab_of(verts);
        if (m.face_elements[2 * f + 1] >= 0) {
            for (int k = 0; k < fv; ++k) verts[k] = si.faces[fR][m.face_perm[f * fv + k]];
            P.face_tab_index[2 * f + 1] = tab_of(verts);
        } else {  // boundary face: no right side; its index repeats the left one
            P.face_tab_index[2 * f + 1] = P.face_tab_index[2 * f];
        }

        // normal (FaceGeometry::getNormalVector): tangents J * d(face map), wedge, outward
        const double *J = &P.jacobians[L * d * d];
        double n[3] = {1.0, 0.0, 0.0};
        if (d > 1) {
            double T[3][2];
            for (int c = 0; c < d - 1; ++c) {
                double a[3], b[3], xp[3] = {fcentre[0], fcentre[1], fcentre[2]};
                double xm[3] = {fcentre[0], fcentre[1], fcentre[2]};
                xp[c] += 0.5;
                xm[c] -= 0.5;
                face_to_element(m.shape, si.faces[fL], xp, a);
                face_to_element(m.shape, si.faces[fL], xm, b);
                for (int r = 0; r < d; ++r) {
                    double s = 0.0;
                    for (int k = 0; k < d; ++k) s += J[r * d + k] * (a[k] - b[k]);
                    T[r][c] = s;
                }
            }
            if (d == 2) {
                n[0] = T[1][0];
                n[1] = -T[0][0];
            } else {
                n[0] = T[1][0] * T[2][1] - T[2][0] * T[1][1];
                n[1] = T[2][0] * T[0][1] - T[0][0] * T[2][1];
                n[2] = T[0][0] * T[1][1] - T[1][0] * T[0][1];
            }
        }
        double ec[3] = {0, 0, 0}, fc[3] = {0, 0, 0};
        for (int k = 0; k < si.n_vertices; ++k)
            for (int c = 0; c < d; ++c) ec[c] += m.coords[(L * si.n_vertices + k) * d + c] / si.n_vertices;
        for (int k = 0; k < fv; ++k)
            for (int c = 0; c < d; ++c) fc[c] += m.coords[(L * si.n_vertices + si.faces[fL][k]) * d + c] / fv;
        double dot = 0.0;
        for (int c = 0; c < d; ++c) dot += n[c] * (fc[c] - ec[c]);
        for (int c = 0; c < d; ++c) P.normals[f * d + c] = dot < 0 ? -n[c] : n[c];
    }
    P.n_face_tabs = (int)tabs.size();
    return P;
}

}  // namespace hgg
