// Reference shapes and hpGEM's default H1 DG basis, evaluated on the host.
//
// Shapes (vertex coordinates, local vertex lists of faces and edges) follow
//   kernel/Geometry/ReferenceLine.cpp:54-61, ReferenceSquare.cpp:60-107,
//   ReferenceTriangle.cpp:59-60, ReferenceCube.cpp:52-74,
//   ReferenceTetrahedron.cpp:56-60.
// Basis sets follow, function by function and in the same order,
//   createDGBasisFunctionSet1DH1Line        kernel/FE/BasisFunctions1DH1ConformingLine.cpp:85-108
//   createDGBasisFunctionSet2DH1Square      kernel/FE/BasisFunctions2DH1ConformingSquare.cpp:164-184
//   createDGBasisFunctions2DH1Triangle      kernel/FE/BasisFunctions2DH1ConformingTriangle.cpp:176-200
//   createDGBasisFunctionSet3DH1Cube        kernel/FE/BasisFunctions3DH1ConformingCube.cpp:434-528
//   createDGBasisFunctionSet3DH1Tetrahedron kernel/FE/BasisFunctions3DH1ConformingTetrahedron.cpp:366-409
// with the Lobatto kernels of kernel/FE/helperFunctions.cpp:49-108.
// Gradients are carried alongside the values by forward-mode automatic
// differentiation (struct Dual), which reproduces the product-rule
// derivatives hpGEM writes out by hand in its evalDeriv* methods.
#pragma once

#include <cmath>
#include <stdexcept>
#include <vector>

namespace hgg {

enum Shape { LINE = 1, SQUARE = 2, TRIANGLE = 3, CUBE = 4, TETRAHEDRON = 5 };

struct ShapeInfo {
    int dim;
    int n_vertices;
    int n_faces;
    int face_shape;  // 0 = point
    int face_vertices;
    double vertices[8][3];
    int faces[6][4];
    int edges[12][2];
    int n_edges;
};

inline const ShapeInfo &shape_info(int shape) {
    static const ShapeInfo line = {1, 2, 2, 0, 1, {{-1}, {1}}, {{0}, {1}}, {}, 0};
    static const ShapeInfo square = {2, 4, 4, LINE, 2,
                                     {{-1, -1}, {1, -1}, {-1, 1}, {1, 1}},
                                     {{0, 1}, {0, 2}, {1, 3}, {2, 3}}, {}, 0};
    static const ShapeInfo triangle = {2, 3, 3, LINE, 2, {{0, 0}, {1, 0}, {0, 1}},
                                       {{0, 1}, {0, 2}, {1, 2}}, {}, 0};
    static const ShapeInfo cube = {3, 8, 6, SQUARE, 4,
                                   {{-1, -1, -1}, {1, -1, -1}, {-1, 1, -1}, {1, 1, -1},
                                    {-1, -1, 1}, {1, -1, 1}, {-1, 1, 1}, {1, 1, 1}},
                                   {{0, 1, 2, 3}, {0, 1, 4, 5}, {0, 2, 4, 6},
                                    {1, 3, 5, 7}, {2, 3, 6, 7}, {4, 5, 6, 7}},
                                   {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3},
                                    {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}},
                                   12};
    static const ShapeInfo tet = {3, 4, 4, TRIANGLE, 3,
                                  {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}},
                                  {{0, 3, 2}, {0, 1, 3}, {0, 2, 1}, {1, 2, 3}},
                                  {{0, 1}, {0, 2}, {0, 3}, {2, 3}, {1, 3}, {1, 2}},
                                  6};
    switch (shape) {
        case LINE: return line;
        case SQUARE: return square;
        case TRIANGLE: return triangle;
        case CUBE: return cube;
        case TETRAHEDRON: return tet;
    }
    throw std::invalid_argument("unknown shape");
}

inline bool is_hypercube(int shape) { return shape == LINE || shape == SQUARE || shape == CUBE; }

// reference measure of the shape (length / area / volume)
inline double shape_measure(int shape) {
    switch (shape) {
        case 0: return 1.0;
        case LINE: return 2.0;
        case SQUARE: return 4.0;
        case TRIANGLE: return 0.5;
        case CUBE: return 8.0;
        case TETRAHEDRON: return 1.0 / 6.0;
    }
    return 0.0;
}

// Shape functions of the vertices: multilinear on hypercubes (vertex k has
// bit i of k set when its coordinate i is +1), barycentric on simplices.
// They define the vertex maps MappingToPhysHypercubeLinear /
// MappingToPhysSimplexLinear (kernel/Geometry/Mappings/) and face maps.
inline void vertex_shape_functions(int shape, const double *xi, double *N, double *dN = nullptr) {
    if (shape == 0) {
        N[0] = 1.0;
        return;
    }
    const ShapeInfo &s = shape_info(shape);
    int d = s.dim;
    if (is_hypercube(shape)) {
        for (int k = 0; k < s.n_vertices; ++k) {
            double v = 1.0;
            for (int i = 0; i < d; ++i) v *= (1.0 + ((k >> i) & 1 ? 1.0 : -1.0) * xi[i]) / 2.0;
            N[k] = v;
            if (dN)
                for (int c = 0; c < d; ++c) {
                    double g = 1.0;
                    for (int i = 0; i < d; ++i) {
                        double sgn = (k >> i) & 1 ? 1.0 : -1.0;
                        g *= (i == c) ? sgn / 2.0 : (1.0 + sgn * xi[i]) / 2.0;
                    }
                    dN[k * d + c] = g;
                }
        }
        return;
    }
    double sum = 0.0;
    for (int i = 0; i < d; ++i) sum += xi[i];
    N[0] = 1.0 - sum;
    for (int i = 0; i < d; ++i) N[i + 1] = xi[i];
    if (dN)
        for (int k = 0; k <= d; ++k)
            for (int c = 0; c < d; ++c) dN[k * d + c] = (k == 0) ? -1.0 : (k == c + 1 ? 1.0 : 0.0);
}

// ---- forward-mode derivatives -----------------------------------------------
struct Dual {
    double v;
    double g[3];
};
inline Dual dconst(double c) { return Dual{c, {0, 0, 0}}; }
inline Dual operator+(Dual a, Dual b) {
    return Dual{a.v + b.v, {a.g[0] + b.g[0], a.g[1] + b.g[1], a.g[2] + b.g[2]}};
}
inline Dual operator-(Dual a, Dual b) {
    return Dual{a.v - b.v, {a.g[0] - b.g[0], a.g[1] - b.g[1], a.g[2] - b.g[2]}};
}
inline Dual operator*(Dual a, Dual b) {
    return Dual{a.v * b.v,
                {a.g[0] * b.v + a.v * b.g[0], a.g[1] * b.v + a.v * b.g[1],
                 a.g[2] * b.v + a.v * b.g[2]}};
}
inline Dual operator*(double c, Dual a) { return Dual{c * a.v, {c * a.g[0], c * a.g[1], c * a.g[2]}}; }
inline Dual operator*(Dual a, double c) { return c * a; }
inline Dual operator/(Dual a, double c) { return Dual{a.v / c, {a.g[0] / c, a.g[1] / c, a.g[2] / c}}; }
inline Dual operator+(double c, Dual a) { return Dual{c + a.v, {a.g[0], a.g[1], a.g[2]}}; }
inline Dual operator-(double c, Dual a) { return Dual{c - a.v, {-a.g[0], -a.g[1], -a.g[2]}}; }
inline Dual operator-(Dual a, double c) { return Dual{a.v - c, {a.g[0], a.g[1], a.g[2]}}; }
inline Dual operator+(Dual a, double c) { return c + a; }
inline Dual operator-(Dual a) { return Dual{-a.v, {-a.g[0], -a.g[1], -a.g[2]}}; }

// Lobatto kernel of degree k without the (1 - x^2) factor (helperFunctions.cpp:49-92;
// degrees 0..3 are the ones hpGEM can differentiate, which caps p at 5).
inline Dual lobatto(int k, Dual x) {
    switch (k) {
        case 0: return dconst(std::sqrt(3. / 2.) * -2.);
        case 1: return std::sqrt(5. / 2.) * x * -2.;
        case 2: return std::sqrt(7. / 2.) * (5 * x * x - 1.0) / -2.;
        case 3: return std::sqrt(9. / 2.) * (7 * x * x - 3.0) * x / -2.;
    }
    throw std::invalid_argument("Lobatto kernels above degree 3 (p > 5) are not supported");
}

// Evaluate every basis function of hpGEM's default DG set of order p at x.
inline void eval_basis(int shape, int p, const double *x, std::vector<Dual> &out) {
    out.clear();
    Dual X[3];
    const ShapeInfo &s = shape_info(shape);
    for (int d = 0; d < 3; ++d) {
        X[d] = dconst(d < s.dim ? x[d] : 0.0);
        if (d < s.dim) X[d].g[d] = 1.0;
    }
    if (p < 1) throw std::invalid_argument("order p must be at least 1");
    if (p > 5) throw std::invalid_argument("order p above 5 is not supported");
    switch (shape) {
        case LINE: {
            for (int node = 0; node < 2; ++node) out.push_back((1.0 + (2 * node - 1) * X[0]) / 2.);
            for (int i = 0; i + 2 <= p; ++i)
                out.push_back((1.0 + X[0]) * (1.0 - X[0]) * lobatto(i, X[0]) / 4.);
            break;
        }
        case SQUARE: {
            for (int node = 0; node < 4; ++node) {
                double n0 = (node % 2) * 2 - 1, n1 = (node / 2) * 2 - 1;
                out.push_back((1.0 + n0 * X[0]) * (1.0 + n1 * X[1]) / 4.);
            }
            auto face0 = [&](int a, int b, int k) {  // BasisFunction2DFaceSquare_0
                double mir = a > b ? -1 : 1, ep = a + b < 3 ? -1 : 1;
                return (1.0 + ep * X[1]) * (1.0 - X[0]) * (1.0 + X[0]) * lobatto(k, mir * X[0]) / 8.;
            };
            auto face1 = [&](int a, int b, int k) {  // BasisFunction2DFaceSquare_1
                double mir = a > b ? -1 : 1, ep = a + b < 3 ? -1 : 1;
                return (1.0 + ep * X[0]) * (1.0 - X[1]) * (1.0 + X[1]) * lobatto(k, mir * X[1]) / 8.;
            };
            for (int i = 0; i + 2 <= p; ++i) {
                out.push_back(face0(0, 1, i));
                out.push_back(face0(2, 3, i));
                out.push_back(face1(0, 2, i));
                out.push_back(face1(1, 3, i));
                for (int j = 0; j + 2 <= p; ++j)
                    out.push_back((1.0 - X[0]) * (1.0 + X[0]) * (1.0 - X[1]) * (1.0 + X[1]) *
                                  lobatto(i, X[0]) * lobatto(j, X[1]) / 16.);
            }
            break;
        }
        case TRIANGLE: {
            Dual l[3] = {1.0 - X[0] - X[1], X[0], X[1]};
            for (int i = 0; i < 3; ++i) out.push_back(l[i]);
            for (int k = 0; k + 2 <= p; ++k) {
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < i; ++j)  // BasisFunction2DFaceTriangle(i, j, k)
                        out.push_back(l[i] * l[j] * lobatto(k, l[j] - l[i]));
                if (k + 3 <= p)
                    for (int j = 0; j <= k; ++j)  // BasisFunction2DInteriorTriangle(k-j, j)
                        out.push_back(l[0] * l[1] * l[2] * lobatto(k - j, l[0] - l[1]) *
                                      lobatto(j, l[1] - l[2]));
            }
            break;
        }
        case CUBE: {
            for (int node = 0; node < 8; ++node) {
                double n0 = (node % 2) * 2 - 1, n1 = ((node / 2) % 2) * 2 - 1, n2 = (node / 4) * 2 - 1;
                out.push_back((1.0 + n0 * X[0]) * (1.0 + n1 * X[1]) * (1.0 + n2 * X[2]) / 8.);
            }
            auto pos = [](int node, int axis) {
                int b = axis == 0 ? node % 2 : (axis == 1 ? (node / 2) % 2 : node / 4);
                return double(b * 2 - 1);
            };
            auto edge = [&](int axis, int a, int b, int k) {  // BasisFunction3DEdgeCube_{axis}
                double m = a < b ? 1 : -1;
                int o0 = axis == 0 ? 1 : 0, o1 = axis == 2 ? 1 : 2;
                return (1.0 - X[axis]) * (1.0 + X[axis]) * (1.0 + pos(a, o0) * X[o0]) *
                       (1.0 + pos(a, o1) * X[o1]) * lobatto(k, m * X[axis]) / 16.;
            };
            auto face = [&](int axis, int n0, int n1, int n2, int ka, int kb) {  // FaceCube_{axis}
                double fp = pos(n0, axis), ma = n0 < n1 ? 1 : -1, mb = n0 < n2 ? 1 : -1;
                int a = axis == 0 ? 1 : 0, b = axis == 2 ? 1 : 2;
                return (1.0 + fp * X[axis]) * (1.0 - X[a]) * (1.0 + X[a]) * (1.0 - X[b]) *
                       (1.0 + X[b]) * lobatto(ka, ma * X[a]) * lobatto(kb, mb * X[b]) / 32.;
            };
            auto interior = [&](int k0, int k1, int k2) {
                return (1.0 - X[0]) * (1.0 + X[0]) * (1.0 - X[1]) * (1.0 + X[1]) * (1.0 - X[2]) *
                       (1.0 + X[2]) * lobatto(k0, X[0]) * lobatto(k1, X[1]) * lobatto(k2, X[2]) / 64.;
            };
            auto faces = [&](int i, int j) {
                out.push_back(face(2, 0, 1, 2, i, j));
                out.push_back(face(1, 0, 1, 4, i, j));
                out.push_back(face(0, 0, 2, 4, i, j));
                out.push_back(face(0, 1, 3, 5, i, j));
                out.push_back(face(1, 2, 3, 6, i, j));
                out.push_back(face(2, 4, 5, 6, i, j));
            };
            for (int j = 0; j + 2 <= p; ++j) {
                for (int e = 0; e < 12; ++e) out.push_back(edge(e / 4, s.edges[e][0], s.edges[e][1], j));
                faces(j, j);
                out.push_back(interior(j, j, j));
                for (int i = 0; i < j; ++i) {
                    faces(i, j);
                    faces(j, i);
                    out.push_back(interior(i, i, j));
                    out.push_back(interior(i, j, i));
                    out.push_back(interior(j, i, i));
                    out.push_back(interior(j, j, i));
                    out.push_back(interior(j, i, j));
                    out.push_back(interior(i, j, j));
                    for (int k = 0; k < i; ++k) {
                        out.push_back(interior(i, j, k));
                        out.push_back(interior(i, k, j));
                        out.push_back(interior(j, i, k));
                        out.push_back(interior(j, k, i));
                        out.push_back(interior(k, i, j));
                        out.push_back(interior(k, j, i));
                    }
                }
            }
            break;
        }
        case TETRAHEDRON: {
            Dual l[4] = {1.0 - X[0] - X[1] - X[2], X[0], X[1], X[2]};
            for (int i = 0; i < 4; ++i) out.push_back(l[i]);
            for (int j = 0; j + 2 <= p; ++j) {
                for (int e = 0; e < 6; ++e) {  // BasisFunction3DEdgeTetrahedron: l0 l1 L(l0 - l1)
                    int a = s.edges[e][0], b = s.edges[e][1];
                    out.push_back(l[a] * l[b] * lobatto(j, l[a] - l[b]));
                }
                if (j > 0)
                    for (int f = 0; f < 4; ++f) {
                        int a = s.faces[f][0], b = s.faces[f][1], c = s.faces[f][2];
                        for (int k = 0; k + 1 <= j; ++k)
                            out.push_back(l[a] * l[b] * l[c] * lobatto(j - k - 1, l[a] - l[b]) *
                                          lobatto(k, l[b] - l[c]));
                    }
                if (j > 1)
                    for (int i = 0; i + 2 <= j; ++i)
                        for (int k = 0; (i + k) + 2 <= j; ++k)
                            out.push_back(l[0] * l[1] * l[2] * l[3] * lobatto(i, l[0] - l[1]) *
                                          lobatto(j - i - k - 2, l[1] - l[2]) * lobatto(k, l[2] - l[3]));
            }
            break;
        }
        default:
            throw std::invalid_argument("unknown shape");
    }
}

inline int basis_count(int shape, int p) {
    switch (shape) {
        case LINE: return p + 1;
        case SQUARE: return (p + 1) * (p + 1);
        case TRIANGLE: return (p + 1) * (p + 2) / 2;
        case CUBE: return (p + 1) * (p + 1) * (p + 1);
        case TETRAHEDRON: return (p + 1) * (p + 2) * (p + 3) / 6;
    }
    return 0;
}

}  // namespace hgg
