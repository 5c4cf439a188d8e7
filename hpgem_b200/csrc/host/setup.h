// Host-side set-up that hpGEM performs before its time loop, restated:
// quadrature rules, Preprocessor structured meshes, face pairing, element
// geometry and the tabulations that fill an hgg_problem_desc.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "refshapes.h"

namespace hgg {

struct Rule {
    std::string name;
    int order = 0;
    int dim = 0;
    std::vector<double> points;   // [n][dim]
    std::vector<double> weights;  // [n]
    int size() const { return (int)weights.size(); }
};

// AllGaussQuadratureRules::getRule (kernel/Integration/QuadratureRules/
// AllGaussQuadratureRules.cpp:138-158): first rule of order >= `order`.
// shape 0 is the point.
Rule get_rule(int shape, int order);

struct StructuredDescription {
    std::vector<int64_t> n;
    std::vector<double> lower, upper;
    bool triangular = false;
    std::vector<bool> periodic;
};

// Parses "structured 1 <dim> / n... / lower... / upper... / triangular|rectangular / periodic..."
StructuredDescription parse_structured(const std::string &text);

struct Mesh {
    int shape = 0;
    int dim = 0;
    int64_t n_elements = 0;
    int n_vertices = 0;
    std::vector<int64_t> nodes;    // [E][nv] global node numbers
    std::vector<double> coords;    // [E][nv][dim] physical vertex coordinates
    // faces, numbered in order of first appearance
    std::vector<int64_t> face_elements;  // [F][2]
    std::vector<int32_t> face_local;     // [F][2]
    std::vector<int32_t> face_perm;      // [F][face_vertices]: right-face slot of each left-face vertex
    int64_t n_faces() const { return (int64_t)face_local.size() / 2; }
};

// StructuredReader (applications/Preprocessor/lib/hpgem.cpp:55-265) + face pairing.
Mesh structured_mesh(const StructuredDescription &d);

// Face pairing by global node sets (periodic copies of a node share its number).
void pair_faces(Mesh &m);

// A Preprocessor "mesh 2" file's text (MeshManipulator::readMesh's input) -> Mesh.
Mesh read_mesh2(const std::string &text);

// Element reference point -> physical point through the vertex map.
void reference_to_physical(const Mesh &m, int64_t e, const double *xi, double *x);

// Reference-face point -> element reference point through the local face whose
// vertices (element-local numbers) are `face_vertices`.
void face_to_element(int shape, const int *face_vertices, const double *xi_face, double *xi);

// Everything needed to fill an hgg_problem_desc for a structured mesh.
struct StructuredProblem {
    Mesh mesh;
    int order = 0, physics = 0, n_vars = 1, n_basis = 0;
    double advection[3] = {0, 0, 0};
    double c_inv = 1.0;
    Rule rule, face_rule, error_rule;
    std::vector<double> basis_values, basis_grads;  // element rule
    std::vector<double> face_tabs;                  // [tabs][nQf][nB]
    std::vector<int32_t> face_tab_index;            // [F][2]
    int n_face_tabs = 0;
    std::vector<double> jacobians;                  // [E][d][d]
    std::vector<double> normals;                    // [F][d]
    std::vector<double> error_basis;                // [nQerr][nB]
    std::vector<double> rk_a, rk_b, rk_c;
    int n_stages = 0;
};

// boundary_faces: the mesh may have faces with one element (right element -1),
// as the stored-matrix path takes; otherwise every face must have two.
StructuredProblem build_structured(const std::string &description, int order, int physics,
                                   const double *params, const std::string &tableau, bool boundary_faces = false);
StructuredProblem build_problem(Mesh mesh, int order, int physics, const double *params, const std::string &tableau,
                                bool boundary_faces = false);

bool butcher_tableau(const std::string &name, std::vector<double> &a, std::vector<double> &b,
                     std::vector<double> &c, int &stages);

// Error coefficients b_i - b*_i and order of an embedded tableau (DormandPrince.cpp:75-82,
// order 5; BogackiShampine.cpp:61-67, order 3); false for tableaux without an error estimate.
bool butcher_error_estimate(const std::string &name, std::vector<double> &error, int &order);

}  // namespace hgg
