// Source terms of HpgemAPILinear for the GPU: addSourceTerm and
// addSourceTermAtBoundary (kernel/Base/HpgemAPILinear_Impl.h:437-469) add, in
// every stage and before the mass solve, the integral of phi_i g_v(x, t) over
// each element (computeIntegrandSourceTermAtElement, :201-229; ElementIntegral:
// weights times |J|) and over each boundary face into its left element (the
// application's computeIntegrandSourceTermAtFace; FaceIntegral: weights times
// |n|).  The caller gives g at quadrature points; the plan below turns those
// point values into coefficient increments with the element's mass inverse
// folded in:  k_e += sum_entries L g_entry,
//   L[r][q V + v] = sum_j Minv_e[r][v nB + j] w_q s phi_j(q),
// s = |J_e| for the element entry, |n_f| for a boundary face entry.
#pragma once

#include <cstdint>
#include <vector>

#include "setup.h"

namespace hgg {

struct SourcePlan {
    int R = 0, V = 1, nB = 0, dim = 0, nQ = 0, nQf = 0;
    bool element = false, boundary = false;
    // points at which the caller evaluates g ([points][dim]); unit normals of the
    // boundary points (FaceGeometry normal out of the left element, normalised)
    int64_t n_elem_points = 0, n_face_points = 0;
    std::vector<double> elem_xyz, face_xyz, face_normals;
    // values per evaluation time: element points first, then boundary points,
    // n_vars each ([point][v])
    int64_t values = 0;
    // distinct lifts, each stored transposed [cols][R], column c = point * V + v
    std::vector<double> table;
    std::vector<int64_t> table_off;
    std::vector<int32_t> table_cols;
    // per element with a source: its entries (element source first, then its
    // boundary faces in face order, the order in which the reference adds them)
    std::vector<int32_t> elem, ptr, lift;
    std::vector<int64_t> off;  // first value of each entry
};

// mass: the distinct element mass matrices [n][R][R] (row-major), mass_of[E] the
// one of each element.  Throws std::invalid_argument.
SourcePlan plan_sources(const StructuredProblem &P, const std::vector<double> &mass,
                        const std::vector<int32_t> &mass_of, bool element_source, bool boundary_source);

}  // namespace hgg
