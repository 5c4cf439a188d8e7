// HpgemAPILinear (kernel/Base/HpgemAPILinear_Impl.h) for the GPU: the stored
// element and face matrices, kept once per distinct matrix, and their folded
// form k_e = D_e w_e + sum_s N_{e,s} w_{n(e,s)} that the stage kernel applies.
#pragma once

#include <cstdint>
#include <unordered_map>
#include <vector>

#include "../../../include/hpgem_b200.h"

namespace hgg {

// Square R x R matrices, each distinct one (bit for bit) stored once.
class MatrixPool {
   public:
    explicit MatrixPool(int R = 0) : R_(R) {}
    int rows() const { return R_; }
    int size() const { return (int)(data_.size() / ((size_t)R_ * R_)); }
    const double *get(int id) const { return data_.data() + (size_t)id * R_ * R_; }
    // id of the matrix equal to m (added when new)
    int add(const double *m);

   private:
    int R_;
    std::vector<double> data_;
    std::unordered_multimap<uint64_t, int> index_;
};

// HpgemAPILinear's stored matrices of one mesh, as pool ids.
struct LinearSystem {
    int R = 0;
    int64_t E = 0, F = 0;
    MatrixPool pool;
    std::vector<int32_t> mass_id, stiffness_id;  // [E]
    std::vector<int64_t> face_elements;          // [F][2], right = -1 on a boundary face
    std::vector<int32_t> face_id;                // [F][4] blocks (LL, LR, RL, RR); -1 where absent
};

// From hpGEM's arrays (hgg_linear_desc).  Throws std::invalid_argument.
LinearSystem linear_from_desc(const hgg_linear_desc &d);

// The matrices of the reference's linear applications, from a problem's
// tabulations and geometry: advection with the integrands of
// tests/self/Basic/080AdvectionLinear_SelfTest.cpp:108-168, the wave with
// those of applications/ExampleMultipleVariableProblem/AcousticWaveLinear_Impl.h:98-284.
LinearSystem assemble_linear(const hgg_problem_desc &desc);

// Folded form.  Every element has `slots` neighbour slots (the largest count
// of neighbour blocks of any element); unused slots hold -1.
struct LinearOperators {
    int R = 0, slots = 0;
    int64_t E = 0;
    std::vector<double> table;      // [n_mats][R][R] row-major, distinct matrices
    std::vector<int32_t> self_mat;  // [E]
    std::vector<int32_t> nbr;       // [E][slots]
    std::vector<int32_t> nbr_mat;   // [E][slots]
    int n_mats() const { return R ? (int)(table.size() / ((size_t)R * R)) : 0; }
};

LinearOperators fold_linear(const LinearSystem &s);

}  // namespace hgg
