// Reference-element operators and per-element geometry for the GPU kernels.
//
// On affine elements hpGEM's quadrature integrands (advection weak form, wave
// strong form, face fluxes) are polynomials of degree <= 2p, which the rules of
// order 2p+1 integrate exactly; the element mass matrix is |J| times the
// reference mass matrix.  So every per-element integral of hpGEM's loop
// (HpgemAPISimplified_Impl.h:625-695 followed by the mass solve :205-225) is a
// fixed reference matrix applied to the coefficients, scaled by per-element
// geometry.  The operators are built here once, in FP64, from the caller's
// tabulations:
//   Mhat    = sum_q w_q phi phi^T                    (reference mass matrix)
//   vol[c]  = Mhat^{-1} sum_q w_q dphi_c phi^T        advection:  k += ahat_c vol[c] w, ahat = J^{-1} a
//           = Mhat^{-1} sum_q w_q phi dphi_c^T        wave: derivative matrices (strong form)
//   pair(s,n) = Mhat^{-1} sum_q wf_q phi_s phi_n^T    face term with test side s, trial side n
// and per element e and local face slot:
//   advection: sigma = (a . n_e/|n_e|) |n_e| / |J_e|, the upwind mode of
//              090Advection_SelfTest.cpp:165-191 (self / neighbour / average / none)
//   wave:      nu = 0.5 n_e / |J_e|   (central flux, AcousticWave_Impl.h:289-373)
// where n_e is the outward normal of e with length = area ratio.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../../include/hpgem_b200.h"

namespace hgg {

enum FaceMode : int8_t { MODE_NONE = 0, MODE_SELF = 1, MODE_NBR = 2, MODE_AVG = 3 };

struct HostOperators {
    int shape = 0, dim = 0, order = 0, nB = 0, V = 1, physics = 0, nfl = 0;
    int64_t nE = 0;
    double c_inv = 1.0;
    // dense reference-operator form
    std::vector<double> mass_inv;   // [nB][nB]
    std::vector<double> vol;        // [dim][nB][nB]
    std::vector<double> pairs;      // [n_pairs][nB][nB]
    int n_pairs = 0;
    std::vector<int32_t> nbr;       // [E][nfl]
    std::vector<int32_t> self_pair; // [E][nfl]
    std::vector<int32_t> nbr_pair;  // [E][nfl]
    std::vector<int8_t> mode;       // [E][nfl] (advection)
    std::vector<double> elem_geo;   // advection [E][dim] ahat; wave [E][dim][dim] G = J^{-T}
    std::vector<double> face_geo;   // advection [E][nfl] sigma; wave [E][nfl][dim] nu
    std::vector<double> abs_det;    // [E]

    // tensor-product form (hypercubes, advection), valid when tensor == true
    bool tensor = false;
    int np = 0;                     // 1D modes per direction (p + 1)
    std::vector<double> D1;         // [np][np] = M1^{-1} S1
    std::vector<double> lift;       // [2][np]: M1^{-1} psi(-1), M1^{-1} psi(+1)
    int trace_pos[2] = {0, 0};      // the 1D mode that is 1 at -1 / +1 (all others vanish there)
    std::vector<int32_t> tpos;      // [nB] hpGEM index -> tensor position (x fastest)
    std::vector<double> tsign;      // [nB] hpGEM function = tsign * tensor product
    std::vector<int32_t> t_nbr;     // [E][2*dim] in tensor slot order (x-, x+, y-, y+, z-, z+)
    std::vector<int8_t> t_mode;     // [E][2*dim]
    std::vector<double> t_sigma;    // [E][2*dim]
    std::string tensor_reason;      // why the tensor form was not taken
};

// Throws std::invalid_argument / std::runtime_error with a message on bad input.
// faces = false: element data only (the stored-matrix path applies its own face
// matrices and takes meshes with boundary faces)
HostOperators build_operators(const hgg_problem_desc &desc, bool faces = true);

// small dense helpers
void invert_matrix(int n, const double *A, double *Ainv);

}  // namespace hgg
