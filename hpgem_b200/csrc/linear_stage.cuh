// Runge-Kutta stage kernel of HpgemAPILinear's stored-matrix form
// (kernel/Base/HpgemAPILinear_Impl.h): per element
//   w_e = u_e + sum_j dt a_ij k_j,e                     (getLinearCombinationOfVectors)
//   k_e = D_e w_e + sum_s N_{e,s} w_{n(e,s)}            (multiplyStiffnessMatrices, :360-434,
//                                                        then solveMassMatrixEquations, :143-156,
//                                                        with M_e^{-1} folded into D and N)
// and in the final stage u_new = u + sum_j dt b_j k_j.  The distinct matrices
// are few on structured meshes, so they stay in L1/L2 while the per-element
// stage vectors stream from HBM.
#pragma once

#include <cstdint>

#include "dg_kernels.cuh"

namespace hgg {

struct LinearGeom {
    const double *table;      // [n_mats][R][R] transposed: table[m][j][i] = (matrix m)_{ij}
    const float *table_f;     // the same in FP32 (FP32-mixed form with FP32 contractions), else null
    const int32_t *self_mat;  // [E]
    const int32_t *nbr;       // [E][slots], -1: unused slot
    const int32_t *nbr_mat;   // [E][slots]
    int R, slots, epb, n_mats;
};

template <typename CT>
__device__ __forceinline__ const CT *linear_table(const LinearGeom &g);
template <>
__device__ __forceinline__ const double *linear_table<double>(const LinearGeom &g) { return g.table; }
template <>
__device__ __forceinline__ const float *linear_table<float>(const LinearGeom &g) { return g.table_f; }

// threads and dynamic shared memory of one block of `epb` elements
__host__ __device__ inline int linear_threads(int R, int epb) { return ((epb * R + 31) / 32) * 32; }
__host__ __device__ inline size_t linear_smem(int R, int slots, int epb, size_t elem) {
    return elem * (size_t)epb * R * (1 + slots);
}

// Thread (el, r) of the block produces row r of element el: the matrices are
// stored transposed, so at every column j the threads of one element read
// consecutive entries.  KT: stage-vector type; CT: contraction type.
template <typename KT, typename CT>
__global__ void __launch_bounds__(256) linear_stage(const StageIOT<KT> io, const LinearGeom g) {
    extern __shared__ __align__(16) unsigned char linear_shared[];
    const int R = g.R, S = g.slots, epb = g.epb;
    CT *W = reinterpret_cast<CT *>(linear_shared);  // [epb][R]
    CT *WN = W + (size_t)epb * R;                  // [epb][S][R]
    const int tid = threadIdx.x;
    const int64_t e0 = (int64_t)blockIdx.x * epb;
    const int el = tid / R, r = tid % R;
    const int64_t e = e0 + el;
    const bool active = el < epb && e < io.n_elements;
    double u_own = 0.0;
    if (active) {
        const int64_t idx = e * R + r;
        u_own = io.u[idx];
        double w = u_own;
        for (int j = 0; j < io.nin; ++j) w += io.cin[j] * (double)io.kin[j][idx];
        W[el * R + r] = (CT)w;
    }
    for (int k = tid; k < epb * S * R; k += blockDim.x) {
        const int l = k / (S * R), s = (k / R) % S, rr = k % R;
        const int64_t ee = e0 + l;
        double v = 0.0;
        if (ee < io.n_elements) {
            const int32_t n = g.nbr[ee * S + s];
            if (n >= 0 && n < io.n_elements) v = stage_input(io, (int64_t)n * R + rr);
            else if (n >= 0) atomicOr(io.status, 1);
        }
        WN[(size_t)(l * S + s) * R + rr] = (CT)v;
    }
    __syncthreads();
    if (!active) return;

    const CT *T = linear_table<CT>(g);
    const size_t RR = (size_t)R * R;
    CT acc = CT(0);
    int32_t m = g.self_mat[e];
    if (m >= 0 && m < g.n_mats) {
        const CT *op = T + (size_t)m * RR + r;
        const CT *w = W + el * R;
#pragma unroll 8
        for (int j = 0; j < R; ++j) acc += op[(size_t)j * R] * w[j];
    } else {
        atomicOr(io.status, 2);
    }
    for (int s = 0; s < S; ++s) {
        m = g.nbr_mat[e * S + s];
        if (m < 0) continue;
        if (m >= g.n_mats) {
            atomicOr(io.status, 2);
            continue;
        }
        const CT *op = T + (size_t)m * RR + r;
        const CT *wn = WN + (size_t)(el * S + s) * R;
#pragma unroll 8
        for (int j = 0; j < R; ++j) acc += op[(size_t)j * R] * wn[j];
    }
    stage_output(io, e * R + r, u_own, (double)acc);
}

}  // namespace hgg
