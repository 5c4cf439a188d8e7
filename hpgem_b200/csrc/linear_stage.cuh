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

// Status word bits set here: 1 a neighbour index out of range, 4 a matrix
// index out of range (2 is the bounded-wait bit of the persistent kernels).
struct LinearGeom {
    const double *table;      // [n_mats][R][R] transposed: table[m][j][i] = (matrix m)_{ij}
    const double *table_rm;   // [n_mats][R][R] row-major (the grouped kernel's copy), or null
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
        atomicOr(io.status, 4);
    }
    for (int s = 0; s < S; ++s) {
        m = g.nbr_mat[e * S + s];
        if (m < 0) continue;
        if (m >= g.n_mats) {
            atomicOr(io.status, 4);
            continue;
        }
        const CT *op = T + (size_t)m * RR + r;
        const CT *wn = WN + (size_t)(el * S + s) * R;
#pragma unroll 8
        for (int j = 0; j < R; ++j) acc += op[(size_t)j * R] * wn[j];
    }
    stage_output(io, e * R + r, u_own, (double)acc);
}

// ---------------------------------------------------------------------------
// grouped form: tiles of kLinTileN elements that share all their matrices
// ---------------------------------------------------------------------------
// On a structured mesh the elements fall into a few groups with identical
// matrices (one group on a hexahedral mesh, ten on the five-tetrahedron split),
// so a tile's stage is a dense product Out[R][64] = sum_s A_s[R][R] W_s[R][64]
// with W_s the stage inputs of the tile's elements (s = 0) or of their
// neighbours in slot s.  It runs on the FP64 tensor cores (DMMA, m8n8k4):
// 8 warps, warp w owns elements 8w..8w+7, each warp all row bands of 8.
constexpr int kLinTileN = 64;            // elements per tile
constexpr int kLinKC = 32;               // k (column) chunk staged in shared memory
constexpr int kLinRows = 64;             // output rows per pass
constexpr int kLinStride = kLinKC + 4;   // padded row stride (doubles): fragment loads conflict-free
constexpr int kLinOutStride = kLinRows + 1;
constexpr int kLinTileMinRows = 15;      // smaller elements run the row kernel

struct LinearTiles {
    const int32_t *elems;  // [n_tiles][kLinTileN] element ids, -1: padding
    const int32_t *mats;   // [n_tiles][1 + slots] the tile's matrices (-1: unused slot)
};

__device__ __forceinline__ void dmma_m8n8k4(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// One tile (256 threads).  Called by the one-problem launch (tile = blockIdx.x)
// and by the batch's persistent launch (tile = the block's index in its problem).
template <typename KT>
__device__ __forceinline__ void linear_tile_body(const StageIOT<KT> &io, const LinearGeom &g, const LinearTiles &t,
                                                 int64_t tile) {
    // A chunk [kLinRows][kLinStride] and B chunk [kLinTileN][kLinStride]; the
    // output tile [kLinTileN][kLinOutStride] reuses the same memory
    __shared__ __align__(16) double sm[(kLinRows + kLinTileN) * kLinStride];
    __shared__ int32_t tel[kLinTileN], src[kLinTileN];
    static_assert(kLinTileN * kLinOutStride <= (kLinRows + kLinTileN) * kLinStride, "output staging fits");
    double *As = sm, *Bs = sm + kLinRows * kLinStride;
    const int R = g.R, S = g.slots;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, gid = lane >> 2, tig = lane & 3;
    if (tid < kLinTileN) tel[tid] = t.elems[tile * kLinTileN + tid];
    const int passes = (R + kLinRows - 1) / kLinRows;
    for (int pass = 0; pass < passes; ++pass) {
        const int r0 = pass * kLinRows;
        const int rows = min(kLinRows, R - r0);
        double acc[8][2];
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[b][0] = acc[b][1] = 0.0;
        for (int s = 0; s <= S; ++s) {
            const int32_t m = t.mats[tile * (S + 1) + s];  // the same for the whole block
            if (m < 0) continue;
            if (m >= g.n_mats) {
                if (tid == 0) atomicOr(io.status, 4);
                continue;
            }
            __syncthreads();  // tel written; src, As, Bs free
            if (tid < kLinTileN) {
                const int32_t e = tel[tid];
                int32_t se = -1;
                if (e >= 0 && e < io.n_elements) se = s == 0 ? e : g.nbr[(int64_t)e * S + (s - 1)];
                if (se >= io.n_elements || se < -1) {
                    atomicOr(io.status, 1);
                    se = -1;
                }
                src[tid] = se;
            }
            const double *A = g.table_rm + (size_t)m * R * R;
            for (int kc = 0; kc < R; kc += kLinKC) {
                // only the fragments' extent is staged: rows up to the next band of 8,
                // columns up to the next multiple of 4 (zeros beyond R)
                const int kmax = min(kLinKC, R - kc), kw = (kmax + 3) & ~3, rw = (rows + 7) & ~7;
                __syncthreads();  // src written; the previous chunk's fragments read
                // lane = column, warp = row (no integer division; a row's columns coalesce)
                if (lane < kw) {
                    for (int r = warp; r < rw; r += 8) {
                        double v = 0.0;
                        if (r < rows && lane < kmax) v = A[(size_t)(r0 + r) * R + kc + lane];
                        As[r * kLinStride + lane] = v;
                    }
#pragma unroll
                    for (int n = warp; n < kLinTileN; n += 8) {  // eight passes: loads issue together
                        const int32_t se = src[n];
                        double v = 0.0;
                        if (se >= 0 && lane < kmax) v = stage_input_few(io, (int64_t)se * R + kc + lane);
                        Bs[n * kLinStride + lane] = v;
                    }
                }
                __syncthreads();
                for (int k4 = 0; k4 < kmax; k4 += 4) {
                    const double b = Bs[(warp * 8 + gid) * kLinStride + k4 + tig];
#pragma unroll
                    for (int band = 0; band < 8; ++band)
                        if (band * 8 < rows) dmma_m8n8k4(acc[band][0], acc[band][1],
                                                         As[(band * 8 + gid) * kLinStride + k4 + tig], b);
                }
            }
        }
        __syncthreads();  // fragments read: stage the outputs as [element][row]
        double *Os = sm;
#pragma unroll
        for (int band = 0; band < 8; ++band)
            if (band * 8 < rows) {
                const int n = warp * 8 + tig * 2;
                Os[n * kLinOutStride + band * 8 + gid] = acc[band][0];
                Os[(n + 1) * kLinOutStride + band * 8 + gid] = acc[band][1];
            }
        __syncthreads();
        for (int i = tid; i < kLinTileN * kLinRows; i += blockDim.x) {
            const int n = i / kLinRows, r = i % kLinRows;
            const int32_t e = tel[n];
            if (e < 0 || e >= io.n_elements || r >= rows) continue;
            const int64_t idx = (int64_t)e * R + r0 + r;
            stage_output(io, idx, io.u[idx], Os[n * kLinOutStride + r]);
        }
    }
}

template <typename KT>
__global__ void __launch_bounds__(256) linear_tile_stage(const StageIOT<KT> io, const LinearGeom g,
                                                          const LinearTiles t) {
    linear_tile_body<KT>(io, g, t, blockIdx.x);
}

}  // namespace hgg
