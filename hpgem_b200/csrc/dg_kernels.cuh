// Runge-Kutta stage kernels of the explicit DG step (sm_100a, FP64).
//
// One launch = one Runge-Kutta stage of hpGEM's computeOneTimeStep
// (kernel/Base/HpgemAPISimplified_Impl.h:788-820) for every element:
//   w      = u + sum_j dt a_ij k_j                  (getLinearCombinationOfVectors, :599-620)
//   k_i    = M^{-1} [ volume(w) + sum_faces flux ]  (computeRightHandSide :625-695 +
//                                                    solveMassMatrixEquations :205-225)
//   last stage only: u_new = u + sum_j dt b_j k_j    (scaleAndAddVector, :707-717, :812-816)
// Each element gathers its own faces (element-centric, as hpGEM evaluates
// every internal face once per side, :662-668): no atomics, deterministic.
// The mass solve is folded into the reference operators (operators.h).
//
// Two kernel families:
//   tensor_stage  hypercube advection, sum-factorised: the default H1 basis
//                 is a signed tensor product of 1D hierarchical functions, so
//                 the volume term is one 1D matrix per axis and every face
//                 term is a 1D lift times a single-mode trace.
//   dense_stage   any shape / physics: dense reference operators per element.
#pragma once

#include <cstdint>
#include <type_traits>

namespace hgg {

constexpr int kMaxStages = 8;

// Linear combination inputs and the fused final update of one stage.
// Inputs and outputs of one stage launch.  KT is the storage type of the
// stage vectors: double in the FP64 form, float in the FP32-mixed form (the
// solution and the Runge-Kutta accumulation stay FP64 in both).
template <typename KT>
struct StageIOT {
    const double *u;                 // current solution
    const KT *kin[kMaxStages];       // stage vectors entering the stage input
    double cin[kMaxStages];          // their coefficients dt * a_ij
    int nin;
    KT *kout;                        // this stage's derivative (nullptr: not stored)
    double *unew;                    // final stage: new solution (nullptr otherwise)
    const KT *kfin[kMaxStages];      // earlier stage vectors of the final update
    double bfin[kMaxStages];         // their weights dt * b_j
    int nfin;
    double blast;                    // dt * b_S for the derivative computed in this stage
    int64_t n_elements;
    int *status;                     // device status word, bit 0: bad neighbour index
    // The grouped wave kernel with a tableau whose every stage input has one earlier
    // vector, the previous one (explicit RK4, midpoint): the stage input was formed by
    // the previous stage (win, else null), and this stage forms the next one
    // (wnext = u + wcoef k, else null), so the gathers read one vector instead of two.
    const double *win;
    double *wnext;
    double wcoef;
};
using StageIO = StageIOT<double>;

// stage input u + sum_j cin_j k_j of entry idx, formed in FP64
template <typename KT>
__device__ __forceinline__ double stage_input(const StageIOT<KT> &io, int64_t idx) {
    double w = io.u[idx];
#pragma unroll 1
    for (int j = 0; j < io.nin; ++j) w += io.cin[j] * (double)io.kin[j][idx];
    return w;
}

// the same for the common case of at most one stage vector in the input (the explicit
// RK4, midpoint and Heun tableaux), without a loop the compiler cannot unroll
template <typename KT>
__device__ __forceinline__ double stage_input_few(const StageIOT<KT> &io, int64_t idx) {
    if (io.win) return io.win[idx];  // the same value, formed by the previous stage
    if (io.nin == 0) return io.u[idx];
    if (io.nin == 1) return io.u[idx] + io.cin[0] * (double)io.kin[0][idx];
    return stage_input(io, idx);
}

// this stage's derivative k of entry idx (stored as KT) and, in the final stage,
// the new solution u + sum_j bfin_j k_j + blast k accumulated in FP64
template <typename KT>
__device__ __forceinline__ void stage_output(const StageIOT<KT> &io, int64_t idx, double u, double k) {
    if (io.kout) io.kout[idx] = (KT)k;
    if (io.unew) {
        double r = u;
#pragma unroll 1
        for (int j = 0; j < io.nfin; ++j) r += io.bfin[j] * (double)io.kfin[j][idx];
        r += io.blast * k;
        io.unew[idx] = r;
    }
}

// stage_output with the final update's loop unrolled (predicated on nfin, same
// summation order), so its loads issue together
template <typename KT>
__device__ __forceinline__ void stage_output_few(const StageIOT<KT> &io, int64_t idx, double u, double k) {
    if (io.kout) io.kout[idx] = (KT)k;
    if (io.wnext) io.wnext[idx] = u + io.wcoef * (double)(KT)k;  // as stage_input_few forms it
    if (io.unew) {
        double r = u;
#pragma unroll
        for (int j = 0; j < kMaxStages; ++j)
            if (j < io.nfin) r += io.bfin[j] * (double)io.kfin[j][idx];
        r += io.blast * k;
        io.unew[idx] = r;
    }
}

// ---------------------------------------------------------------------------
// sum-factorised hypercube advection
// ---------------------------------------------------------------------------
template <int P, int DIM>
struct TensorConsts {
    static constexpr int NP = P + 1;
    static constexpr int NB = DIM == 2 ? NP * NP : NP * NP * NP;
    static constexpr int NF = DIM == 2 ? NP : NP * NP;
    static constexpr int NS = 2 * DIM;
    double D1[NP * NP];
    double lift[2 * NP];
    int trace_pos[2];
    short tpos[NB];    // hpGEM index -> tensor position (x fastest)
    short tinv[NB];    // tensor position -> hpGEM index
    double tsign[NB];  // sign of hpGEM function i relative to its tensor product
};

struct TensorGeom {
    const double *ahat;    // [E][DIM]  J^{-1} a
    const int32_t *nbr;    // [E][2*DIM] slots x-, x+, y-, y+, z-, z+
    const int8_t *mode;    // [E][2*DIM]
    const double *sigma;   // [E][2*DIM]
};

// One block's work: elements [block * EPB, block * EPB + EPB).  Called by the
// one-shot launch (block = blockIdx.x) and by the grouped launch of many
// problems (block = the block's index inside its problem).
template <typename KT, int P, int DIM, int EPB>
__device__ __forceinline__ void tensor_stage_body(const StageIOT<KT> &io, const TensorGeom &geo,
                                                  const TensorConsts<P, DIM> &tc, int64_t block) {
    using TC = TensorConsts<P, DIM>;
    using CT = KT;  // contraction type
    constexpr int NP = TC::NP, NB = TC::NB, NF = TC::NF, NS = TC::NS;
    __shared__ CT W[EPB][NB];
    __shared__ CT TR[EPB][NS][NF];
    // the small tables live in shared memory: indexing kernel parameters with a
    // thread-dependent index would serialise the warp on the constant cache
    __shared__ CT sD1[NP * NP], slift[2 * NP], ssign[NB];
    __shared__ short spos[NB], sinv[NB];

    const int tid = threadIdx.x;
    for (int i = tid; i < NB; i += EPB * NB) {
        spos[i] = tc.tpos[i];
        sinv[i] = tc.tinv[i];
        ssign[i] = (CT)tc.tsign[i];
    }
    if (tid < NP * NP) sD1[tid] = (CT)tc.D1[tid];
    if (tid < 2 * NP) slift[tid] = (CT)tc.lift[tid];
    __syncthreads();

    const int el = tid / NB;
    const int t = tid % NB;  // hpGEM basis index of this thread's DoF
    const int64_t e0 = block * EPB;
    const int64_t e = e0 + el;
    const bool active = e < io.n_elements;

    double u_own = 0.0;
    if (active) {
        const int64_t idx = e * NB + t;
        u_own = io.u[idx];
        double w = u_own;
        for (int j = 0; j < io.nin; ++j) w += io.cin[j] * (double)io.kin[j][idx];
        W[el][spos[t]] = ssign[t] * (CT)w;
    }
    __syncthreads();

    // flux traces, already multiplied by sigma, per element slot
    for (int i = tid; i < EPB * NS * NF; i += EPB * NB) {
        const int l = i / (NS * NF);
        const int s = (i / NF) % NS;
        const int m = i % NF;
        const int64_t ee = e0 + l;
        CT val = CT(0);
        if (ee < io.n_elements) {
            const int axis = s >> 1, side = s & 1;
            const int8_t mode = geo.mode[ee * NS + s];
            // tangential coordinates of trace entry m
            int c[3];
            if (DIM == 2) {
                c[1 - axis] = m;
            } else {
                const int a0 = m % NP, a1 = m / NP;
                if (axis == 0) { c[1] = a0; c[2] = a1; }
                else if (axis == 1) { c[0] = a0; c[2] = a1; }
                else { c[0] = a0; c[1] = a1; }
            }
            CT tself = CT(0), tnbr = CT(0);
            if (mode == 1 || mode == 3) {
                c[axis] = tc.trace_pos[side];
                int pos = c[0] + NP * c[1] + (DIM == 3 ? NP * NP * c[2] : 0);
                tself = W[l][pos];
            }
            if (mode == 2 || mode == 3) {
                const int32_t n = geo.nbr[ee * NS + s];
                if (n >= 0 && n < io.n_elements) {
                    c[axis] = tc.trace_pos[1 - side];
                    int pos = c[0] + NP * c[1] + (DIM == 3 ? NP * NP * c[2] : 0);
                    const int hi = sinv[pos];
                    tnbr = ssign[hi] * (CT)stage_input(io, (int64_t)n * NB + hi);
                } else {
                    atomicOr(io.status, 1);
                }
            }
            const CT sg = (CT)geo.sigma[ee * NS + s];
            val = mode == 1 ? sg * tself : (mode == 2 ? sg * tnbr : (mode == 3 ? CT(0.5) * sg * (tself + tnbr) : CT(0)));
        }
        TR[l][s][m] = val;
    }
    __syncthreads();

    if (!active) return;
    const int pos = spos[t];
    int a[3];
    a[0] = pos % NP;
    a[1] = (pos / NP) % NP;
    a[2] = DIM == 3 ? pos / (NP * NP) : 0;
    CT acc = CT(0);
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
        const CT ah = (CT)geo.ahat[e * DIM + c];
        const int stride = c == 0 ? 1 : (c == 1 ? NP : NP * NP);
        const int base = pos - a[c] * stride;
        CT s = CT(0);
#pragma unroll
        for (int b = 0; b < NP; ++b) s += sD1[a[c] * NP + b] * W[el][base + b * stride];
        acc += ah * s;
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int axis = s >> 1, side = s & 1;
        int m;
        if (DIM == 2) m = a[1 - axis];
        else m = axis == 0 ? a[1] + NP * a[2] : (axis == 1 ? a[0] + NP * a[2] : a[0] + NP * a[1]);
        acc -= slift[side * NP + a[axis]] * TR[el][s][m];
    }
    stage_output(io, e * NB + t, u_own, (double)(ssign[t] * acc));
}

template <typename KT, int P, int DIM, int EPB>
__global__ void __launch_bounds__(EPB *TensorConsts<P, DIM>::NB)
    tensor_stage(const StageIOT<KT> io, const TensorGeom geo, const TensorConsts<P, DIM> tc) {
    tensor_stage_body<KT, P, DIM, EPB>(io, geo, tc, blockIdx.x);
}

// ---------------------------------------------------------------------------
// dense reference operators, any shape and physics
// ---------------------------------------------------------------------------
// Dense reference operators of one problem, in FP64 and (FP32-mixed form) FP32;
// the geometry is FP64 in both forms.
struct DenseGeom {
    const double *vol;         // [DIM][NB][NB], transposed: vol[c][j][i] = (Mhat^{-1} K_c)_{ij}
    const double *pairs;       // [n_pairs][NB][NB], transposed the same way
    const float *vol_f;        // the same in FP32 (FP32-mixed form only, else null)
    const float *pairs_f;
    const int32_t *nbr;        // [E][NFL]
    const int32_t *self_pair;  // [E][NFL]
    const int32_t *nbr_pair;   // [E][NFL]
    const int8_t *mode;        // [E][NFL] advection
    const double *elem_geo;    // advection [E][DIM]; wave [E][DIM][DIM]
    const double *face_geo;    // advection [E][NFL]; wave [E][NFL][DIM]
    double inv_cinv;           // 1 / c_inv (wave)
    double upwind_c;           // wave: 0 for the central flux, c = 1 / sqrt(c_inv) for the upwind flux
    int nB;
    int epb;                   // elements per block
};

// Contraction type of the dense kernel: FP64 in the FP64 form; in the FP32-mixed
// form FP32 up to kMixedFp32MaxBasis basis functions and FP64 above, where the
// operators Mhat^{-1} K (the mass inverse folded in) grow large with cancelling
// entries and FP32 contractions would cost the mixed form its accuracy target
// (observed: triangles at p = 5, 21 functions, 1.0e-6 L2 distance to FP64 after
// 100 steps in FP32 contractions).  The stage vectors stay FP32 either way.
constexpr int kMixedFp32MaxBasis = 20;
template <typename KT, int NB>
using DenseCT = std::conditional_t<std::is_same_v<KT, float> && NB <= kMixedFp32MaxBasis, float, double>;

template <typename CT>
__device__ __forceinline__ const CT *dense_vol(const DenseGeom &g);
template <>
__device__ __forceinline__ const double *dense_vol<double>(const DenseGeom &g) { return g.vol; }
template <>
__device__ __forceinline__ const float *dense_vol<float>(const DenseGeom &g) { return g.vol_f; }
template <typename CT>
__device__ __forceinline__ const CT *dense_pairs(const DenseGeom &g);
template <>
__device__ __forceinline__ const double *dense_pairs<double>(const DenseGeom &g) { return g.pairs; }
template <>
__device__ __forceinline__ const float *dense_pairs<float>(const DenseGeom &g) { return g.pairs_f; }

// One block's work: elements [block * epb, block * epb + epb) (see tensor_stage_body).
// Thread (el, r) produces output row r of element el (advection, and the wave in
// one dimension).  The operators are stored transposed, so at every column j the
// threads of a warp read consecutive rows' entries: one or two sectors per warp
// instead of one per thread.  NB (basis functions) is a compile-time constant, so
// the row loops unroll and the index arithmetic needs no runtime division.  KT is
// the stage vectors' type and the contraction type (see StageIOT).
template <typename KT, int DIM, int NFL, int WAVE, int NB>
__device__ __forceinline__ void dense_stage_body(const StageIOT<KT> &io, const DenseGeom &g, int64_t block) {
    static_assert(!(WAVE && DIM >= 2), "the wave in 2D and 3D runs wave_stage_body");
    using CT = DenseCT<KT, NB>;
    const CT *gvol = dense_vol<CT>(g), *gpairs = dense_pairs<CT>(g);
    constexpr int V = WAVE ? DIM + 1 : 1;
    constexpr int nB = NB, R = V * NB;
    extern __shared__ __align__(16) unsigned char dense_shared[];
    const int epb = g.epb;
    CT *W = reinterpret_cast<CT *>(dense_shared);  // [epb][R]
    CT *WN = W + (size_t)epb * R;                 // [epb][NFL][R]
    const int tid = threadIdx.x;
    const int64_t e0 = block * epb;

    const int el = tid / R, r = tid % R;
    const int64_t e = e0 + el;
    const bool active = el < epb && e < io.n_elements;
    double u_own = 0.0;
    if (active) {
        const int64_t idx = e * R + r;
        u_own = io.u[idx];
        W[el * R + r] = (CT)stage_input_few(io, idx);
    }
#pragma unroll 4
    for (int i = tid; i < epb * NFL * R; i += blockDim.x) {
        const int l = i / (NFL * R), f = (i / R) % NFL, rr = i % R;
        const int64_t ee = e0 + l;
        double v = 0.0;
        if (ee < io.n_elements && !(WAVE == 0 && g.mode[ee * NFL + f] == 1)) {
            const int32_t n = g.nbr[ee * NFL + f];
            if (n >= 0 && n < io.n_elements) v = stage_input_few(io, (int64_t)n * R + rr);
            else atomicOr(io.status, 1);
        }
        WN[(size_t)(l * NFL + f) * R + rr] = (CT)v;
    }
    __syncthreads();
    if (!active) return;

    const CT *w = W + el * R;
    const CT *wn = WN + (size_t)el * NFL * R;
    CT acc = CT(0);
    if (!WAVE) {
        const int i = r;
        for (int c = 0; c < DIM; ++c) {
            const CT *op = gvol + (size_t)c * nB * nB + i;
            CT s = CT(0);
#pragma unroll
            for (int j = 0; j < nB; ++j) s += op[(size_t)j * nB] * w[j];
            acc += (CT)g.elem_geo[e * DIM + c] * s;
        }
        for (int f = 0; f < NFL; ++f) {
            const int8_t mode = g.mode[e * NFL + f];
            const CT sg = (CT)g.face_geo[e * NFL + f];
            CT ts = CT(0), tn = CT(0);
            if (mode == 1 || mode == 3) {
                const CT *op = gpairs + (size_t)g.self_pair[e * NFL + f] * nB * nB + i;
#pragma unroll
                for (int j = 0; j < nB; ++j) ts += op[(size_t)j * nB] * w[j];
            }
            if (mode == 2 || mode == 3) {
                const CT *op = gpairs + (size_t)g.nbr_pair[e * NFL + f] * nB * nB + i;
#pragma unroll
                for (int j = 0; j < nB; ++j) tn += op[(size_t)j * nB] * wn[f * R + j];
            }
            acc -= mode == 1 ? sg * ts : (mode == 2 ? sg * tn : (mode == 3 ? CT(0.5) * sg * (ts + tn) : CT(0)));
        }
    } else {
        // the wave in one dimension: G and the normal are scalars
        const int v = r / nB, i = r % nB;
        const CT G = (CT)g.elem_geo[e];
        const CT cu = (CT)g.upwind_c;
        if (v == 0) {
            const CT *op = gvol + i;
            CT s = CT(0);
#pragma unroll
            for (int j = 0; j < nB; ++j) s += op[(size_t)j * nB] * w[nB + j];
            acc += G * s;
            for (int f = 0; f < NFL; ++f) {
                const CT nu = (CT)g.face_geo[(size_t)e * NFL + f];
                const CT *ops = gpairs + (size_t)g.self_pair[e * NFL + f] * nB * nB + i;
                const CT *opn = gpairs + (size_t)g.nbr_pair[e * NFL + f] * nB * nB + i;
                CT t = CT(0);
#pragma unroll
                for (int j = 0; j < nB; ++j) t += ops[(size_t)j * nB] * w[nB + j] - opn[(size_t)j * nB] * wn[f * R + nB + j];
                acc -= nu * t;
                if (cu != CT(0)) {  // upwind: c |nu| times the lifted pressure jump
                    CT b = CT(0);
#pragma unroll
                    for (int j = 0; j < nB; ++j) b += ops[(size_t)j * nB] * w[j] - opn[(size_t)j * nB] * wn[f * R + j];
                    acc -= cu * (nu < CT(0) ? -nu : nu) * b;
                }
            }
        } else {
            // k_s = (1/cInv) [ G vol q - face jumps of q ]
            const CT *op = gvol + i;
            CT s = CT(0);
#pragma unroll
            for (int j = 0; j < nB; ++j) s += op[(size_t)j * nB] * w[j];
            acc += G * s;
            CT up = CT(0);
            for (int f = 0; f < NFL; ++f) {
                const CT nud = (CT)g.face_geo[(size_t)e * NFL + f];
                const CT *ops = gpairs + (size_t)g.self_pair[e * NFL + f] * nB * nB + i;
                const CT *opn = gpairs + (size_t)g.nbr_pair[e * NFL + f] * nB * nB + i;
                CT t = CT(0);
#pragma unroll
                for (int j = 0; j < nB; ++j) t += ops[(size_t)j * nB] * w[j] - opn[(size_t)j * nB] * wn[f * R + j];
                acc -= nud * t;
                if (cu != CT(0)) {  // upwind: c |nu| times the lifted velocity jump (one component)
                    CT b = CT(0);
#pragma unroll
                    for (int j = 0; j < nB; ++j)
                        b += ops[(size_t)j * nB] * w[nB + j] - opn[(size_t)j * nB] * wn[f * R + nB + j];
                    up += cu * (nud < CT(0) ? -nud : nud) * b;
                }
            }
            acc *= (CT)g.inv_cinv;
            acc -= up;
        }
    }
    stage_output(io, e * R + r, u_own, (double)acc);
}

// Acoustic wave in 2D and 3D: thread (el, i) produces row i of all DIM + 1
// fields of element el.  The velocity rows of one basis row share the
// pressure contractions (vol_c q and the face brackets S_f q - N_f q_n), so
// they are formed once per row instead of once per velocity component; the
// pressure row uses t_c = sum_d G[d][c] s_d and the normal jumps n . s of both
// sides, formed once per element and column.
template <typename KT, int DIM, int NFL, int NB>
__device__ __forceinline__ void wave_stage_body(const StageIOT<KT> &io, const DenseGeom &g, int64_t block) {
    using CT = DenseCT<KT, NB>;
    const CT *gvol = dense_vol<CT>(g), *gpairs = dense_pairs<CT>(g);
    constexpr int V = DIM + 1, R = V * NB, NX = DIM + 2 * NFL;
    extern __shared__ __align__(16) unsigned char dense_shared[];
    const int epb = g.epb;
    CT *W = reinterpret_cast<CT *>(dense_shared);  // [epb][R]
    CT *WN = W + (size_t)epb * R;                 // [epb][NFL][R]
    CT *X = WN + (size_t)epb * NFL * R;           // [epb][NX][NB]: t_c, then n . s self, then n . s neighbour
    const int tid = threadIdx.x;
    const int64_t e0 = block * epb;
    const int el = tid / NB, i = tid % NB;
    const int64_t e = e0 + el;
    const bool active = el < epb && e < io.n_elements;

    double u_own[V];
    if (active) {
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int64_t idx = e * R + v * NB + i;
            u_own[v] = io.u[idx];
            W[el * R + v * NB + i] = (CT)stage_input_few(io, idx);
        }
    }
#pragma unroll 4
    for (int k = tid; k < epb * NFL * R; k += blockDim.x) {
        const int l = k / (NFL * R), f = (k / R) % NFL, rr = k % R;
        const int64_t ee = e0 + l;
        double v = 0.0;
        if (ee < io.n_elements) {
            const int32_t n = g.nbr[ee * NFL + f];
            if (n >= 0 && n < io.n_elements) v = stage_input_few(io, (int64_t)n * R + rr);
            else atomicOr(io.status, 1);
        }
        WN[(size_t)(l * NFL + f) * R + rr] = (CT)v;
    }
    __syncthreads();
    const CT *w = W + el * R;
    const CT *wn = WN + (size_t)el * NFL * R;
    CT *x = X + (size_t)el * NX * NB;
    if (active) {
        const double *G = g.elem_geo + e * DIM * DIM;  // G[d][c] = (J^{-T})_{dc}
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
            CT t = CT(0);
#pragma unroll
            for (int d = 0; d < DIM; ++d) t += (CT)G[d * DIM + c] * w[(d + 1) * NB + i];
            x[c * NB + i] = t;
        }
#pragma unroll
        for (int f = 0; f < NFL; ++f) {
            const double *nu = g.face_geo + ((size_t)e * NFL + f) * DIM;
            CT a = CT(0), b = CT(0);
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                a += (CT)nu[d] * w[(d + 1) * NB + i];
                b += (CT)nu[d] * wn[f * R + (d + 1) * NB + i];
            }
            x[(DIM + f) * NB + i] = a;
            x[(DIM + NFL + f) * NB + i] = b;
        }
    }
    __syncthreads();
    if (!active) return;

    CT P = CT(0), A[DIM], B[NFL], SP[NFL];
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
        const CT *op = gvol + (size_t)c * NB * NB + i;
        CT sp = CT(0), sa = CT(0);
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            const CT o = op[(size_t)j * NB];
            sp += o * x[c * NB + j];
            sa += o * w[j];
        }
        P += sp;
        A[c] = sa;
    }
#pragma unroll
    for (int f = 0; f < NFL; ++f) {
        const CT *ops = gpairs + (size_t)g.self_pair[e * NFL + f] * NB * NB + i;
        const CT *opn = gpairs + (size_t)g.nbr_pair[e * NFL + f] * NB * NB + i;
        const CT *js = x + (DIM + f) * NB, *jn = x + (DIM + NFL + f) * NB;
        CT sp = CT(0), sb = CT(0);
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            const CT os = ops[(size_t)j * NB], on = opn[(size_t)j * NB];
            sp += os * js[j] - on * jn[j];
            sb += os * w[j] - on * wn[f * R + j];
        }
        P -= sp;
        B[f] = sb;
        SP[f] = sp;
    }
    const CT cu = (CT)g.upwind_c;
    CT nrm[NFL];
    if (cu != CT(0)) {
        // upwind: the pressure row gets c |nu| times the lifted pressure jump, velocity
        // component d gets c (nu_d / |nu|) times the lifted normal velocity jump (nu . s)
#pragma unroll
        for (int f = 0; f < NFL; ++f) {
            const double *nu = g.face_geo + ((size_t)e * NFL + f) * DIM;
            double q = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) q += nu[d] * nu[d];
            nrm[f] = (CT)sqrt(q);
            P -= cu * nrm[f] * B[f];
        }
    }
    stage_output(io, e * R + i, u_own[0], (double)P);
    const double *G = g.elem_geo + e * DIM * DIM;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        CT acc = CT(0);
#pragma unroll
        for (int c = 0; c < DIM; ++c) acc += (CT)G[d * DIM + c] * A[c];
#pragma unroll
        for (int f = 0; f < NFL; ++f) acc -= (CT)g.face_geo[((size_t)e * NFL + f) * DIM + d] * B[f];
        acc *= (CT)g.inv_cinv;
        if (cu != CT(0))
#pragma unroll
            for (int f = 0; f < NFL; ++f) acc -= cu * ((CT)g.face_geo[((size_t)e * NFL + f) * DIM + d] / nrm[f]) * SP[f];
        stage_output(io, e * R + (d + 1) * NB + i, u_own[d + 1], (double)acc);
    }
}

// threads and dynamic shared memory of one dense-kernel block of `epb` elements
// (elem: bytes of the contraction type)
__host__ __device__ inline int dense_rows(int dim, int wave, int nb) { return wave && dim >= 2 ? nb : (wave ? dim + 1 : 1) * nb; }
__host__ __device__ inline int dense_threads(int dim, int wave, int nb, int epb) {
    return ((epb * dense_rows(dim, wave, nb) + 31) / 32) * 32;
}
__host__ __device__ inline size_t dense_smem(int dim, int nfl, int wave, int nb, int epb, size_t elem = 8) {
    const int R = (wave ? dim + 1 : 1) * nb;
    size_t d = (size_t)epb * R * (1 + nfl);
    if (wave && dim >= 2) d += (size_t)epb * (dim + 2 * nfl) * nb;
    return elem * d;
}

template <typename KT, int DIM, int NFL, int WAVE, int NB>
__device__ __forceinline__ void dense_any_body(const StageIOT<KT> &io, const DenseGeom &g, int64_t block) {
    if constexpr (WAVE && DIM >= 2) wave_stage_body<KT, DIM, NFL, NB>(io, g, block);
    else dense_stage_body<KT, DIM, NFL, WAVE, NB>(io, g, block);
}

template <typename KT, int DIM, int NFL, int WAVE, int NB>
__global__ void __launch_bounds__(256) dense_stage(const StageIOT<KT> io, const DenseGeom g) {
    dense_any_body<KT, DIM, NFL, WAVE, NB>(io, g, blockIdx.x);
}

// ---------------------------------------------------------------------------
// grouped dense kernels: lane = element, warp = basis row
// ---------------------------------------------------------------------------
// The elements of a structured mesh fall into a few groups with the same
// operator signature (the pair operators of every face; for the wave, whose
// per-element work is the largest).  A
// tile holds group_tile_elems(NB) elements of one group (32, or 16 above 24 basis
// functions); a block of that many threads per basis row runs it with lane =
// element and warp = output row (two rows above 24), so every operator
// entry a warp reads is the same address for all its lanes (one broadcast
// instead of one sector per element), and the per-element staging arrays have
// odd strides (in elements of CT), so the lanes' reads hit distinct banks.  The
// stage inputs are staged and the outputs written through shared memory, both
// coalesced along an element's coefficients.
constexpr int kGroupTile = 32;  // the largest tile (elements)
// elements per tile: 32 (a warp of lanes per basis row), 16 above 24 basis functions (a
// warp then covers two basis rows of 16 elements; the block stays within 1024 threads)
__host__ __device__ constexpr int group_tile_elems(int nb) { return nb <= 24 ? 32 : 16; }

// odd stride (in CT elements) at least n
__host__ __device__ constexpr int odd_stride(int n) { return n | 1; }

// Per-tile set-up: the tile's element ids, its
// operator signature (the same for all its elements: taken from the first) and
// every element's geometry record, staged coalesced; lanes then read their
// element's record from shared memory (odd stride) instead of 32 scattered
// global addresses per load.
template <int NFL>
struct GroupTileInfo {
    int32_t tel[kGroupTile];
    int32_t self_pair[NFL], nbr_pair[NFL];
    int8_t mode[NFL];
};

template <int NFL, int TE>
__device__ __forceinline__ void group_tile_setup(const DenseGeom &g, const int32_t *tiles, int64_t tile,
                                                 int64_t n_elements, GroupTileInfo<NFL> &ti) {
    const int tid = threadIdx.x;
    if (tid < TE) ti.tel[tid] = tiles[tile * TE + tid];
    if (tid < NFL) {
        const int32_t e0 = tiles[tile * TE];  // the first slot of a tile is never padding
        const bool ok = e0 >= 0 && e0 < n_elements;
        ti.self_pair[tid] = ok ? g.self_pair[(int64_t)e0 * NFL + tid] : 0;
        ti.nbr_pair[tid] = ok ? g.nbr_pair[(int64_t)e0 * NFL + tid] : 0;
        ti.mode[tid] = ok ? g.mode[(int64_t)e0 * NFL + tid] : 0;
    }
    __syncthreads();
}

// Acoustic wave in 2D and 3D (the arithmetic of wave_stage_body).  Shared:
// W [tile][R] stage inputs (then the outputs), WN [tile][NFL][2 NB] neighbour
// pressure and n . s_n per face, X [tile][DIM + NFL][NB] t_c and n . s, GE
// [tile][DIM^2 + NFL DIM] geometry (FP64).
template <int DIM, int NFL, int NB>
struct WaveGroupShape {
    static constexpr int TE = group_tile_elems(NB);
    static constexpr int V = DIM + 1, R = V * NB, EG = DIM * DIM, FG = NFL * DIM;
    static constexpr int WS = odd_stride(R), WNS = odd_stride(NFL * 2 * NB), XS = odd_stride((DIM + NFL) * NB);
    static constexpr int GS = odd_stride(EG + FG);
    static constexpr int OPS = (DIM + 2 * NFL) * NB * NB;
    static constexpr int ELEMS = TE * (WS + WNS + XS) + OPS;  // CT elements after GE (doubles)
    static constexpr int GEO = TE * GS;
};

template <typename KT, int DIM, int NFL, int NB>
__device__ __forceinline__ void wave_group_body(const StageIOT<KT> &io, const DenseGeom &g, const int32_t *tiles,
                                                int64_t tile) {
    using CT = DenseCT<KT, NB>;
    using SH = WaveGroupShape<DIM, NFL, NB>;
    constexpr int R = SH::R, WS = SH::WS, WNS = SH::WNS, XS = SH::XS, GS = SH::GS, EG = SH::EG, TE = SH::TE;
    extern __shared__ __align__(16) unsigned char dense_shared[];
    double *GE = reinterpret_cast<double *>(dense_shared);
    CT *W = reinterpret_cast<CT *>(GE + SH::GEO);
    CT *WN = W + TE * WS;
    CT *X = WN + TE * WNS;
    CT *OP = X + TE * XS;  // [DIM + 2 NFL][NB][NB]
    __shared__ GroupTileInfo<NFL> ti;
    const int tid = threadIdx.x, el = tid & (TE - 1), i = tid / TE;
    group_tile_setup<NFL, TE>(g, tiles, tile, io.n_elements, ti);
    constexpr int T = TE * NB;  // the block's threads (see the gathers below)
    {
        constexpr int Q = EG + NFL * DIM, NG = (TE * Q + T - 1) / T;
#pragma unroll
        for (int it = 0; it < NG; ++it) {
            const int k = tid + it * T;
            if (k < TE * Q) {
                const int l = k / Q, q = k % Q;
                const int32_t e = ti.tel[l];
                double v = 0.0;
                if (e >= 0 && e < io.n_elements)
                    v = q < EG ? g.elem_geo[(int64_t)e * EG + q] : g.face_geo[(int64_t)e * (NFL * DIM) + q - EG];
                GE[l * GS + q] = v;
            }
        }
        constexpr int NN = NB * NB, TOT = (DIM + 2 * NFL) * NN, NO = (TOT + T - 1) / T;
        const CT *gvol = dense_vol<CT>(g), *gpairs = dense_pairs<CT>(g);
#pragma unroll 1
        for (int it = 0; it < NO; ++it) {
            const int k = tid + it * T;
            if (k < TOT) {
                const int m = k / NN, q = k % NN;
                CT v;
                if (m < DIM) v = gvol[(size_t)m * NN + q];
                else {
                    const int f = (m - DIM) >> 1;
                    const int32_t pair = ((m - DIM) & 1) ? ti.nbr_pair[f] : ti.self_pair[f];
                    v = gpairs[(size_t)pair * NN + q];
                }
                OP[k] = v;
            }
        }
    }
    // The block has exactly T = TE * NB threads, so every staging loop takes a fixed
    // number of passes per thread (the gathers below: V and NFL): unrolled, every pass's
    // loads are issued before the first is used.
#pragma unroll
    for (int it = 0; it < SH::V; ++it) {
        const int k = tid + it * T;
        const int l = k / R, rr = k % R;
        const int32_t ee = ti.tel[l];
        double v = 0.0;
        if (ee >= 0 && ee < io.n_elements) v = stage_input_few(io, (int64_t)ee * R + rr);
        W[l * WS + rr] = (CT)v;
    }
    // neighbour indices of every pass first, then their values
    int32_t nbi[NFL];
#pragma unroll
    for (int it = 0; it < NFL; ++it) {
        const int k = tid + it * T;
        const int l = k / (NFL * NB), f = (k / NB) % NFL;
        const int32_t ee = ti.tel[l];
        nbi[it] = -2;  // padding element
        if (ee >= 0 && ee < io.n_elements) {
            const int32_t n = g.nbr[(int64_t)ee * NFL + f];
            nbi[it] = n >= 0 && n < io.n_elements ? n : -1;
        }
    }
    __syncthreads();  // GE staged (the neighbour loop reads the normals)
    // neighbours: pressure and n . s (this element's normal) per face and basis row
#pragma unroll
    for (int it = 0; it < NFL; ++it) {
        const int k = tid + it * T;
        const int l = k / (NFL * NB), f = (k / NB) % NFL, j = k % NB;
        const int32_t n = nbi[it];
        double pn = 0.0, jn = 0.0;
        if (n >= 0) {
            const double *nu = GE + l * GS + EG + f * DIM;
            pn = stage_input_few(io, (int64_t)n * R + j);
#pragma unroll
            for (int d = 0; d < DIM; ++d)
                jn += nu[d] * (double)(CT)stage_input_few(io, (int64_t)n * R + (d + 1) * NB + j);
        } else if (n == -1) {
            atomicOr(io.status, 1);
        }
        WN[l * WNS + f * 2 * NB + j] = (CT)pn;
        WN[l * WNS + f * 2 * NB + NB + j] = (CT)jn;
    }
    __syncthreads();
    const int32_t e = ti.tel[el];
    const bool active = e >= 0 && e < io.n_elements && i < NB;
    const CT *w = W + el * WS;
    const CT *wn = WN + el * WNS;
    const double *G = GE + el * GS;        // G[d][c] = (J^{-T})_{dc}
    const double *nus = GE + el * GS + EG;  // [NFL][DIM]
    CT *x = X + el * XS;
    if (active) {
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
            CT t = CT(0);
#pragma unroll
            for (int d = 0; d < DIM; ++d) t += (CT)G[d * DIM + c] * w[(d + 1) * NB + i];
            x[c * NB + i] = t;
        }
#pragma unroll
        for (int f = 0; f < NFL; ++f) {
            CT a = CT(0);
#pragma unroll
            for (int d = 0; d < DIM; ++d) a += (CT)nus[f * DIM + d] * w[(d + 1) * NB + i];
            x[(DIM + f) * NB + i] = a;
        }
    }
    __syncthreads();
    CT P = CT(0), A[DIM], B[NFL], SP[NFL], nrm[NFL];
    const CT cu = (CT)g.upwind_c;
    if (active) {
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
            const CT *op = OP + c * NB * NB + i;
            CT sp = CT(0), sa = CT(0);
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                const CT o = op[j * NB];
                sp += o * x[c * NB + j];
                sa += o * w[j];
            }
            P += sp;
            A[c] = sa;
        }
#pragma unroll
        for (int f = 0; f < NFL; ++f) {
            const CT *ops = OP + (DIM + 2 * f) * NB * NB + i;
            const CT *opn = OP + (DIM + 2 * f + 1) * NB * NB + i;
            const CT *js = x + (DIM + f) * NB, *jn = wn + f * 2 * NB + NB, *pn = wn + f * 2 * NB;
            CT sp = CT(0), sb = CT(0);
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                const CT os = ops[j * NB], on = opn[j * NB];
                sp += os * js[j] - on * jn[j];
                sb += os * w[j] - on * pn[j];
            }
            P -= sp;
            B[f] = sb;
            SP[f] = sp;
        }
        if (cu != CT(0)) {
#pragma unroll
            for (int f = 0; f < NFL; ++f) {
                double q = 0.0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) q += nus[f * DIM + d] * nus[f * DIM + d];
                nrm[f] = (CT)sqrt(q);
                P -= cu * nrm[f] * B[f];
            }
        }
    }
    __syncthreads();  // W, WN, X read: stage the outputs in W as [element][R]
    if (active) {
        W[el * WS + i] = P;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            CT acc = CT(0);
#pragma unroll
            for (int c = 0; c < DIM; ++c) acc += (CT)G[d * DIM + c] * A[c];
#pragma unroll
            for (int f = 0; f < NFL; ++f) acc -= (CT)nus[f * DIM + d] * B[f];
            acc *= (CT)g.inv_cinv;
            if (cu != CT(0))
#pragma unroll
                for (int f = 0; f < NFL; ++f) acc -= cu * ((CT)nus[f * DIM + d] / nrm[f]) * SP[f];
            W[el * WS + (d + 1) * NB + i] = acc;
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < SH::V; ++it) {
        const int k = tid + it * T;
        const int l = k / R, rr = k % R;
        const int32_t ee = ti.tel[l];
        if (ee < 0 || ee >= io.n_elements) continue;
        const int64_t idx = (int64_t)ee * R + rr;
        stage_output_few(io, idx, io.u[idx], (double)W[l * WS + rr]);
    }
}

// basis rows of a grouped block; 0: no grouped kernel (the wave in 2D and 3D
// only).  Up to 24 basis functions a tile is 32 elements (32 x NB threads), up to
// 35 (tetrahedra at p = 4) 16 elements, whose operators (11 x 35^2 doubles) still
// fit one block's shared memory; above that the per-element-row kernel runs.
constexpr int kGroupMaxRows = 24;
constexpr int kGroupMaxBasis = 35;
__host__ __device__ inline int group_rows(int dim, int wave, int nb) {
    if (dim < 2 || !wave) return 0;
    return nb <= kGroupMaxBasis ? nb : 0;
}
__host__ __device__ constexpr int group_threads(int nb) { return group_tile_elems(nb) * nb; }
template <typename CT, int DIM, int NFL, int NB>
constexpr size_t group_smem() {
    using SH = WaveGroupShape<DIM, NFL, NB>;
    return sizeof(double) * SH::GEO + sizeof(CT) * SH::ELEMS;
}

template <typename KT, int DIM, int NFL, int NB>
__global__ void __launch_bounds__(group_threads(NB), 1024 / group_threads(NB) > 0 ? 1024 / group_threads(NB) : 1)
    dense_group_stage(const StageIOT<KT> io, const DenseGeom g, const int32_t *tiles) {
    wave_group_body<KT, DIM, NFL, NB>(io, g, tiles, blockIdx.x);
}

// basis sizes of the shapes the dense kernel serves, orders 1..5
template <int DIM, int NFL> struct DenseSizes;
template <> struct DenseSizes<1, 2> { static constexpr int nb[5] = {2, 3, 4, 5, 6}; };
template <> struct DenseSizes<2, 3> { static constexpr int nb[5] = {3, 6, 10, 15, 21}; };
template <> struct DenseSizes<2, 4> { static constexpr int nb[5] = {4, 9, 16, 25, 36}; };
template <> struct DenseSizes<3, 4> { static constexpr int nb[5] = {4, 10, 20, 35, 56}; };
template <> struct DenseSizes<3, 6> { static constexpr int nb[5] = {8, 27, 64, 125, 216}; };

// calls f(std::integral_constant<int, NB>) for the runtime nB, if it is one of
// the shape's sizes and fits the kernel (at most 256 coefficients per element);
// returns false otherwise
template <int DIM, int NFL, int WAVE, typename F>
bool dense_dispatch(int nB, F &&f) {
    using S = DenseSizes<DIM, NFL>;
    constexpr int V = WAVE ? DIM + 1 : 1;
    bool done = false;
    auto one = [&](auto k) {
        constexpr int NB = S::nb[decltype(k)::value];
        if constexpr (V * NB <= 256) {
            if (!done && nB == NB) {
                f(std::integral_constant<int, NB>{});
                done = true;
            }
        }
    };
    one(std::integral_constant<int, 0>{});
    one(std::integral_constant<int, 1>{});
    one(std::integral_constant<int, 2>{});
    one(std::integral_constant<int, 3>{});
    one(std::integral_constant<int, 4>{});
    return done;
}

}  // namespace hgg
