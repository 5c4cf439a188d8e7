// Slice stage kernel for hexahedra of order p = 3 (tiled device layout).
//
// Device layout.  Vectors of a hexahedral p = 3 handle are stored in tiles of
// 32 elements; inside a tile coefficient j of element e sits at
//     (e / 32) * 2048 + j * 32 + e % 32,
// with j the tensor position a + 4 b + 16 c (signs folded in).  A warp whose
// lanes are the 32 elements of a tile therefore reads or writes any one
// coefficient as 256 contiguous bytes, and so does a warp reading one
// coefficient of 32 consecutive neighbours (the y and z neighbours of a tile
// of a structured mesh are again whole tiles).
//
// Thread organisation.  One block of 128 threads per tile: lane = element,
// warp c = the z-slice c of that element, so each thread owns the 16
// coefficients (a, b, c), a, b = 0..3.  The x and y derivatives and the x and
// y face traces of its outputs come from registers; only the z derivative and
// the z faces need other slices, through a padded staged tile in shared
// memory.  The L1 data path, which limits per-element-per-thread layouts on
// this part, sees about a third of their shared and global wavefronts.
//   phase 1  tile geometry records (coalesced copy into shared memory), the
//            thread's 16 coefficients of u and of the stage vectors, stage
//            input w staged in shared memory (element stride 65 doubles:
//            lanes hit distinct banks);
//   phase 2  face fluxes: x faces (entries (b, c)) and y faces (entries
//            (a, c)) into registers, neighbour traces from the staged tile
//            when the neighbour is in the tile, else from global memory; z
//            faces (16 entries per side) are spread over the four warps and
//            go to a padded trace tile;
//   phase 3  the 16 outputs: x and y derivatives from registers, z derivative
//            from the staged tile, lifts of the six face fluxes; kout and the
//            final Runge-Kutta update are written coefficient by coefficient.
//
// Precision.  KT is the type of the stage vectors and of the contractions:
// double (FP64 form) or float (FP32-mixed form: stage vectors stored in FP32,
// stage input formed in FP64 from the FP64 solution and rounded once, the
// derivative, lift and flux arithmetic in FP32, the geometry computed and
// stored in FP64, the final update u + dt sum b_j k_j accumulated in FP64).
#pragma once

#include <cstdint>

#include "dg_kernels.cuh"

namespace hgg {

struct SliceOps {
    double D[16];    // M1^{-1} S1 (row-major, D[i][k])
    double L[2][4];  // M1^{-1} psi(-1), M1^{-1} psi(+1)
};

struct SliceShape {
    static constexpr int TE = 32, THREADS = 128;
    static constexpr int TILE = TE * 64;  // doubles per tile of one vector
    static constexpr int WS = 65;         // staged tile: element stride (doubles)
    static constexpr int ZS = 33;         // z-face trace tile: element stride (doubles)
    static constexpr int GR = 13;         // geometry record (doubles): ahat[3], sigma[6], nbr[6] int32, mode[6] int8
};

// index of coefficient j of element n in the tiled layout
__device__ __forceinline__ int64_t tiled_index(int64_t n, int j) {
    return (n >> 5) * SliceShape::TILE + j * 32 + (n & 31);
}

__device__ __forceinline__ double ldg_f64(const double *p) {
    double v;
    asm("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ float ldg_f32(const float *p) {
    float v;
    asm("ld.global.nc.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ double ldg_k(const double *p) { return ldg_f64(p); }
__device__ __forceinline__ double ldg_k(const float *p) { return (double)ldg_f32(p); }

template <typename CT>
__device__ __forceinline__ CT slice_flux(int md, CT sg, CT self, CT nbr) {
    return md == 1 ? sg * self : (md == 2 ? sg * nbr : (md == 3 ? CT(0.5) * sg * (self + nbr) : CT(0)));
}

// NIN / NFIN: number of stage vectors in the stage input / in the final
// update, fixed at compile time for the common Runge-Kutta stages (so every
// load loop unrolls and all loads of a phase are in flight together), or -1
// for a count read from io.
// L2 prefetch of `bytes` (a multiple of 16) from a 16-byte aligned global address
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Tiles of one vector are contiguous runs (TILE coefficients), so the inputs a
// later block will read are a handful of bulk prefetches.
template <typename KT>
__device__ __forceinline__ void prefetch_tile(const StageIOT<KT> &io, const double *geo, int64_t tile, int nin,
                                              int nfin) {
    constexpr int TILE = SliceShape::TILE;
    prefetch_l2(io.u + tile * TILE, TILE * sizeof(double));
    for (int j = 0; j < nin; ++j) prefetch_l2(io.kin[j] + tile * TILE, TILE * sizeof(KT));
    if (io.unew)
        for (int j = 0; j < nfin; ++j) prefetch_l2(io.kfin[j] + tile * TILE, TILE * sizeof(KT));
    prefetch_l2(geo + tile * SliceShape::TE * SliceShape::GR, SliceShape::TE * SliceShape::GR * sizeof(double));
}

// prefetch_ahead: this block asks L2 for the inputs of tile + prefetch_ahead (the
// tile a block of the next resident wave runs), 0 for none; n_tiles bounds it.
template <typename KT, int NIN, int NFIN>
__device__ __forceinline__ void tensor_slice_body(const StageIOT<KT> &io, const double *__restrict__ geo,
                                                  const SliceOps &op, int64_t tile, int64_t prefetch_ahead = 0,
                                                  int64_t n_tiles = 0) {
    using CT = KT;  // contraction type
    constexpr int TE = SliceShape::TE, WS = SliceShape::WS, ZS = SliceShape::ZS, GR = SliceShape::GR;
    constexpr int TILE = SliceShape::TILE;
    constexpr int tp0 = 0, tp1 = 1;  // psi_0 only mode at -1, psi_1 only mode at +1
    __shared__ CT W[TE * WS];
    __shared__ CT TZ[TE * ZS];
    __shared__ double G[TE * GR];

    const int el = threadIdx.x & 31;
    const int c = threadIdx.x >> 5;  // z-slice, uniform in the warp
    const int64_t t0 = tile * TE;
    const int64_t e = t0 + el;
    const bool active = e < io.n_elements;
    // own coefficient j of this element: base + 32 j (padding lanes read their own zero slots)
    const int64_t base = tile * TILE + el;
    const int nin = NIN >= 0 ? NIN : io.nin;
    const int nfin = NFIN >= 0 ? NFIN : io.nfin;

    // ---- phase 1: geometry records, own slice, stage input -------------------------
    if (prefetch_ahead > 0 && threadIdx.x == 0 && tile + prefetch_ahead < n_tiles)
        prefetch_tile(io, geo, tile + prefetch_ahead, nin, nfin);
    for (int i = threadIdx.x; i < TE * GR; i += SliceShape::THREADS) G[i] = ldg_f64(geo + t0 * GR + i);
    CT w[16];
    {
        double wd[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) wd[i] = ldg_f64(io.u + base + 32 * (i + 16 * c));
#pragma unroll
        for (int jj = 0; jj < nin; ++jj) {
            const double cj = io.cin[jj];
            const KT *kj = io.kin[jj] + base;
#pragma unroll
            for (int i = 0; i < 16; ++i) wd[i] += cj * ldg_k(kj + 32 * (i + 16 * c));
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) w[i] = (CT)wd[i];
    }
    CT *wrow = W + el * WS;
#pragma unroll
    for (int i = 0; i < 16; ++i) wrow[i + 16 * c] = w[i];
    __syncthreads();

    // ---- phase 2: face fluxes -------------------------------------------------------
    const double *g = G + el * GR;
    const int32_t *gn = reinterpret_cast<const int32_t *>(g + 9);
    const int8_t *gm = reinterpret_cast<const int8_t *>(g + 12);
    int md[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        md[s] = active ? (int)gm[s] : 0;
        if (md[s] >= 2 && (gn[s] < 0 || gn[s] >= io.n_elements)) {
            atomicOr(io.status, 1);
            md[s] = 0;
        }
    }
    const int zside = c >> 1, zs = 4 + zside, zm0 = 8 * (c & 1);
    // neighbour traces, all requested before any is used: entries (b, c) of the x faces,
    // (a, c) of the y faces, 8 of the 16 entries (a, b) of z face zs
    auto nbr_pos = [&](int s, int q) {  // neighbour position of entry q of face s (this warp's part)
        const int tpo = (s & 1) ? tp0 : tp1;
        return s < 2 ? tpo + 4 * q + 16 * c : (s < 4 ? q + 4 * tpo + 16 * c : zm0 + q + 16 * tpo);
    };
    CT NB[5][8];
#pragma unroll
    for (int f = 0; f < 5; ++f) {
        const int s = f < 4 ? f : zs;
        const int nq = f < 4 ? 4 : 8;
#pragma unroll
        for (int q = 0; q < 8; ++q) NB[f][q] = CT(0);
        const int32_t n = gn[s];
        if (md[s] >= 2) {
            if (n >= t0 && n < t0 + TE) {
                const CT *nrow = W + (int)(n - t0) * WS;
#pragma unroll
                for (int q = 0; q < nq; ++q) NB[f][q] = nrow[nbr_pos(s, q)];
            } else {
                const int64_t nbase = ((int64_t)n >> 5) * TILE + (n & 31);
                double v[8];
#pragma unroll
                for (int q = 0; q < nq; ++q) v[q] = ldg_f64(io.u + nbase + 32 * nbr_pos(s, q));
#pragma unroll
                for (int jj = 0; jj < nin; ++jj) {
                    const double cj = io.cin[jj];
#pragma unroll
                    for (int q = 0; q < nq; ++q) v[q] += cj * ldg_k(io.kin[jj] + nbase + 32 * nbr_pos(s, q));
                }
#pragma unroll
                for (int q = 0; q < nq; ++q) NB[f][q] = (CT)v[q];
            }
        }
    }
    CT FX[2][4], FY[2][4];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const int tps = side ? tp1 : tp0;
        const CT sgx = (CT)g[3 + side], sgy = (CT)g[5 + side];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            FX[side][q] = slice_flux<CT>(md[side], sgx, w[tps + 4 * q], NB[side][q]);
            FY[side][q] = slice_flux<CT>(md[2 + side], sgy, w[q + 4 * tps], NB[2 + side][q]);
        }
    }
    {
        const int tps = zside ? tp1 : tp0;
        const CT sgz = (CT)g[3 + zs];
#pragma unroll
        for (int q = 0; q < 8; ++q)
            TZ[el * ZS + 16 * zside + zm0 + q] = slice_flux<CT>(md[zs], sgz, wrow[zm0 + q + 16 * tps], NB[4][q]);
    }
    __syncthreads();
    if (!active) return;

    // ---- phase 3: the 16 outputs of the slice ---------------------------------------
    double fu[16];
    if (io.unew) {
#pragma unroll
        for (int i = 0; i < 16; ++i) fu[i] = ldg_f64(io.u + base + 32 * (i + 16 * c));
#pragma unroll
        for (int jj = 0; jj < nfin; ++jj) {
            const double bj = io.bfin[jj];
            const KT *kj = io.kfin[jj] + base;
#pragma unroll
            for (int i = 0; i < 16; ++i) fu[i] += bj * ldg_k(kj + 32 * (i + 16 * c));
        }
    }
    const CT ax = (CT)g[0], ay = (CT)g[1], az = (CT)g[2];
    CT D[16], L0[4], L1[4], Dc[4], Lc0, Lc1;
#pragma unroll
    for (int k = 0; k < 16; ++k) D[k] = (CT)op.D[k];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        L0[k] = (CT)op.L[0][k];
        L1[k] = (CT)op.L[1][k];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) Dc[k] = c == 0 ? D[k] : (c == 1 ? D[4 + k] : (c == 2 ? D[8 + k] : D[12 + k]));
    Lc0 = c == 0 ? L0[0] : (c == 1 ? L0[1] : (c == 2 ? L0[2] : L0[3]));
    Lc1 = c == 0 ? L1[0] : (c == 1 ? L1[1] : (c == 2 ? L1[2] : L1[3]));
    const CT *zrow = TZ + el * ZS;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = a + 4 * b;
            CT sx = CT(0), sy = CT(0), sz = CT(0);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                sx += D[a * 4 + k] * w[k + 4 * b];
                sy += D[b * 4 + k] * w[a + 4 * k];
                sz += Dc[k] * (k == c ? w[i] : wrow[i + 16 * k]);
            }
            CT r = ax * sx + ay * sy + az * sz;
            r -= L0[a] * FX[0][b] + L1[a] * FX[1][b];
            r -= L0[b] * FY[0][a] + L1[b] * FY[1][a];
            r -= Lc0 * zrow[i] + Lc1 * zrow[16 + i];
            const int64_t off = base + 32 * (i + 16 * c);
            if (io.kout) io.kout[off] = r;
            if (io.unew) io.unew[off] = fu[i] + io.blast * (double)r;
        }
    }
}

// One block per 32-element tile of one problem.  Five blocks per SM (102
// registers, a little spilling) for the stages without the final update: the
// extra resident warps measured 1.6 % faster per RK4 step than four blocks;
// the final stage, which holds 16 more values per thread, keeps four.
template <typename KT, int NIN, int NFIN>
__global__ void __launch_bounds__(SliceShape::THREADS, sizeof(KT) == 4 ? 5 : (NFIN == 0 ? 5 : 4))
    tensor_slice(const StageIOT<KT> io, const double *__restrict__ geo, const SliceOps op, int64_t prefetch_ahead) {
    tensor_slice_body<KT, NIN, NFIN>(io, geo, op, blockIdx.x, prefetch_ahead, gridDim.x);
}

}  // namespace hgg
