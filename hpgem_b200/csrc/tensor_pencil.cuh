// Pencil stage kernel for hexahedra of order p = 3 (tensor-order device layout).
//
// A block handles 32 consecutive elements with 16 warps: lane = element,
// warp = x-pencil (b, c) of that element (4 outputs a = 0..3 per thread).
// Because (b, c) is uniform across a warp, the rows D[b][:] and D[c][:] of the
// 1D operator and the lifts at b and c are broadcast loads from the kernel
// parameters, and the remaining operator entries are compile-time indices.
//
// The limit of this organisation is the L1 request rate, not DRAM: each warp
// instruction whose 32 lanes touch 32 elements costs at least 32 sector
// lookups.  So every global access is either a 32-byte vector (one full sector
// per lane) or a coalesced block-wide copy:
//   phase 1  the tile's geometry records (ahat, sigma, neighbours, modes: 104
//            bytes per element, padded to whole tiles) come in with one
//            coalesced 8-byte load per thread into shared memory; each thread
//            brings its pencil of u and of the stage vectors with one 32-byte
//            load each, forms the stage input and stages it in a padded tile
//            (element stride 65 doubles: lanes hit distinct banks);
//   phase 2  neighbour traces of the y and z faces: a y-face trace is 4 runs
//            of 4 consecutive coefficients of the neighbour, a z-face trace 16
//            consecutive ones, so warp q fetches run q & 3 of face 2 + (q >> 2)
//            with one 32-byte load per vector.  An x-face neighbour inside the
//            tile is read from the staged tile later; one outside it (tile
//            edges, periodic wrap) is fetched entry by entry;
//   phase 3  flux values of the six faces (one entry per thread per face),
//            scaled by sigma, into a padded trace tile;
//   phase 4  derivative along x from registers, along y and z from the staged
//            tile, face lifts from the trace tile; the 4 outputs leave in one
//            32-byte store, and the final Runge-Kutta update is applied in
//            place of a separate pass.
#pragma once

#include <cstdint>

#include "dg_kernels.cuh"
#include "tensor_reg.cuh"

namespace hgg {

struct PencilShape {
    static constexpr int TE = 32, THREADS = 512;
    static constexpr int WS = 65;  // staged tile: element stride (doubles)
    static constexpr int TS = 97;  // trace tile: element stride (doubles), 6 faces x 16 entries + pad
    static constexpr int GR = 13;  // geometry record (doubles): ahat[3], sigma[6], nbr[6] int32, mode[6] int8
};

__device__ __forceinline__ double ldg_f64(const double *p) {
    double v;
    asm("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}

__global__ void __launch_bounds__(PencilShape::THREADS, 2)
    tensor_pencil(const StageIO io, const double *__restrict__ geo, const RegOps op) {
    constexpr int TE = PencilShape::TE, WS = PencilShape::WS, TS = PencilShape::TS, GR = PencilShape::GR;
    constexpr int tp0 = 0, tp1 = 1;  // psi_0 only mode at -1, psi_1 only mode at +1
    __shared__ double W[TE * WS];
    __shared__ double TR[TE * TS];
    __shared__ double G[TE * GR];

    const int el = threadIdx.x & 31;
    const int q = threadIdx.x >> 5;  // pencil (b, c), uniform in the warp
    const int b = q & 3, c = q >> 2;
    const int64_t t0 = (int64_t)blockIdx.x * TE;
    const int64_t e = t0 + el;
    const bool active = e < io.n_elements;
    const int64_t ec = active ? e : 0;
    const int nin = io.nin;

    // ---- phase 1: geometry records, own pencil, stage input -------------------------
    if (threadIdx.x < TE * GR) G[threadIdx.x] = ldg_f64(geo + t0 * GR + threadIdx.x);
    const int64_t own = ec * 64 + 4 * b + 16 * c;
    double w4[4];
    run4(io, own, w4);
    double *wrow = W + el * WS;
#pragma unroll
    for (int a = 0; a < 4; ++a) wrow[4 * b + 16 * c + a] = w4[a];
    __syncthreads();

    const double *g = G + el * GR;
    const int32_t *gn = reinterpret_cast<const int32_t *>(g + 9);
    const int8_t *gm = reinterpret_cast<const int8_t *>(g + 12);
    double *trow = TR + el * TS;
    const int m0 = q & 3, m1 = q >> 2;  // entry m = q of a face slot
    auto valid = [&](int32_t n) { return n >= 0 && n < io.n_elements; };
    auto local = [&](int32_t n) { return valid(n) && n >= t0 && n < t0 + TE; };

    // ---- phase 2: neighbour traces that are not in the staged tile ------------------
    {
        const int s = 2 + (q >> 2), r = q & 3;
        const int tpo = (s & 1) ? tp0 : tp1;
        const int32_t n = gn[s];
        if (active && gm[s] >= 2) {
            if (valid(n)) {
                const int start = s < 4 ? 4 * tpo + 16 * r : 4 * r + 16 * tpo;
                double v[4];
                run4(io, (int64_t)n * 64 + start, v);
#pragma unroll
                for (int a = 0; a < 4; ++a) trow[16 * s + 4 * r + a] = v[a];
            } else {
                atomicOr(io.status, 1);
            }
        }
    }
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const int32_t n = gn[s];
        if (active && gm[s] >= 2 && !local(n)) {
            if (valid(n)) {
                const int64_t off = (int64_t)n * 64 + ((s & 1) ? tp0 : tp1) + 4 * m0 + 16 * m1;
                double v = io.u[off];
                for (int j = 0; j < nin; ++j) v += io.cin[j] * io.kin[j][off];
                trow[16 * s + q] = v;
            } else {
                atomicOr(io.status, 1);
            }
        }
    }
    __syncthreads();

    // ---- phase 3: flux entries of the six faces -------------------------------------
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        const int axis = s >> 1, tps = (s & 1) ? tp1 : tp0, tpo = (s & 1) ? tp0 : tp1;
        const int pos = axis == 0 ? tps + 4 * m0 + 16 * m1 : (axis == 1 ? m0 + 4 * tps + 16 * m1 : m0 + 4 * m1 + 16 * tps);
        const int32_t n = gn[s];
        int md = active ? gm[s] : 0;
        if (md >= 2 && !valid(n)) md = 0;
        double nb = 0.0;
        if (md >= 2) {
            if (axis == 0 && local(n))
                nb = W[(int)(n - t0) * WS + tpo + 4 * m0 + 16 * m1];
            else
                nb = trow[16 * s + q];
        }
        trow[16 * s + q] = reg_flux(md, g[3 + s], wrow[pos], nb);
    }
    __syncthreads();
    if (!active) return;

    // ---- phase 4: four outputs of the pencil ----------------------------------------
    const double ax = g[0], ay = g[1], az = g[2];
    double Db[4], Dc[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        Db[k] = op.D[b * 4 + k];
        Dc[k] = op.D[c * 4 + k];
    }
    const double lb0 = op.L[0][b], lb1 = op.L[1][b], lc0 = op.L[0][c], lc1 = op.L[1][c];
    const double fxm = trow[16 * 0 + b + 4 * c], fxp = trow[16 * 1 + b + 4 * c];
    double kv[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            sx += op.D[a * 4 + k] * w4[k];
            sy += Db[k] * (k == b ? w4[a] : wrow[a + 4 * k + 16 * c]);
            sz += Dc[k] * (k == c ? w4[a] : wrow[a + 4 * b + 16 * k]);
        }
        double r = ax * sx + ay * sy + az * sz;
        r -= op.L[0][a] * fxm + op.L[1][a] * fxp;
        r -= lb0 * trow[16 * 2 + a + 4 * c] + lb1 * trow[16 * 3 + a + 4 * c];
        r -= lc0 * trow[16 * 4 + a + 4 * b] + lc1 * trow[16 * 5 + a + 4 * b];
        kv[a] = r;
    }
    if (io.kout) st4(io.kout + own, kv[0], kv[1], kv[2], kv[3]);
    if (io.unew) {
        double u[4];
        ld4(io.u + own, u[0], u[1], u[2], u[3]);
        for (int j = 0; j < io.nfin; ++j) {
            double k0, k1, k2, k3;
            ld4(io.kfin[j] + own, k0, k1, k2, k3);
            u[0] += io.bfin[j] * k0;
            u[1] += io.bfin[j] * k1;
            u[2] += io.bfin[j] * k2;
            u[3] += io.bfin[j] * k3;
        }
        st4(io.unew + own, u[0] + io.blast * kv[0], u[1] + io.blast * kv[1], u[2] + io.blast * kv[2],
            u[3] + io.blast * kv[3]);
    }
}

}  // namespace hgg
