// Pencil stage kernel for hexahedra of order p = 3 (tensor-order device layout).
//
// A block handles 32 consecutive elements with 16 warps: lane = element,
// warp = x-pencil (b, c) of that element (4 outputs a = 0..3 per thread).
// Because (b, c) is uniform across a warp, the rows D[b][:] and D[c][:] of the
// 1D operator and the lifts at b and c are broadcast loads from the kernel
// parameters, and the remaining operator entries are compile-time indices.
//   phase 1  each thread brings its pencil of u and of the stage vectors with
//            one 32-byte load each, forms the stage input, stages it in a
//            padded tile (element stride 65 doubles: lanes hit distinct banks),
//            and loads the one entry of each neighbour face slice it is
//            responsible for; all of these loads are independent and issued
//            together;
//   phase 2  flux values of the tile's faces (one entry per thread per face),
//            scaled by sigma, into a padded trace tile;
//   phase 3  derivative along x from registers, along y and z from the staged
//            tile, face lifts from the trace tile; the 4 outputs leave in one
//            32-byte store, and the final Runge-Kutta update is applied in
//            place of a separate pass.
// Small code, few shared accesses per coefficient (~12), two blocks per SM.
#pragma once

#include <cstdint>

#include "dg_kernels.cuh"
#include "tensor_reg.cuh"

namespace hgg {

struct PencilShape {
    static constexpr int TE = 32, THREADS = 512;
    static constexpr int WS = 65;  // staged tile: element stride (doubles)
    static constexpr int TS = 97;  // trace tile: element stride (doubles), 6 faces x 16 entries + pad
};

__global__ void __launch_bounds__(PencilShape::THREADS, 2)
    tensor_pencil(const StageIO io, const RegGeom geo, const RegOps op) {
    constexpr int TE = PencilShape::TE, WS = PencilShape::WS, TS = PencilShape::TS;
    constexpr int tp0 = 0, tp1 = 1;  // psi_0 only mode at -1, psi_1 only mode at +1
    __shared__ double W[TE * WS];
    __shared__ double TR[TE * TS];

    const int el = threadIdx.x & 31;
    const int q = threadIdx.x >> 5;  // pencil (b, c), uniform in the warp
    const int b = q & 3, c = q >> 2;
    const int64_t e = (int64_t)blockIdx.x * TE + el;
    const bool active = e < io.n_elements;
    const int64_t ec = active ? e : 0;
    const int nin = io.nin;

    // ---- phase 1: own pencil, stage input, neighbour slice entries ------------------
    const int64_t own = ec * 64 + 4 * b + 16 * c;
    double w4[4];
    ld4(io.u + own, w4[0], w4[1], w4[2], w4[3]);
    for (int j = 0; j < nin; ++j) {
        double k0, k1, k2, k3;
        ld4(io.kin[j] + own, k0, k1, k2, k3);
        const double cj = io.cin[j];
        w4[0] += cj * k0;
        w4[1] += cj * k1;
        w4[2] += cj * k2;
        w4[3] += cj * k3;
    }
    // entry m = q of every face slot: x (b', c') = (q & 3, q >> 2); y (a', c'); z (a', b')
    const int m0 = q & 3, m1 = q >> 2;
    int md[6];
    double tn[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        md[s] = active ? geo.mode[ec * 6 + s] : 0;
        tn[s] = 0.0;
        if (md[s] >= 2) {
            const int32_t n = geo.nbr[ec * 6 + s];
            if (n >= 0 && n < io.n_elements) {
                const int axis = s >> 1, tpo = (s & 1) ? tp0 : tp1;
                const int pos = axis == 0 ? tpo + 4 * m0 + 16 * m1
                                          : (axis == 1 ? m0 + 4 * tpo + 16 * m1 : m0 + 4 * m1 + 16 * tpo);
                const int64_t off = (int64_t)n * 64 + pos;
                double v = io.u[off];
                for (int j = 0; j < nin; ++j) v += io.cin[j] * io.kin[j][off];
                tn[s] = v;
            } else {
                atomicOr(io.status, 1);
                md[s] = 0;
            }
        }
    }
    double *wrow = W + el * WS;
#pragma unroll
    for (int a = 0; a < 4; ++a) wrow[4 * b + 16 * c + a] = w4[a];
    __syncthreads();

    // ---- phase 2: flux entries of the six faces -------------------------------------
    double *trow = TR + el * TS;
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        const int axis = s >> 1, tps = (s & 1) ? tp1 : tp0;
        const int pos = axis == 0 ? tps + 4 * m0 + 16 * m1 : (axis == 1 ? m0 + 4 * tps + 16 * m1 : m0 + 4 * m1 + 16 * tps);
        const double self = wrow[pos];
        const double sg = active ? geo.sigma[ec * 6 + s] : 0.0;
        trow[16 * s + q] = reg_flux(md[s], sg, self, tn[s]);
    }
    __syncthreads();
    if (!active) return;

    // ---- phase 3: four outputs of the pencil ----------------------------------------
    const double ax = geo.ahat[ec * 3], ay = geo.ahat[ec * 3 + 1], az = geo.ahat[ec * 3 + 2];
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
