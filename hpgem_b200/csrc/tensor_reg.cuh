// Register-resident sum-factorised stage kernel for hexahedra of order p = 3.
//
// One thread owns one element: its 64 stage-input coefficients live in
// registers for the whole stage, so the volume term and the element's own face
// traces need no shared memory at all.  Data movement:
//   * the element's slice of u and of the stage vectors arrives with 32-byte
//     vector loads (ld.global.v4.f64), each a full DRAM sector, all
//     independent, so every thread has dozens of loads in flight;
//   * the x-neighbours of consecutive elements are neighbouring lanes: their
//     face traces cross with warp shuffles of the already formed stage input;
//   * y and z neighbour slices are 4 and 1 runs of 32 bytes in the tensor
//     layout (z slice: 16 contiguous coefficients), loaded where they are
//     used (mostly L2 hits: the neighbours were read moments earlier);
//   * each x-pencil of 4 outputs leaves with one 32-byte store; the final
//     Runge-Kutta update is applied pencil by pencil.
// Device vectors are in tensor order (a + 4 b + 16 c, signs folded in).
#pragma once

#include <cstdint>

#include "dg_kernels.cuh"

namespace hgg {

struct RegOps {
    double D[16];    // M1^{-1} S1
    double L[2][4];  // M1^{-1} psi(-1), M1^{-1} psi(+1)
};

struct RegGeom {
    const double *ahat;   // [E][3]
    const int32_t *nbr;   // [E][6] slots x-, x+, y-, y+, z-, z+
    const int8_t *mode;   // [E][6]
    const double *sigma;  // [E][6]
};

// 32-byte loads of data that no thread writes during the launch (the stage's
// inputs are never its outputs), so they may take the read-only path
__device__ __forceinline__ void ld4(const double *p, double &a, double &b, double &c, double &d) {
    asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
}
__device__ __forceinline__ void st4(double *p, double a, double b, double c, double d) {
    asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(a), "d"(b), "d"(c), "d"(d) : "memory");
}

__device__ __forceinline__ double reg_flux(int md, double sg, double self, double nbr) {
    return md == 1 ? sg * self : (md == 2 ? sg * nbr : (md == 3 ? 0.5 * sg * (self + nbr) : 0.0));
}

// stage input of 4 consecutive coefficients of element n (32-byte aligned run)
__device__ __forceinline__ void run4(const StageIO &io, int64_t off, double v[4]) {
    ld4(io.u + off, v[0], v[1], v[2], v[3]);
    for (int j = 0; j < io.nin; ++j) {
        double k0, k1, k2, k3;
        ld4(io.kin[j] + off, k0, k1, k2, k3);
        v[0] += io.cin[j] * k0;
        v[1] += io.cin[j] * k1;
        v[2] += io.cin[j] * k2;
        v[3] += io.cin[j] * k3;
    }
}

__global__ void __launch_bounds__(128)
    tensor_reg(const StageIO io, const RegGeom geo, const RegOps op) {
    // hpGEM's 1D set: psi_0 is the only mode at -1, psi_1 the only one at +1
    constexpr int tp0 = 0, tp1 = 1;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = e < io.n_elements;
    const int lane = threadIdx.x & 31;
    const int64_t ec = active ? e : io.n_elements - 1;  // inactive lanes still take part in shuffles
    const int64_t base = ec * 64;

    double w[64];
#pragma unroll
    for (int r = 0; r < 16; ++r) ld4(io.u + base + 4 * r, w[4 * r], w[4 * r + 1], w[4 * r + 2], w[4 * r + 3]);
    for (int j = 0; j < io.nin; ++j) {
        const double cj = io.cin[j];
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            double k0, k1, k2, k3;
            ld4(io.kin[j] + base + 4 * r, k0, k1, k2, k3);
            w[4 * r] += cj * k0;
            w[4 * r + 1] += cj * k1;
            w[4 * r + 2] += cj * k2;
            w[4 * r + 3] += cj * k3;
        }
    }

    int md[6];
    int32_t nb[6];
    double sg[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        md[s] = geo.mode[ec * 6 + s];
        nb[s] = geo.nbr[ec * 6 + s];
        sg[s] = geo.sigma[ec * 6 + s];
        if (md[s] >= 2 && (nb[s] < 0 || nb[s] >= io.n_elements)) {
            atomicOr(io.status, 1);
            md[s] = 0;
        }
        if (!active) md[s] = 0;
    }
    const double ax = geo.ahat[ec * 3], ay = geo.ahat[ec * 3 + 1], az = geo.ahat[ec * 3 + 2];

    // x faces: neighbour traces of the previous / next lane when they are the x-neighbours
    const bool need_xm = md[0] >= 2, need_xp = md[1] >= 2;
    const bool shfl_xm = need_xm && lane > 0 && nb[0] == e - 1;
    const bool shfl_xp = need_xp && lane < 31 && nb[1] == e + 1;
    const bool any_xm = __any_sync(0xffffffffu, need_xm), any_xp = __any_sync(0xffffffffu, need_xp);

#pragma unroll
    for (int c = 0; c < 4; ++c) {
        // y faces of plane c: flux entries (a, c), one 32-byte run of the neighbour
        double FY[2][4];
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const int s = 2 + side, tps = side ? tp1 : tp0, tpo = side ? tp0 : tp1;
            double v[4] = {0.0, 0.0, 0.0, 0.0};
            if (md[s] >= 2) run4(io, (int64_t)nb[s] * 64 + 4 * tpo + 16 * c, v);
#pragma unroll
            for (int a = 0; a < 4; ++a) FY[side][a] = reg_flux(md[s], sg[s], w[a + 4 * tps + 16 * c], v[a]);
        }
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            // x faces of pencil (b, c)
            double xm = 0.0, xp = 0.0;
            if (any_xm) xm = __shfl_up_sync(0xffffffffu, w[tp1 + 4 * b + 16 * c], 1);
            if (any_xp) xp = __shfl_down_sync(0xffffffffu, w[tp0 + 4 * b + 16 * c], 1);
            if (need_xm && !shfl_xm) {
                const int64_t off = (int64_t)nb[0] * 64 + tp1 + 4 * b + 16 * c;
                double t = io.u[off];
                for (int j = 0; j < io.nin; ++j) t += io.cin[j] * io.kin[j][off];
                xm = t;
            }
            if (need_xp && !shfl_xp) {
                const int64_t off = (int64_t)nb[1] * 64 + tp0 + 4 * b + 16 * c;
                double t = io.u[off];
                for (int j = 0; j < io.nin; ++j) t += io.cin[j] * io.kin[j][off];
                xp = t;
            }
            const double fxm = reg_flux(md[0], sg[0], w[tp0 + 4 * b + 16 * c], xm);
            const double fxp = reg_flux(md[1], sg[1], w[tp1 + 4 * b + 16 * c], xp);
            // z faces of pencil (b, c): flux entries (a, b), one 32-byte run of the neighbour
            double FZ[2][4];
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const int s = 4 + side, tps = side ? tp1 : tp0, tpo = side ? tp0 : tp1;
                double v[4] = {0.0, 0.0, 0.0, 0.0};
                if (md[s] >= 2) run4(io, (int64_t)nb[s] * 64 + 16 * tpo + 4 * b, v);
#pragma unroll
                for (int a = 0; a < 4; ++a) FZ[side][a] = reg_flux(md[s], sg[s], w[a + 4 * b + 16 * tps], v[a]);
            }
            double kv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    sx += op.D[a * 4 + k] * w[k + 4 * b + 16 * c];
                    sy += op.D[b * 4 + k] * w[a + 4 * k + 16 * c];
                    sz += op.D[c * 4 + k] * w[a + 4 * b + 16 * k];
                }
                double r = ax * sx + ay * sy + az * sz;
                r -= op.L[0][a] * fxm + op.L[1][a] * fxp;
                r -= op.L[0][b] * FY[0][a] + op.L[1][b] * FY[1][a];
                r -= op.L[0][c] * FZ[0][a] + op.L[1][c] * FZ[1][a];
                kv[a] = r;
            }
            if (active) {
                const int64_t off = base + 4 * b + 16 * c;
                if (io.kout) st4(io.kout + off, kv[0], kv[1], kv[2], kv[3]);
                if (io.unew) {
                    double u[4];
                    ld4(io.u + off, u[0], u[1], u[2], u[3]);
                    for (int j = 0; j < io.nfin; ++j) {
                        double k0, k1, k2, k3;
                        ld4(io.kfin[j] + off, k0, k1, k2, k3);
                        u[0] += io.bfin[j] * k0;
                        u[1] += io.bfin[j] * k1;
                        u[2] += io.bfin[j] * k2;
                        u[3] += io.bfin[j] * k3;
                    }
                    st4(io.unew + off, u[0] + io.blast * kv[0], u[1] + io.blast * kv[1], u[2] + io.blast * kv[2],
                        u[3] + io.blast * kv[3]);
                }
            }
        }
    }
}

}  // namespace hgg
