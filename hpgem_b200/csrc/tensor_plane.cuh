// Sum-factorised stage kernel for hexahedra of order p = 3, organised around
// shared-memory traffic (the bound of the pencil kernels).
//
// The coefficient vectors of a sum-factorised handle are stored on the device
// in tensor order (index a + 4 b + 16 c of the 1D modes along x, y, z, signs
// folded in); hgg_set_state / hgg_get_state convert from and to hpGEM's order.
// In that layout the face slices of an element are: z-faces 16 contiguous
// values, y-faces 4 runs of 4, x-faces 16 values with stride 4.
//
// A persistent block walks tiles of TE = 32 consecutive elements:
//   * bulk asynchronous copies (cp.async.bulk, mbarrier ring) bring the tile's
//     slice of u, of the stage vectors and its packed geometry records;
//   * face slices of neighbours outside the tile follow a plan built on the
//     host (per tile: which element, which slice, which halo slot) and are
//     gathered one tile ahead with cp.async 16- or 8-byte copies into the
//     slot's halo area; neighbours inside the tile are read from the tile;
//   * the stage input is formed once per tile into a padded tile W (element
//     stride 65 doubles, so a warp reading one entry of 32 elements touches 32
//     different banks);
//   * each thread owns half of one z-plane of one element (8 outputs); the
//     plane index and the half are uniform per warp, so the operator rows
//     they select are shared-memory broadcasts and every other operator entry
//     is a compile-time index into the kernel parameters;
//   * stage derivatives leave from registers in 32-byte runs; the final RK
//     update runs over the tile in coefficient order from the staged k.
// Every mbarrier wait is bounded (status bit 1 on expiry).
#pragma once

#include <cstdint>

#include "dg_kernels.cuh"
#include "tensor_pipe.cuh"

namespace hgg {

namespace ptx {

// 16-byte (cg, L2 only) and 8-byte (ca) asynchronous global -> shared copies
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

}  // namespace ptx

struct PlaneShape {
    static constexpr int NP = 4, NB = 64, TE = 32, THREADS = 256;
    static constexpr int ES = 65;                // padded element stride of the staged tiles
    static constexpr int GEO_WORDS = 17;         // packed record, 136 bytes
    static constexpr int GEO_BYTES = 8 * GEO_WORDS;
    static constexpr int TILE_VEC_BYTES = TE * NB * 8;    // 16 KB
    static constexpr int TILE_GEO_BYTES = TE * GEO_BYTES;  // 4352
};

// Geometry record per element (136 bytes):
//   double ahat[3]; double sigma[6];            words 0..8
//   int8   mode[6]; int8 nloc[6];                 bytes 72..83 (neighbour index inside the tile or -1)
//   int16  hslot[6];                              bytes 84..95 (halo slot when outside, else -1)
// Face slots s: x-, x+, y-, y+, z-, z+ (axis = s / 2, side = s % 2).
// Plan entry (int64): element (bits 0..31), neighbour slice axis*2+side (bits 32..39), halo slot (40..55).

struct PlaneArgs {
    const unsigned char *geo;  // [E_pad][136]
    const int64_t *plan;       // gather entries of all tiles
    const int32_t *plan_off;   // [n_tiles + 1]
    int64_t n_tiles;
    int nbuf;
    int nv;                    // vectors bulk-loaded per tile: u, kin[..], then kfin[..] not already loaded
    const double *lv[1 + 2 * kMaxStages];  // the loaded vectors
    int fin_idx[kMaxStages];   // position in lv of each kfin vector
    int nhv;                   // vectors gathered per halo slice: u, kin[..] (1 + nin)
    int halo_slots;            // slices per tile
    uint32_t slot_bytes;       // nv * 16 KB + geo
    uint32_t halo_bytes;       // halo area per slot
    int trace_pos[2];          // the 1D mode that is 1 at -1 / +1
};

struct PlaneOps {
    double D[16];    // 1D derivative operator M1^{-1} S1
    double L[2][4];  // lifts M1^{-1} psi(-1), M1^{-1} psi(+1)
};

// neighbour trace entry: from the staged tile when the neighbour is inside it,
// else from the gathered halo (stage input formed from u and one stage vector)
__device__ __forceinline__ double plane_nbr(const double *W, const double *halo, int halo_stride, int nl, int hs,
                                            int m, int gpos, int nin, double cin0) {
    if (nl >= 0) return W[nl * PlaneShape::ES + gpos];
    const double *hp = halo + hs * halo_stride;
    double v = hp[m];
    if (nin >= 1) v += cin0 * hp[16 + m];
    return v;
}

__device__ __forceinline__ double plane_flux(int md, double sg, double self, double nbr) {
    return md == 1 ? sg * self : (md == 2 ? sg * nbr : (md == 3 ? 0.5 * sg * (self + nbr) : 0.0));
}

// Eight outputs (a = 0..3, b = 2H, 2H+1) of plane C of element `el`; written to
// k (global, two 32-byte runs) and/or to the staged tile KS for the final update.
// C and H are uniform across the warp: the operator rows they select are read
// from shared memory as broadcasts, while every other operator entry has a
// compile-time index into the kernel parameters.
__device__ __forceinline__ void plane_compute(const PlaneOps &op, const double *sD, const double *sL,
                                              const double *W, const unsigned char *geo, const double *halo,
                                              int halo_stride, int el, int C, int H, int nin, double cin0,
                                              double *kout, double *ks) {
    const double *w = W + el * PlaneShape::ES;
    const double *wc = w + 16 * C;
    const double *g = reinterpret_cast<const double *>(geo);
    const int8_t *mode = reinterpret_cast<const int8_t *>(geo + 72);
    const int8_t *nloc = reinterpret_cast<const int8_t *>(geo + 78);
    const int16_t *hslot = reinterpret_cast<const int16_t *>(geo + 84);
    const double ax = g[0], ay = g[1], az = g[2];
    // hpGEM's 1D hierarchical set: psi_0 = (1-x)/2 is the only mode at -1 and
    // psi_1 = (1+x)/2 the only one at +1 (checked on the host before this kernel is chosen)
    constexpr int tp0 = 0, tp1 = 1;

    double Db[2][4], Dc[4];  // derivative rows of b = 2H + bb and of c = C
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        Db[0][k] = sD[(2 * H) * 4 + k];
        Db[1][k] = sD[(2 * H + 1) * 4 + k];
        Dc[k] = sD[C * 4 + k];
    }

    double acc[2][4];
    {
        double P[4][4];  // P[b][a] of plane C
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int a = 0; a < 4; ++a) P[b][a] = wc[a + 4 * b];
        double R[2][4];  // the two rows b = 2H, 2H+1 owned by this thread
#pragma unroll
        for (int bb = 0; bb < 2; ++bb)
#pragma unroll
            for (int a = 0; a < 4; ++a) R[bb][a] = H ? P[2 + bb][a] : P[bb][a];
#pragma unroll
        for (int bb = 0; bb < 2; ++bb)
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                double sx = 0.0, sy = 0.0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    sx += op.D[a * 4 + k] * R[bb][k];
                    sy += Db[bb][k] * P[k][a];
                }
                acc[bb][a] = ax * sx + ay * sy;
            }
        // x faces (entry b + 4C at (b, C)) and y faces (entry a + 4C at (a, C))
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const int tps = side ? tp1 : tp0, tpo = side ? tp0 : tp1;
            const int mx = mode[side], my = mode[2 + side];
            const double sgx = g[3 + side], sgy = g[5 + side];
#pragma unroll
            for (int bb = 0; bb < 2; ++bb) {
                const int b = 2 * H + bb;
                const double nb = mx >= 2 ? plane_nbr(W, halo, halo_stride, nloc[side], hslot[side], b + 4 * C,
                                                      tpo + 4 * b + 16 * C, nin, cin0)
                                          : 0.0;
                const double f = plane_flux(mx, sgx, R[bb][tps], nb);
#pragma unroll
                for (int a = 0; a < 4; ++a) acc[bb][a] -= op.L[side][a] * f;
            }
            const double lb0 = sL[side * 4 + 2 * H], lb1 = sL[side * 4 + 2 * H + 1];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const double nb = my >= 2 ? plane_nbr(W, halo, halo_stride, nloc[2 + side], hslot[2 + side],
                                                      a + 4 * C, a + 4 * tpo + 16 * C, nin, cin0)
                                          : 0.0;
                const double f = plane_flux(my, sgy, P[tps][a], nb);
                acc[0][a] -= lb0 * f;
                acc[1][a] -= lb1 * f;
            }
        }
    }
    // z derivative over the planes, then z faces (entry a + 4b at (a, b))
    const double lc0 = sL[C], lc1 = sL[4 + C];
    const int mz0 = mode[4], mz1 = mode[5];
#pragma unroll
    for (int bb = 0; bb < 2; ++bb) {
        const int b = 2 * H + bb;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            double sz = 0.0, z0 = 0.0, z1 = 0.0;
#pragma unroll
            for (int c2 = 0; c2 < 4; ++c2) {
                const double v = w[16 * c2 + a + 4 * b];
                sz += Dc[c2] * v;
                if (c2 == tp0) z0 = v;
                if (c2 == tp1) z1 = v;
            }
            double r = acc[bb][a] + az * sz;
            const double n0 = mz0 >= 2 ? plane_nbr(W, halo, halo_stride, nloc[4], hslot[4], a + 4 * b,
                                                   a + 4 * b + 16 * tp1, nin, cin0)
                                       : 0.0;
            const double n1 = mz1 >= 2 ? plane_nbr(W, halo, halo_stride, nloc[5], hslot[5], a + 4 * b,
                                                   a + 4 * b + 16 * tp0, nin, cin0)
                                       : 0.0;
            r -= lc0 * plane_flux(mz0, g[7], z0, n0);
            r -= lc1 * plane_flux(mz1, g[8], z1, n1);
            acc[bb][a] = r;
        }
    }
    if (kout) {
        double2 *dst = reinterpret_cast<double2 *>(kout + 16 * C + 8 * H);
        dst[0] = make_double2(acc[0][0], acc[0][1]);
        dst[1] = make_double2(acc[0][2], acc[0][3]);
        dst[2] = make_double2(acc[1][0], acc[1][1]);
        dst[3] = make_double2(acc[1][2], acc[1][3]);
    }
    if (ks) {
#pragma unroll
        for (int bb = 0; bb < 2; ++bb)
#pragma unroll
            for (int a = 0; a < 4; ++a) ks[16 * C + 8 * H + 4 * bb + a] = acc[bb][a];
    }
}

__global__ void __launch_bounds__(PlaneShape::THREADS, 1)
    tensor_plane(const StageIO io, const PlaneArgs pa, const PlaneOps op) {
    using S = PlaneShape;
    constexpr int TE = S::TE, NB = S::NB, ES = S::ES, TV = S::TILE_VEC_BYTES;
    extern __shared__ __align__(128) unsigned char plane_smem_raw[];
    unsigned char *smem = plane_smem_raw;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem);             // [nbuf <= 8], bytes 0..63
    unsigned char *ring = smem + 256;  // bytes 64..255: operator tables
    double *W = reinterpret_cast<double *>(ring + (size_t)pa.nbuf * pa.slot_bytes);  // [TE][ES]
    double *KS = W + TE * ES;                                                         // [TE][ES]
    double *sD = reinterpret_cast<double *>(smem + 64);  // 16 + 8 doubles: D, lifts (fits before the ring)
    // per slot: vectors [nv][TE*NB], geometry [TE][136], halo [halo_slots][stride]
    const int halo_stride = pa.nhv * 16 + 2;

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int el = tid & 31;
    const int nin = io.nin, nfin = io.nfin;
    const int64_t my_tiles = (pa.n_tiles - blockIdx.x + gridDim.x - 1) / gridDim.x;
    if (my_tiles <= 0) return;

    if (tid == 0) {
        for (int s = 0; s < pa.nbuf; ++s) ptx::mbar_init(&mbar[s], 1);
        ptx::fence_mbar_init();
    }
    if (tid < 16) sD[tid] = op.D[tid];
    if (tid >= 16 && tid < 24) sD[tid] = op.L[(tid - 16) / 4][(tid - 16) % 4];
    __syncthreads();
    const double *sL = sD + 16;

    auto vec_ptr = [&](int v) -> const double * { return pa.lv[v]; };
    auto slot_of = [&](int64_t j) { return ring + (size_t)(j % pa.nbuf) * pa.slot_bytes; };
    auto issue = [&](int64_t j) {  // thread 0: bulk loads of local tile j
        const int64_t tile = blockIdx.x + j * gridDim.x;
        const int slot = (int)(j % pa.nbuf);
        unsigned char *dst = slot_of(j);
        const uint32_t bytes = (uint32_t)pa.nv * TV + S::TILE_GEO_BYTES;
        ptx::mbar_arrive_expect_tx(&mbar[slot], bytes);
        for (int v = 0; v < pa.nv; ++v)
            ptx::bulk_load(dst + (size_t)v * TV, vec_ptr(v) + tile * TE * NB, TV, &mbar[slot]);
        ptx::bulk_load(dst + (size_t)pa.nv * TV, pa.geo + tile * S::TILE_GEO_BYTES, S::TILE_GEO_BYTES, &mbar[slot]);
    };
    auto wait_slot = [&](int64_t j) -> bool {
        const int slot = (int)(j % pa.nbuf);
        const uint32_t parity = (uint32_t)((j / pa.nbuf) & 1);
        for (uint32_t it = 0; it < kWaitPolls; ++it)
            if (ptx::mbar_try_wait(&mbar[slot], parity)) return true;
        return false;
    };
    // halo gathers of local tile j into its slot (all threads; cp.async group)
    auto gather = [&](int64_t j) {
        const int64_t tile = blockIdx.x + j * gridDim.x;
        double *halo = reinterpret_cast<double *>(slot_of(j) + (size_t)pa.nv * TV + S::TILE_GEO_BYTES);
        const int p0 = pa.plan_off[tile], p1 = pa.plan_off[tile + 1];
        // work items: (entry, vector, chunk) with 8 chunks of 16 B (y, z) or 16 of 8 B (x)
        const int per_entry = pa.nhv * 16;
        for (int w = tid; w < (p1 - p0) * per_entry; w += S::THREADS) {
            const int64_t ent = pa.plan[p0 + w / per_entry];
            const int r = w % per_entry, v = r / 16, k = r % 16;
            const int64_t n = ent & 0xffffffffll;
            const int slice = (int)((ent >> 32) & 0xff), hs = (int)((ent >> 40) & 0xffff);
            const int axis = slice >> 1, side = slice & 1;
            const int tp = pa.trace_pos[side];
            const double *src = vec_ptr(v) + n * NB;
            double *dst = halo + hs * halo_stride + v * 16;
            if (axis == 0) {  // x slice: entry m = b + 4c at tp + 4b + 16c, 8-byte copies
                ptx::cp_async8(dst + k, src + tp + 4 * (k & 3) + 16 * (k >> 2));
            } else if (k < 8) {
                if (axis == 1)  // y slice: entry m = a + 4c, runs of 4 at 4 tp + 16 c
                    ptx::cp_async16(dst + 2 * k, src + 4 * tp + 16 * (k >> 1) + 2 * (k & 1));
                else  // z slice: 16 contiguous at 16 tp
                    ptx::cp_async16(dst + 2 * k, src + 16 * tp + 2 * k);
            }
        }
        ptx::cp_async_commit();
    };

    if (tid == 0) {
        ptx::fence_proxy_async();
        for (int64_t j = 0; j < my_tiles && j < pa.nbuf; ++j) issue(j);
    }
    bool ok = wait_slot(0);
    if (__syncthreads_or(!ok)) {
        if (tid == 0) atomicOr(io.status, 2);
        return;
    }
    gather(0);

    for (int64_t j = 0; j < my_tiles; ++j) {
        const int64_t tile = blockIdx.x + j * gridDim.x;
        const int64_t e0 = tile * TE;
        const unsigned char *slot = slot_of(j);
        const double *ru = reinterpret_cast<const double *>(slot);
        const unsigned char *geo = slot + (size_t)pa.nv * TV;
        const double *halo = reinterpret_cast<const double *>(geo + S::TILE_GEO_BYTES);

        // 1. stage input into the padded tile
        for (int i = tid; i < TE * NB; i += S::THREADS) {
            double w = ru[i];
            for (int v = 0; v < nin; ++v) w += io.cin[v] * reinterpret_cast<const double *>(slot + (size_t)(1 + v) * TV)[i];
            W[(i >> 6) * ES + (i & 63)] = w;
        }
        ptx::cp_async_wait_all();  // this tile's halo gathers (issued one tile ago)
        __syncthreads();
        // 2. next tile: its bulk data, then its halo gathers (overlap this tile's work)
        if (j + 1 < my_tiles) {
            ok = wait_slot(j + 1);
            if (ok) gather(j + 1);
        }

        // 3. half-plane of this thread
        {
            const unsigned char *g = geo + el * S::GEO_BYTES;
            const double cin0 = nin >= 1 ? io.cin[0] : 0.0;
            double *kdst = io.kout ? io.kout + (e0 + el) * NB : nullptr;
            double *ks = io.unew ? KS + el * ES : nullptr;
            plane_compute(op, sD, sL, W, g, halo, halo_stride, el, warp & 3, warp >> 2, nin, cin0, kdst, ks);
        }
        if (__syncthreads_or(!ok)) break;

        // 4. final stage: u_new = u + sum_j dt b_j k_j + dt b_S k_S, in coefficient order
        if (io.unew) {
            for (int i = tid; i < TE * NB; i += S::THREADS) {
                double r = ru[i];
                for (int v = 0; v < nfin; ++v)
                    r += io.bfin[v] * reinterpret_cast<const double *>(slot + (size_t)pa.fin_idx[v] * TV)[i];
                r += io.blast * KS[(i >> 6) * ES + (i & 63)];
                io.unew[e0 * NB + i] = r;
            }
            __syncthreads();
        }
        // 5. refill the slot just consumed
        if (tid == 0 && j + pa.nbuf < my_tiles) {
            ptx::fence_proxy_async();
            issue(j + pa.nbuf);
        }
    }
    ptx::cp_async_wait_all();
    if (!ok && tid == 0) atomicOr(io.status, 2);
}

}  // namespace hgg
