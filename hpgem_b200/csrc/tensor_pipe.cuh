// Persistent, TMA-fed variant of the sum-factorised hypercube stage kernel.
//
// Same arithmetic as tensor_stage (dg_kernels.cuh); what changes is how the
// data reaches the SM:
//   * each block walks a strided list of tiles of TE consecutive elements;
//   * one thread issues bulk asynchronous copies (cp.async.bulk, the
//     non-tensor TMA path) of the tile's slice of every input vector plus its
//     packed geometry records into a ring of NBUF shared-memory slots, each
//     guarded by an mbarrier with a transaction count, so several tiles of
//     loads are in flight per SM while the current tile is computed;
//   * the neighbour face traces a tile needs (single coefficients of other
//     elements, scattered in memory) are gathered into registers one tile
//     ahead, so their latency overlaps the current tile's work;
//   * every thread computes one x-pencil (NP coefficients) of one element,
//     reusing the pencil's values for the x-derivative and reading only
//     warp-uniform or bank-disjoint entries of the 1D operators;
//   * results are staged in shared memory (hpGEM order) and written back with
//     bulk asynchronous stores.
// Every wait on an mbarrier is bounded; a wait that runs out sets bit 1 of the
// status word and the block stops after draining its own copies: it waits
// (bounded again) for every tile load it issued and not yet consumed, and for
// its bulk stores, so that no asynchronous copy targets the block's shared
// memory after it has exited.
#pragma once

#include <cstdint>

#include "dg_kernels.cuh"

namespace hgg {

namespace ptx {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bulk global -> shared copy completing on `bar`; 16-byte aligned, size % 16 == 0
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void bulk_store(void *dst, const void *src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

__device__ __forceinline__ void bulk_wait_read_all() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

}  // namespace ptx

// upper bound on try_wait polls of one mbarrier before the kernel gives up
constexpr uint32_t kWaitPolls = 1u << 22;

template <int P, int DIM>
struct PipeShape {
    static constexpr int NP = P + 1;
    static constexpr int NB = DIM == 2 ? NP * NP : NP * NP * NP;
    static constexpr int NF = NB / NP;  // x-pencils per element = trace entries per face
    static constexpr int NS = 2 * DIM;
    static constexpr int TE0 = 256 / NF;
    static constexpr int TE = (TE0 * NB) % 2 == 0 ? TE0 : TE0 - 1;  // tile bytes multiple of 16
    static constexpr int THREADS = TE * NF;
    // packed per-element geometry: ahat[DIM], sigma[NS] (double), nbr[NS] (int32), mode[NS] (int8)
    static constexpr int GEO_RAW = 8 * (DIM + NS) + 4 * NS + NS;
    static constexpr int GEO_BYTES = (GEO_RAW + 15) / 16 * 16;
    static constexpr int TILE_VEC_BYTES = TE * NB * 8;
    static constexpr int TILE_GEO_BYTES = TE * GEO_BYTES;
    static constexpr int GMAX = 2;  // u + one stage vector gathered ahead
};

struct PipeArgs {
    const unsigned char *geo;  // [E_pad][GEO_BYTES]
    int64_t n_tiles;
    int nbuf;                   // ring slots
    int nv;                     // vectors loaded per tile: u, kin[0..nin), kfin[0..nfin)
    uint32_t slot_bytes;
    uint32_t polls;             // try_wait polls of one mbarrier before giving up (kWaitPolls)
    int32_t arm_only;           // test of the bounded wait: this local tile's mbarrier is armed with
                                // the slot's byte count but no copy is issued (-1: off)
};

template <int P, int DIM>
__global__ void __launch_bounds__(PipeShape<P, DIM>::THREADS)
    tensor_pipe(const StageIO io, const PipeArgs pa, const TensorConsts<P, DIM> tc) {
    using S = PipeShape<P, DIM>;
    constexpr int NP = S::NP, NB = S::NB, NF = S::NF, NS = S::NS, TE = S::TE;
    constexpr int TV = S::TILE_VEC_BYTES;
    extern __shared__ __align__(128) unsigned char pipe_smem_raw[];
    unsigned char *smem = pipe_smem_raw;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem);  // [nbuf] (<= 8)
    double *sD1 = reinterpret_cast<double *>(smem + 64);
    double *slift = sD1 + NP * NP;
    double *ssign = slift + 2 * NP;
    short *spos = reinterpret_cast<short *>(ssign + NB);
    short *sinv = spos + NB;
    const size_t tab_end = (64 + 8 * (NP * NP + 2 * NP + NB) + 4 * NB + 127) / 128 * 128;
    unsigned char *ring = smem + tab_end;
    double *Wt = reinterpret_cast<double *>(ring + (size_t)pa.nbuf * pa.slot_bytes);  // [TE][NB]
    double *TR = Wt + TE * NB;                                                        // [TE][NS][NF]
    double *outk = TR + TE * NS * NF;                                                 // [TE][NB]
    double *outu = outk + TE * NB;                                                    // [TE][NB]

    const int tid = threadIdx.x;
    const int el = tid / NF;  // element of this thread within the tile
    const int q = tid % NF;   // pencil (b, c) / trace entry of this thread
    const int nin = io.nin, nfin = io.nfin;
    const int64_t my_tiles = (pa.n_tiles - blockIdx.x + gridDim.x - 1) / gridDim.x;
    if (my_tiles <= 0) return;

    for (int i = tid; i < NB; i += blockDim.x) {
        spos[i] = tc.tpos[i];
        sinv[i] = tc.tinv[i];
        ssign[i] = tc.tsign[i];
    }
    if (tid < NP * NP) sD1[tid] = tc.D1[tid];
    if (tid < 2 * NP) slift[tid] = tc.lift[tid];
    if (tid == 0) {
        for (int s = 0; s < pa.nbuf; ++s) ptx::mbar_init(&mbar[s], 1);
        ptx::fence_mbar_init();
    }
    __syncthreads();

    auto vec_ptr = [&](int v) -> const double * {
        return v == 0 ? io.u : (v <= nin ? io.kin[v - 1] : io.kfin[v - 1 - nin]);
    };
    auto issue = [&](int64_t j) {  // thread 0 only: loads of local tile j into its slot
        const int64_t tile = blockIdx.x + j * gridDim.x;
        const int slot = (int)(j % pa.nbuf);
        unsigned char *dst = ring + (size_t)slot * pa.slot_bytes;
        ptx::mbar_arrive_expect_tx(&mbar[slot], pa.slot_bytes);
        if (j == pa.arm_only) return;  // nothing in flight: the wait for this tile runs out
        for (int v = 0; v < pa.nv; ++v)
            ptx::bulk_load(dst + (size_t)v * TV, vec_ptr(v) + tile * TE * NB, TV, &mbar[slot]);
        ptx::bulk_load(dst + (size_t)pa.nv * TV, pa.geo + tile * S::TILE_GEO_BYTES, S::TILE_GEO_BYTES,
                       &mbar[slot]);
    };
    auto wait_slot = [&](int64_t j) -> bool {
        const int slot = (int)(j % pa.nbuf);
        const uint32_t parity = (uint32_t)((j / pa.nbuf) & 1);
        for (uint32_t it = 0; it < pa.polls; ++it)
            if (ptx::mbar_try_wait(&mbar[slot], parity)) return true;
        return false;
    };
    // after a wait ran out: thread 0 waits (bounded) for the loads of local tiles
    // [first, last] that were issued and not consumed, then for its stores
    auto drain = [&](int64_t first, int64_t last) {
        if (tid != 0) return;
        for (int64_t t = first; t <= last && t < my_tiles; ++t) wait_slot(t);
        ptx::bulk_wait_all();
        atomicOr(io.status, 2);
    };
    auto geo_of = [&](int64_t j, int e_local) -> const unsigned char * {
        return ring + (size_t)(j % pa.nbuf) * pa.slot_bytes + (size_t)pa.nv * TV + (size_t)e_local * S::GEO_BYTES;
    };

    if (tid == 0) {
        ptx::fence_proxy_async();
        for (int64_t j = 0; j < my_tiles && j < pa.nbuf; ++j) issue(j);
    }

    // neighbour trace gathers for a tile, into registers (one tile ahead)
    double G[NS][S::GMAX];
    auto gather = [&](int64_t j) {
        const unsigned char *g = geo_of(j, el);
        const int32_t *nbr = reinterpret_cast<const int32_t *>(g + 8 * (DIM + NS));
        const int8_t *mode = reinterpret_cast<const int8_t *>(g + 8 * (DIM + NS) + 4 * NS);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            G[s][0] = 0.0;
            G[s][1] = 0.0;
            const int md = mode[s];
            if (md == 2 || md == 3) {
                const int32_t n = nbr[s];
                if (n >= 0 && n < io.n_elements) {
                    const int axis = s >> 1, side = s & 1;
                    int c[3] = {0, 0, 0};
                    if (DIM == 2) {
                        c[1 - axis] = q;
                    } else {
                        const int a0 = q % NP, a1 = q / NP;
                        if (axis == 0) { c[1] = a0; c[2] = a1; }
                        else if (axis == 1) { c[0] = a0; c[2] = a1; }
                        else { c[0] = a0; c[1] = a1; }
                    }
                    c[axis] = tc.trace_pos[1 - side];
                    const int pos = c[0] + NP * c[1] + (DIM == 3 ? NP * NP * c[2] : 0);
                    const int hi = sinv[pos];
                    const int64_t idx = (int64_t)n * NB + hi;
                    if (nin <= 1) {
                        G[s][0] = io.u[idx];
                        if (nin == 1) G[s][1] = io.kin[0][idx];
                    } else {
                        G[s][0] = stage_input(io, idx);  // wide tableaux: combine now
                    }
                    if (ssign[hi] < 0) { G[s][0] = -G[s][0]; G[s][1] = -G[s][1]; }
                } else {
                    atomicOr(io.status, 1);
                }
            }
        }
    };

    bool ok = wait_slot(0);
    if (__syncthreads_or(!ok)) {
        drain(0, (int64_t)pa.nbuf - 1);  // tiles 0 .. nbuf-1 were issued
        return;
    }
    gather(0);

    for (int64_t j = 0; j < my_tiles; ++j) {
        const int64_t tile = blockIdx.x + j * gridDim.x;
        const int64_t e0 = tile * TE;
        const unsigned char *slot = ring + (size_t)(j % pa.nbuf) * pa.slot_bytes;
        const double *ru = reinterpret_cast<const double *>(slot);

        // 1. stage input of the tile in tensor order
        for (int i = tid; i < TE * NB; i += S::THREADS) {
            const int l = i / NB, t = i - l * NB;
            double w = ru[i];
            for (int v = 0; v < nin; ++v)
                w += io.cin[v] * reinterpret_cast<const double *>(slot + (size_t)(1 + v) * TV)[i];
            Wt[l * NB + spos[t]] = ssign[t] * w;
        }
        __syncthreads();

        // 2. flux traces of this thread's (element, entry), scaled by sigma
        {
            const unsigned char *g = geo_of(j, el);
            const double *sigma = reinterpret_cast<const double *>(g) + DIM;
            const int8_t *mode = reinterpret_cast<const int8_t *>(g + 8 * (DIM + NS) + 4 * NS);
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const int axis = s >> 1, side = s & 1;
                const int md = mode[s];
                double tself = 0.0;
                if (md == 1 || md == 3) {
                    int c[3] = {0, 0, 0};
                    if (DIM == 2) {
                        c[1 - axis] = q;
                    } else {
                        const int a0 = q % NP, a1 = q / NP;
                        if (axis == 0) { c[1] = a0; c[2] = a1; }
                        else if (axis == 1) { c[0] = a0; c[2] = a1; }
                        else { c[0] = a0; c[1] = a1; }
                    }
                    c[axis] = tc.trace_pos[side];
                    tself = Wt[el * NB + c[0] + NP * c[1] + (DIM == 3 ? NP * NP * c[2] : 0)];
                }
                const double tnbr = (nin == 1) ? G[s][0] + io.cin[0] * G[s][1] : G[s][0];
                const double sg = sigma[s];
                TR[(el * NS + s) * NF + q] =
                    md == 1 ? sg * tself : (md == 2 ? sg * tnbr : (md == 3 ? 0.5 * sg * (tself + tnbr) : 0.0));
            }
        }
        // prefetch the next tile's neighbour traces; the out buffers must be free
        if (j + 1 < my_tiles) {
            ok = wait_slot(j + 1);
            if (ok) gather(j + 1);
        }
        if (tid == 0) ptx::bulk_wait_read_all();
        if (__syncthreads_or(!ok)) {
            drain(j + 1, j - 1 + pa.nbuf);  // issued so far: tiles up to j - 1 + nbuf
            return;
        }

        // 3. x-pencil of this thread: volume + face lifts, output in hpGEM order
        {
            const double *ahat = reinterpret_cast<const double *>(geo_of(j, el));
            const int b = q % NP, c = DIM == 3 ? q / NP : 0;
            const double *wb = Wt + el * NB;
            double wx[NP];
#pragma unroll
            for (int a = 0; a < NP; ++a) wx[a] = wb[a + NP * b + NP * NP * c];
            double acc[NP];
#pragma unroll
            for (int a = 0; a < NP; ++a) {
                double sx = 0.0;
#pragma unroll
                for (int a2 = 0; a2 < NP; ++a2) sx += sD1[a * NP + a2] * wx[a2];
                double sy = 0.0;
#pragma unroll
                for (int b2 = 0; b2 < NP; ++b2) sy += sD1[b * NP + b2] * wb[a + NP * b2 + NP * NP * c];
                double r = ahat[0] * sx + ahat[1] * sy;
                if (DIM == 3) {
                    double sz = 0.0;
#pragma unroll
                    for (int c2 = 0; c2 < NP; ++c2) sz += sD1[c * NP + c2] * wb[a + NP * b + NP * NP * c2];
                    r += ahat[DIM - 1] * sz;
                }
                const double *tr = TR + el * NS * NF;
                r -= slift[a] * tr[0 * NF + q] + slift[NP + a] * tr[1 * NF + q];
                const int my = DIM == 2 ? a : a + NP * c;
                r -= slift[b] * tr[2 * NF + my] + slift[NP + b] * tr[3 * NF + my];
                if (DIM == 3) {
                    const int mz = a + NP * b;
                    r -= slift[c] * tr[4 * NF + mz] + slift[NP + c] * tr[5 * NF + mz];
                }
                acc[a] = r;
            }
#pragma unroll
            for (int a = 0; a < NP; ++a) {
                const int hi = sinv[a + NP * b + NP * NP * c];
                outk[el * NB + hi] = ssign[hi] * acc[a];
            }
        }
        __syncthreads();

        // 4. final stage: u_new = u + sum_j dt b_j k_j (+ this stage)
        if (io.unew) {
            for (int i = tid; i < TE * NB; i += S::THREADS) {
                double r = ru[i];
                for (int v = 0; v < nfin; ++v)
                    r += io.bfin[v] * reinterpret_cast<const double *>(slot + (size_t)(1 + nin + v) * TV)[i];
                outu[i] = r + io.blast * outk[i];
            }
        }
        ptx::fence_proxy_async();
        __syncthreads();

        // 5. write back; refill the slot just consumed
        if (tid == 0) {
            if (io.kout) ptx::bulk_store(io.kout + e0 * NB, outk, TV);
            if (io.unew) ptx::bulk_store(io.unew + e0 * NB, outu, TV);
            ptx::bulk_commit();
            if (j + pa.nbuf < my_tiles) issue(j + pa.nbuf);
        }
    }
    if (tid == 0) ptx::bulk_wait_all();
}

}  // namespace hgg
