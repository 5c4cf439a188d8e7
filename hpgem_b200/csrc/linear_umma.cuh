// Grouped stored-matrix stage on the fifth-generation tensor cores (tcgen05,
// sm_100a) for the mixed precision forms.
//
// The stage of a tile of 128 elements that share their matrices (one matrix
// per slot: the element itself, then its neighbour slots) is
//   Out[e][n] = sum_s sum_k W_s[e][k] A_s[n][k],
// W_s[e] the stage input of element e (s = 0) or of its neighbour in slot s,
// A_s the folded matrix (mass inverse times stiffness blocks,
// HpgemAPILinear_Impl.h:360-434 with :143-156).  That is one MMA chain with
// M = 128 elements, N = R output rows, K = R per slot, accumulated in FP32 in
// tensor memory.  Two forms:
//   TF32 (the FP32-mixed form): every operand x is split into hi = x with the
//     low 13 mantissa bits cleared (exact in TF32) and lo = x - hi, and the
//     product is hi*hi + hi*lo + lo*hi (three kind::tf32 MMAs), close to an
//     FP32 product (the dropped lo*lo and the truncation of lo are ~2^-21 of
//     the product);
//   BF16 (the split-BF16 form): hi = bf16(x), lo = bf16(x - hi), the same
//     three products with kind::f16 (BF16 inputs, FP32 accumulate), ~2^-17 of
//     the product.
// The stage input is formed in FP64 from the FP64 solution and the FP32 stage
// vectors and split once; the matrices are split on the host into operand
// images laid out exactly as shared memory holds them, so one bulk copy per
// slot brings them in.  The solution update u + sum_j dt b_j k_j stays FP64.
//
// Organisation: a persistent CTA of 16 warps walks tiles.  Per tile it stages
// the source element of every (slot, row) in shared memory; for every (tile,
// slot) item it bulk-copies the slot's matrix image and gathers + splits the
// 128 input rows (each thread with four 16-byte chunks of loads in flight)
// into one of two shared-memory buffers while the MMAs of the previous item
// run; one thread issues the MMAs and commits them to the buffer's mbarrier.
// After the last slot the warps read the accumulator rows back (warp w owns
// tensor-memory lanes 32 (w % 4) .. + 31, lane = element, and every fourth
// group of 8 columns) into shared memory, then write k and, in the final
// stage, the new solution one element row per warp (coalesced).
//
// Shared-memory operands use the K-major layout without swizzle: core matrices
// of 8 rows x 16 bytes stored as 128 contiguous bytes, the two 16-byte K
// chunks of one MMA 128 bytes apart (leading byte offset), row groups of 8
// KP * element-size * 8 bytes apart (stride byte offset).
//
// Every wait is bounded; a wait that runs out sets bit 1 of the status word,
// and the CTA then waits (bounded again) for its own copies and MMAs in flight
// and frees its tensor memory before it returns.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

#include "dg_kernels.cuh"

namespace hgg {

enum UmmaKind { kUmmaTF32 = 0, kUmmaBF16 = 1 };
constexpr int kUmmaTileN = 128;    // elements per tile = MMA M
constexpr int kUmmaThreads = 512;  // 16 warps; warp w reads tensor-memory lanes 32(w%4)..32(w%4)+31
constexpr uint32_t kUmmaPolls = 1u << 22;

struct UmmaShape {
    int R;               // rows (coefficients) per element
    int NP;              // R rounded up to 16: MMA N
    int KP;              // R rounded up to the MMA K (8 for TF32, 16 for BF16)
    int es;              // bytes per operand element (4 TF32, 2 BF16)
    int W;               // matrix slots per element (self + neighbour slots)
    int slots;           // neighbour slots
    uint32_t a_bytes;    // one part (hi or lo) of the gathered operand: 128 x KP
    uint32_t b_bytes;    // one part of a matrix image: NP x KP
    uint32_t tmem_cols;  // power of two >= NP, >= 32
};

__host__ __device__ inline UmmaShape umma_shape(int R, int slots, int kind) {
    UmmaShape s;
    s.R = R;
    s.slots = slots;
    s.W = slots + 1;
    s.NP = (R + 15) / 16 * 16;
    const int kstep = kind == kUmmaTF32 ? 8 : 16;
    s.KP = (R + kstep - 1) / kstep * kstep;
    s.es = kind == kUmmaTF32 ? 4 : 2;
    s.a_bytes = (uint32_t)(kUmmaTileN * s.KP * s.es);
    s.b_bytes = (uint32_t)(s.NP * s.KP * s.es);
    uint32_t c = 32;
    while (c < (uint32_t)s.NP) c <<= 1;
    s.tmem_cols = c;
    return s;
}

// dynamic shared memory: barriers and the tensor-memory address in the first
// 1 KB, the tile's source elements [W][128] (int32), then two buffers of
// (A hi, A lo, B hi, B lo)
__host__ __device__ inline size_t umma_src_bytes(const UmmaShape &s) {
    return ((size_t)s.W * kUmmaTileN * 4 + 1023) / 1024 * 1024;
}
// the accumulator tile staged for the epilogue: 128 rows of NP + 4 floats (the
// pad keeps the rows' 16-byte stores on distinct banks); it reuses the operand
// buffers, and extends them where they are smaller
__host__ __device__ inline size_t umma_stage_bytes(const UmmaShape &s) { return (size_t)kUmmaTileN * (s.NP + 4) * 4; }
__host__ __device__ inline size_t umma_smem(const UmmaShape &s) {
    const size_t bufs = 2 * (2 * (size_t)s.a_bytes + 2 * (size_t)s.b_bytes);
    const size_t st = umma_stage_bytes(s);
    return 1024 + umma_src_bytes(s) + (bufs > st ? bufs : st);
}

// byte offset of operand element (row, k) in the core-matrix layout
__host__ __device__ inline uint32_t umma_offset(int row, int k, int KP, int es) {
    const int per16 = 16 / es;
    return (uint32_t)((row >> 3) * (KP * es * 8) + (k / per16) * 128 + (row & 7) * 16 + (k % per16) * es);
}

// instruction descriptor: D FP32, A and B K-major, M = 128, N = np
__host__ __device__ inline uint32_t umma_idesc(int kind, int np) {
    const uint32_t fmt = kind == kUmmaTF32 ? 2u : 1u;  // TF32 = 2, BF16 = 1
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(np >> 3) << 17) | ((uint32_t)(kUmmaTileN >> 4) << 24);
}

struct UmmaArgs {
    const unsigned char *img;   // [n_mats][2][NP x KP] matrix operand images (hi, lo)
    const int32_t *tile_elems;  // [n_tiles][128], -1: padding
    const int32_t *tile_mats;   // [n_tiles][W]: matrix of each slot (-1: slot unused)
    const int32_t *nbr;         // [E][slots] neighbour of each slot, -1: none
    int64_t n_tiles;
    int n_mats;
    uint32_t polls;  // bounded waits: try_wait polls of one mbarrier
};

namespace umma {

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100; base offset 0, no swizzle
    return d;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool wait_bounded(uint64_t *bar, uint32_t parity, uint32_t polls) {
    for (uint32_t i = 0; i < polls; ++i)
        if (try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(cols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

template <int KIND>
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    if constexpr (KIND == kUmmaTF32) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(da), "l"(db), "r"(idesc), "r"(acc)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(da), "l"(db), "r"(idesc), "r"(acc)
            : "memory");
    }
}
__device__ __forceinline__ void commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void ld_x8(uint32_t taddr, float *v) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// hi / lo parts of x for the operand type: TF32 (FP32 containers, hi exact in
// TF32) or BF16
__device__ __forceinline__ void split_tf32(double x, uint32_t &hi, uint32_t &lo) {
    const uint32_t h = __float_as_uint((float)x) & 0xFFFFE000u;
    hi = h;
    lo = __float_as_uint((float)(x - (double)__uint_as_float(h)));
}
__device__ __forceinline__ void split_bf16(double x, uint16_t &hi, uint16_t &lo) {
    const __nv_bfloat16 h = __float2bfloat16_rn((float)x);
    const __nv_bfloat16 l = __float2bfloat16_rn((float)(x - (double)__bfloat162float(h)));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
}

}  // namespace umma

// The tiles one CTA walks: tile vt = blockIdx.x, + gridDim.x, ... of `total`,
// each with its stage inputs and arguments (get() false: skip the tile).
struct UmmaOneProblem {
    StageIOT<float> io;
    UmmaArgs a;
    __device__ int64_t total() const { return a.n_tiles; }
    __device__ bool get(int64_t vt, StageIOT<float> &tio, UmmaArgs &ta, int64_t &tile) const {
        tio = io;
        ta = a;
        tile = vt;
        return true;
    }
};

// NIN: stage-input vectors the kernel reads with vector loads (0 or 1, the RK4
// stages; rows 16-byte aligned, R a multiple of 4); -1: any count, scalar loads
template <int KIND, int NIN, typename Src>
__device__ __forceinline__ void umma_persistent(const UmmaShape &sh, const Src &tiles, int *status) {
    extern __shared__ __align__(1024) unsigned char umma_raw[];
    uint64_t *b_full = reinterpret_cast<uint64_t *>(umma_raw);  // [2] matrix image landed
    uint64_t *mma_done = b_full + 2;                             // [2] MMAs reading the buffer done
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(umma_raw + 64);
    int *fail_flag = reinterpret_cast<int *>(umma_raw + 128);
    int32_t *src_ids = reinterpret_cast<int32_t *>(umma_raw + 1024);  // [W][128] source element per slot, row
    unsigned char *ops = umma_raw + 1024 + umma_src_bytes(sh);
    const uint32_t buf_bytes = 2 * sh.a_bytes + 2 * sh.b_bytes;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int per16 = KIND == kUmmaTF32 ? 4 : 8;  // operand elements per 16-byte chunk
    constexpr int GB = KIND == kUmmaTF32 ? 4 : 2;      // gather items (16-byte chunks) per thread in flight
    constexpr bool FAST = NIN >= 0;
    const int cpr = sh.KP / per16;                     // chunks per row
    const int items = kUmmaTileN * cpr;
    const uint32_t sbo = (uint32_t)sh.KP * sh.es * 8;  // bytes between row groups of 8
    const int ksteps = sh.KP / (KIND == kUmmaTF32 ? 8 : 16);
    const uint32_t idesc = umma_idesc(KIND, sh.NP);

    if (tid == 0) {
        for (int i = 0; i < 2; ++i) {
            umma::mbar_init(&b_full[i], 1);
            umma::mbar_init(&mma_done[i], 1);
        }
        umma::fence_mbar_init();
        *fail_flag = 0;
    }
    if (warp == 0) {
        umma::tmem_alloc(tmem_slot, sh.tmem_cols);
        umma::tmem_relinquish();
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    // this thread's gather items are the same for every (tile, slot): their row, first
    // column and shared-memory offset, computed once
    const int n_base = (items + kUmmaThreads * GB - 1) / (kUmmaThreads * GB);
    auto item_of = [&](int bi, int g, int &row, int &k0, uint32_t &off) {
        const int it = bi * kUmmaThreads * GB + g * kUmmaThreads + tid;
        const int m8 = it & 7, rest = it >> 3;
        const int c = rest % cpr;
        const bool in = it < items;
        row = in ? (rest / cpr) * 8 + m8 : -1;
        k0 = c * per16;
        off = in ? umma_offset(row, k0, sh.KP, sh.es) : 0u;
    };
    int p_row[GB], p_k0[GB];  // the first base iteration (all of it for R <= 64)
    uint32_t p_off[GB];
#pragma unroll
    for (int g = 0; g < GB; ++g) item_of(0, g, p_row[g], p_k0[g], p_off[g]);

    uint32_t q = 0;  // (tile, slot) items of this CTA so far
    int64_t last_copy = -1, last_commit = -1;
    bool ok = true;
    for (int64_t vt = blockIdx.x; vt < tiles.total() && ok; vt += gridDim.x) {
        StageIOT<float> io;
        UmmaArgs a;
        int64_t tile;
        if (!tiles.get(vt, io, a, tile)) continue;
        // source element of every (slot, row): the element itself, then its neighbours
        for (int i = tid; i < sh.W * kUmmaTileN; i += kUmmaThreads) {
            const int s = i / kUmmaTileN, row = i % kUmmaTileN;
            const int32_t e = a.tile_elems[tile * kUmmaTileN + row];
            int32_t src = -1;
            if (e >= 0 && e < io.n_elements) {
                if (s == 0) src = e;
                else {
                    const int32_t n = a.nbr[(int64_t)e * sh.slots + s - 1];
                    if (n >= 0 && n < io.n_elements) src = n;
                    else if (n >= io.n_elements) atomicOr(io.status, 1);
                }
            }
            src_ids[i] = src;
        }
        __syncthreads();
        for (int s = 0; s < sh.W && ok; ++s, ++q) {
            const int buf = q & 1;
            unsigned char *A_hi = ops + (size_t)buf * buf_bytes, *A_lo = A_hi + sh.a_bytes;
            unsigned char *B_hi = A_lo + sh.a_bytes;
            const int32_t mat = a.tile_mats[tile * sh.W + s];
            const bool used = mat >= 0 && mat < a.n_mats;
            // the MMAs of item q - 2 read this buffer
            // (one thread polls; the block barrier below releases the others)
            if (tid == 0 && q >= 2 && !umma::wait_bounded(&mma_done[buf], ((q - 2) >> 1) & 1, a.polls))
                *fail_flag = 1;
            if (__syncthreads_or(*fail_flag)) {
                ok = false;
                break;
            }
            if (tid == 0) {
                if (mat >= a.n_mats) atomicOr(io.status, 4);
                umma::arrive_expect_tx(&b_full[buf], used ? 2 * sh.b_bytes : 0);
                if (used) umma::bulk_load(B_hi, a.img + (size_t)mat * 2 * sh.b_bytes, 2 * sh.b_bytes, &b_full[buf]);
                last_copy = q;
            }
            // gather the slot's 128 input rows, split them, store them in the core-matrix
            // layout; every load of GB items is issued before any is used
            const int32_t *srow = src_ids + s * kUmmaTileN;
            for (int bi = 0; bi < n_base; ++bi) {
                int g_row[GB], g_k0[GB];
                uint32_t g_off[GB];
#pragma unroll
                for (int g = 0; g < GB; ++g) {
                    if (bi == 0) {
                        g_row[g] = p_row[g];
                        g_k0[g] = p_k0[g];
                        g_off[g] = p_off[g];
                    } else {
                        item_of(bi, g, g_row[g], g_k0[g], g_off[g]);
                    }
                }
                double x[GB][per16];
                int row_of[GB];
                if (FAST) {
                    double2 uv[GB][per16 / 2];
                    float4 kv[GB][NIN > 0 ? per16 / 4 : 1];
                    bool live[GB];
#pragma unroll
                    for (int g = 0; g < GB; ++g) {
                        const int row = g_row[g], k0 = g_k0[g];
                        row_of[g] = row;
                        const int32_t src = (row >= 0 && used) ? srow[row] : -1;
                        live[g] = src >= 0 && k0 + per16 <= sh.R;
                        const int64_t i0 = live[g] ? (int64_t)src * sh.R + k0 : 0;  // a safe address
#pragma unroll
                        for (int j = 0; j < per16 / 2; ++j) uv[g][j] = __ldg(reinterpret_cast<const double2 *>(io.u + i0) + j);
                        if constexpr (NIN > 0) {
#pragma unroll
                            for (int j = 0; j < per16 / 4; ++j)
                                kv[g][j] = __ldg(reinterpret_cast<const float4 *>(io.kin[0] + i0) + j);
                        }
                    }
#pragma unroll
                    for (int g = 0; g < GB; ++g) {
#pragma unroll
                        for (int j = 0; j < per16 / 2; ++j) {
                            x[g][2 * j] = live[g] ? uv[g][j].x : 0.0;
                            x[g][2 * j + 1] = live[g] ? uv[g][j].y : 0.0;
                        }
                        if constexpr (NIN > 0) {
                            const double cn = io.cin[0];
#pragma unroll
                            for (int j = 0; j < per16 / 4; ++j) {
                                x[g][4 * j] += live[g] ? cn * (double)kv[g][j].x : 0.0;
                                x[g][4 * j + 1] += live[g] ? cn * (double)kv[g][j].y : 0.0;
                                x[g][4 * j + 2] += live[g] ? cn * (double)kv[g][j].z : 0.0;
                                x[g][4 * j + 3] += live[g] ? cn * (double)kv[g][j].w : 0.0;
                            }
                        }
                    }
                } else {
#pragma unroll
                    for (int g = 0; g < GB; ++g) {
                        const int row = g_row[g], k0 = g_k0[g];
                        row_of[g] = row;
                        const int32_t src = (row >= 0 && used) ? srow[row] : -1;
#pragma unroll
                        for (int j = 0; j < per16; ++j) {
                            const int k = k0 + j;
                            x[g][j] = (src >= 0 && k < sh.R) ? stage_input(io, (int64_t)src * sh.R + k) : 0.0;
                        }
                    }
                }
#pragma unroll
                for (int g = 0; g < GB; ++g) {
                    if (row_of[g] < 0) continue;
                    const uint32_t off = g_off[g];
                    if constexpr (KIND == kUmmaTF32) {
                        uint32_t h[4], l[4];
#pragma unroll
                        for (int j = 0; j < 4; ++j) umma::split_tf32(x[g][j], h[j], l[j]);
                        *reinterpret_cast<uint4 *>(A_hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
                        *reinterpret_cast<uint4 *>(A_lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
                    } else {
                        uint16_t h[8], l[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) umma::split_bf16(x[g][j], h[j], l[j]);
                        uint4 hv, lv;
                        hv.x = h[0] | ((uint32_t)h[1] << 16);
                        hv.y = h[2] | ((uint32_t)h[3] << 16);
                        hv.z = h[4] | ((uint32_t)h[5] << 16);
                        hv.w = h[6] | ((uint32_t)h[7] << 16);
                        lv.x = l[0] | ((uint32_t)l[1] << 16);
                        lv.y = l[2] | ((uint32_t)l[3] << 16);
                        lv.z = l[4] | ((uint32_t)l[5] << 16);
                        lv.w = l[6] | ((uint32_t)l[7] << 16);
                        *reinterpret_cast<uint4 *>(A_hi + off) = hv;
                        *reinterpret_cast<uint4 *>(A_lo + off) = lv;
                    }
                }
            }
            umma::fence_proxy_async();  // generic-proxy stores -> visible to the tensor cores
            __syncthreads();
            if (tid == 0) {
                if (!umma::wait_bounded(&b_full[buf], (q >> 1) & 1, a.polls)) {
                    *fail_flag = 1;
                } else if (used) {
                    umma::fence_after_sync();
                    const uint32_t a_hi = umma::smem_addr(A_hi), a_lo = umma::smem_addr(A_lo);
                    const uint32_t b_hi = umma::smem_addr(B_hi), b_lo = b_hi + sh.b_bytes;
                    for (int ks = 0; ks < ksteps; ++ks) {
                        const uint32_t o = (uint32_t)ks * 256;  // two 16-byte K chunks per step
                        const uint64_t dah = umma::desc_kmajor(a_hi + o, 128, sbo);
                        const uint64_t dal = umma::desc_kmajor(a_lo + o, 128, sbo);
                        const uint64_t dbh = umma::desc_kmajor(b_hi + o, 128, sbo);
                        const uint64_t dbl = umma::desc_kmajor(b_lo + o, 128, sbo);
                        const uint32_t first = (s == 0 && ks == 0) ? 0u : 1u;
                        umma::mma<KIND>(tmem, dah, dbh, idesc, first);
                        umma::mma<KIND>(tmem, dah, dbl, idesc, 1u);
                        umma::mma<KIND>(tmem, dal, dbh, idesc, 1u);
                    }
                } else if (s == 0) {
                    // a tile whose self slot has no matrix: start the accumulator at zero
                    const uint64_t dz = umma::desc_kmajor(umma::smem_addr(A_hi), 128, sbo);
                    umma::fence_after_sync();
                    umma::mma<KIND>(tmem, dz, dz, idesc, 0u);  // A_hi is all zero for this slot
                }
                umma::commit(&mma_done[buf]);
                last_commit = q;
            }
        }
        if (!ok) break;
        // epilogue: wait for the tile's last MMAs, read the accumulator rows back; warp w
        // reads lane quadrant w % 4 (rows 32 (w % 4) + lane), every 4th group of 8 columns
        const uint32_t last = q - 1;
        if (tid == 0) {
            if (!umma::wait_bounded(&mma_done[last & 1], (last >> 1) & 1, a.polls)) *fail_flag = 1;
            if (last >= 1 && !umma::wait_bounded(&mma_done[(last - 1) & 1], ((last - 1) >> 1) & 1, a.polls))
                *fail_flag = 1;
        }
        if (__syncthreads_or(*fail_flag)) {
            ok = false;
            break;
        }
        umma::fence_after_sync();
        {
            // accumulator rows -> shared memory (warp w: lane quadrant w % 4, every fourth
            // group of 8 columns); the operand buffers are free once the MMAs are done
            const int quad = warp & 3, cgrp = warp >> 2;
            const int row = quad * 32 + lane;
            const int LD = sh.NP + 4;
            float *Ds = reinterpret_cast<float *>(ops);
            for (int c8 = cgrp; c8 < sh.NP / 8; c8 += kUmmaThreads / 128) {
                float v[8];
                umma::ld_x8(tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(c8 * 8), v);
                umma::wait_ld();
                *reinterpret_cast<float4 *>(Ds + row * LD + c8 * 8) = make_float4(v[0], v[1], v[2], v[3]);
                *reinterpret_cast<float4 *>(Ds + row * LD + c8 * 8 + 4) = make_float4(v[4], v[5], v[6], v[7]);
            }
            umma::fence_before_sync();
            __syncthreads();
            // one element row per warp at a time: every access below is coalesced along the row
            for (int r = warp; r < kUmmaTileN; r += kUmmaThreads / 32) {
                const int32_t e = src_ids[r];
                if (e < 0) continue;
                for (int n = lane; n < sh.R; n += 32) {
                    const int64_t idx = (int64_t)e * sh.R + n;
                    stage_output(io, idx, io.u[idx], (double)Ds[r * LD + n]);
                }
            }
        }
        __syncthreads();
    }
    if (!ok) {
        // drain what this CTA still has in flight (bounded), then report
        if (tid == 0) {
            if (last_copy >= 0) umma::wait_bounded(&b_full[last_copy & 1], (uint32_t)(last_copy >> 1) & 1, kUmmaPolls);
            for (int64_t i = last_commit - 1; i <= last_commit; ++i)
                if (i >= 0) umma::wait_bounded(&mma_done[i & 1], (uint32_t)(i >> 1) & 1, kUmmaPolls);
            atomicOr(status, 2);
        }
        umma::fence_before_sync();
        __syncthreads();
    }
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, sh.tmem_cols);
    }
}

template <int KIND, int NIN>
__global__ void __launch_bounds__(kUmmaThreads, 1)
    linear_umma_stage(const StageIOT<float> io, const UmmaArgs a, const UmmaShape sh) {
    umma_persistent<KIND, NIN>(sh, UmmaOneProblem{io, a}, io.status);
}

}  // namespace hgg
