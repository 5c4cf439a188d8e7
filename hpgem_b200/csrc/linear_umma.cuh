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
// vectors, once per element and stage, and stored split as two planes (hi,
// lo; a row of KP operand elements per element) by umma_planes.  The matrices
// are split on the host into operand images laid out exactly as shared memory
// holds them, so one bulk copy per slot brings them in.  The solution update
// u + sum_j dt b_j k_j stays FP64.
//
// Organisation: a persistent CTA of 16 warps walks tiles.  Per tile it stages
// the source element of every (slot, row) in shared memory; for every (tile,
// slot) item the threads issue asynchronous 16-byte copies of the 128 source
// rows of both planes straight into a ring of 2 to 4 shared-memory operand
// buffers (as many as fit; a missing neighbour reads as zeros) and one thread
// bulk-copies the slot's matrix image, up to three items ahead of the MMAs;
// one thread issues the MMAs and commits them to the buffer's mbarrier.
// After the last slot the warps read the accumulator rows back (warp w owns
// tensor-memory lanes 32 (w % 4) .. + 31, lane = element, and every fourth
// group of 8 columns) into shared memory, then write k and, in the final
// stage, the new solution one element row per warp (coalesced).
//
// Shared-memory operands use the K-major layout with the 128-byte swizzle:
// panels of 128 bytes of K (32 TF32 or 64 BF16 values) for all rows, a row's
// 128 bytes contiguous with its eight 16-byte chunks permuted by chunk ^ (row
// % 8), 8-row groups 1024 bytes apart (stride byte offset); one MMA's K (32
// bytes) lies inside a panel row, so the K steps advance the descriptor's
// start address by 32 bytes and then by one panel.  The copies of a warp then
// read whole rows (coalesced) and write whole 128-byte rows (no bank conflict).
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
    int KP;              // R rounded up to whole 128-byte panels (32 TF32 / 64 BF16 values)
    int es;              // bytes per operand element (4 TF32, 2 BF16)
    int W;               // matrix slots per element (self + neighbour slots)
    int slots;           // neighbour slots
    int panels;          // KP * es / 128
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
    s.es = kind == kUmmaTF32 ? 4 : 2;
    const int panel = 128 / s.es;
    s.KP = (R + panel - 1) / panel * panel;
    s.panels = s.KP / panel;
    s.a_bytes = (uint32_t)(kUmmaTileN * s.KP * s.es);
    s.b_bytes = (uint32_t)(s.NP * s.KP * s.es);
    uint32_t c = 32;
    while (c < (uint32_t)s.NP) c <<= 1;
    s.tmem_cols = c;
    return s;
}

// dynamic shared memory: barriers and the tensor-memory address in the first
// 1 KB, the tile's source elements [W][128] (int32), then two buffers of
// (A hi, A lo, B hi, B lo); the accumulator tile staged for the epilogue (128
// rows of NP + 4 floats: the pad keeps the rows' 16-byte stores on distinct
// banks) reuses the buffers and extends them where they are smaller
__host__ __device__ inline size_t umma_src_bytes(const UmmaShape &s) {
    return ((size_t)s.W * kUmmaTileN * 4 + 1023) / 1024 * 1024;
}
__host__ __device__ inline size_t umma_stage_bytes(const UmmaShape &s) { return (size_t)kUmmaTileN * (s.NP + 4) * 4; }
// operand buffers of the ring: as many as fit (2 to 4), each (A hi, A lo, B hi, B lo)
__host__ __device__ inline int umma_buffers(const UmmaShape &s) {
    const size_t buf = 2 * (size_t)s.a_bytes + 2 * (size_t)s.b_bytes;
    const size_t room = 227 * 1024 - 1024 - umma_src_bytes(s);
    int nb = (int)(room / buf);
    return nb > 4 ? 4 : (nb < 2 ? 2 : nb);
}
__host__ __device__ inline size_t umma_smem(const UmmaShape &s) {
    const size_t bufs = (size_t)umma_buffers(s) * (2 * (size_t)s.a_bytes + 2 * (size_t)s.b_bytes);
    const size_t st = umma_stage_bytes(s);
    return 1024 + umma_src_bytes(s) + (bufs > st ? bufs : st);
}

// byte offset of operand element (row, k) of a `rows`-row operand in the 128-byte
// swizzle layout
__host__ __device__ inline uint32_t umma_offset(int row, int k, int rows, int es) {
    const int byte = k * es, panel = byte >> 7, within = byte & 127, chunk = within >> 4;
    return (uint32_t)(panel * rows * 128 + row * 128 + ((chunk ^ (row & 7)) << 4) + (within & 15));
}

// instruction descriptor: D FP32, A and B K-major, M = 128, N = np
__host__ __device__ inline uint32_t umma_idesc(int kind, int np) {
    const uint32_t fmt = kind == kUmmaTF32 ? 2u : 1u;  // TF32 = 2, BF16 = 1
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(np >> 3) << 17) | ((uint32_t)(kUmmaTileN >> 4) << 24);
}

struct UmmaArgs {
    const unsigned char *img;     // [n_mats][2][NP x KP] matrix operand images (hi, lo)
    const unsigned char *planes;  // [2][E][KP] split stage input (hi plane, lo plane)
    const int32_t *tile_elems;    // [n_tiles][128], -1: padding
    const int32_t *tile_mats;     // [n_tiles][W]: matrix of each slot (-1: slot unused)
    const int32_t *nbr;           // [E][slots] neighbour of each slot, -1: none
    int64_t n_tiles;
    int n_mats;
    uint32_t polls;  // bounded waits: try_wait polls of one mbarrier
};

namespace umma {

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor of a K-major operand in the 128-byte swizzle
// layout: start address, leading byte offset 16 (unused by this layout), stride
// byte offset 1024 (8 rows of 128 bytes), the sm_100 descriptor version, layout
// type 2 (128-byte swizzle)
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
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
// 16-byte asynchronous copy global -> shared (L2 only); src_bytes 0 fills zeros
__device__ __forceinline__ void cp_async16(void *dst, const void *src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

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

// Split stage input w = u + sum_j cin_j k_j of every element into the hi / lo
// planes (row e: KP operand elements, zero beyond R).  One thread per 16-byte
// chunk of a row: every access is coalesced.  NIN: stage-input vectors read
// with vector loads (0 or 1; R a multiple of 4); -1: any count.
template <int KIND, int NIN>
__device__ __forceinline__ void umma_planes_body(const StageIOT<float> &io, unsigned char *planes, int R, int KP,
                                                 int64_t i) {
    constexpr int per16 = KIND == kUmmaTF32 ? 4 : 8;
    const int cpr = KP / per16;
    const int64_t e = i / cpr;
    const int k0 = (int)(i - e * cpr) * per16;
    const int64_t plane = (int64_t)io.n_elements * KP * (KIND == kUmmaTF32 ? 4 : 2);
    double x[per16];
    if (NIN >= 0 && k0 + per16 <= R) {
        const int64_t i0 = e * R + k0;
#pragma unroll
        for (int j = 0; j < per16; j += 2) {
            const double2 uv = __ldg(reinterpret_cast<const double2 *>(io.u + i0 + j));
            x[j] = uv.x;
            x[j + 1] = uv.y;
        }
        if constexpr (NIN > 0) {
            const double c = io.cin[0];
#pragma unroll
            for (int j = 0; j < per16; j += 4) {
                const float4 kv = __ldg(reinterpret_cast<const float4 *>(io.kin[0] + i0 + j));
                x[j] += c * (double)kv.x;
                x[j + 1] += c * (double)kv.y;
                x[j + 2] += c * (double)kv.z;
                x[j + 3] += c * (double)kv.w;
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < per16; ++j) x[j] = k0 + j < R ? stage_input(io, e * R + k0 + j) : 0.0;
    }
    unsigned char *hi = planes + (e * KP + k0) * (KIND == kUmmaTF32 ? 4 : 2);
    if constexpr (KIND == kUmmaTF32) {
        uint32_t h[4], l[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) umma::split_tf32(x[j], h[j], l[j]);
        *reinterpret_cast<uint4 *>(hi) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4 *>(hi + plane) = make_uint4(l[0], l[1], l[2], l[3]);
    } else {
        uint16_t h[8], l[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) umma::split_bf16(x[j], h[j], l[j]);
        uint4 hv, lv;
        hv.x = h[0] | ((uint32_t)h[1] << 16);
        hv.y = h[2] | ((uint32_t)h[3] << 16);
        hv.z = h[4] | ((uint32_t)h[5] << 16);
        hv.w = h[6] | ((uint32_t)h[7] << 16);
        lv.x = l[0] | ((uint32_t)l[1] << 16);
        lv.y = l[2] | ((uint32_t)l[3] << 16);
        lv.z = l[4] | ((uint32_t)l[5] << 16);
        lv.w = l[6] | ((uint32_t)l[7] << 16);
        *reinterpret_cast<uint4 *>(hi) = hv;
        *reinterpret_cast<uint4 *>(hi + plane) = lv;
    }
}

template <int KIND, int NIN>
__global__ void __launch_bounds__(256) umma_planes(const StageIOT<float> io, unsigned char *planes, int R, int KP) {
    constexpr int per16 = KIND == kUmmaTF32 ? 4 : 8;
    const int64_t n = io.n_elements * (KP / per16);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        umma_planes_body<KIND, NIN>(io, planes, R, KP, i);
}

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

template <int KIND, typename Src>
__device__ __forceinline__ void umma_persistent(const UmmaShape &sh, const Src &tiles, int *status) {
    extern __shared__ __align__(1024) unsigned char umma_raw[];
    uint64_t *b_full = reinterpret_cast<uint64_t *>(umma_raw);  // [4] matrix image landed
    uint64_t *mma_done = b_full + 4;                             // [4] MMAs reading the buffer done
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(umma_raw + 128);
    int *fail_flag = reinterpret_cast<int *>(umma_raw + 192);
    int32_t *src_ids = reinterpret_cast<int32_t *>(umma_raw + 1024);  // [W][128] source element per slot, row
    unsigned char *ops = umma_raw + 1024 + umma_src_bytes(sh);
    const uint32_t buf_bytes = 2 * sh.a_bytes + 2 * sh.b_bytes;
    const int NB = umma_buffers(sh);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row_bytes = sh.KP * sh.es;         // one plane row
    const int cpr = row_bytes / 16;              // 16-byte chunks per plane row
    const int copies = 2 * kUmmaTileN * cpr;     // per item: both planes, all rows
    const int kstep_bytes = 32;                  // one MMA's K
    const int ksteps = row_bytes / kstep_bytes;
    const uint32_t idesc = umma_idesc(KIND, sh.NP);

    // this thread's copies are the same for every item: chunks tid, tid + 512, ...
    // (consecutive threads read consecutive chunks of one row); their destination in
    // the buffer, row, plane and byte offset in the row, computed once
    constexpr int MAXC = 16;  // 2 planes x 128 rows x 32 chunks (KP * es <= 512 bytes) / 512 threads
    uint32_t c_dst[MAXC], c_src[MAXC];
    int c_row[MAXC];
#pragma unroll
    for (int c = 0; c < MAXC; ++c) {
        const int i = tid + c * kUmmaThreads;
        const int part = i / (kUmmaTileN * cpr), rest = i - part * kUmmaTileN * cpr;
        const int row = rest / cpr, chunk = rest - row * cpr;
        c_row[c] = i < copies ? row : -1;
        c_src[c] = (uint32_t)(part << 31) | (uint32_t)(chunk * 16);  // plane bit, byte in row
        c_dst[c] = (uint32_t)(part * sh.a_bytes + (chunk >> 3) * (kUmmaTileN * 128) + row * 128 +
                              (((chunk & 7) ^ (row & 7)) << 4));
    }

    if (tid == 0) {
        for (int i = 0; i < 4; ++i) {
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

    uint32_t q = 0;  // (tile, slot) items of this CTA so far; item q uses buffer q % NB
    int64_t last_copy = -1, last_commit = -1;
    bool ok = true;
    // copies of item qq (slot s of the tile) into its buffer: both planes' source rows
    // (asynchronous 16-byte copies, zeros for a missing neighbour) and the slot's matrix
    // image (thread 0, bulk copy); one copy group per item
    auto issue = [&](const UmmaArgs &a, const int64_t tile, const int s, const uint32_t qq, const int64_t E) {
        unsigned char *A_hi = ops + (size_t)(qq % NB) * buf_bytes;
        unsigned char *B_hi = A_hi + 2 * sh.a_bytes;
        const int32_t *srow = src_ids + s * kUmmaTileN;
        const int32_t mat = a.tile_mats[tile * sh.W + s];
        const bool used = mat >= 0 && mat < a.n_mats;
        const int64_t plane_bytes = E * (int64_t)row_bytes;
#pragma unroll
        for (int c = 0; c < MAXC; ++c) {
            if (c_row[c] < 0) continue;
            const int32_t src = used ? srow[c_row[c]] : -1;
            const unsigned char *g = a.planes + ((c_src[c] >> 31) ? plane_bytes : 0) +
                                     (src >= 0 ? (int64_t)src * row_bytes : 0) + (c_src[c] & 0x7FFFFFFFu);
            umma::cp_async16(A_hi + c_dst[c], g, src >= 0 ? 16u : 0u);
        }
        umma::cp_async_commit();
        if (tid == 0) {
            uint64_t *bar = &b_full[qq % NB];
            if (mat >= a.n_mats) atomicOr(status, 4);
            umma::arrive_expect_tx(bar, used ? 2 * sh.b_bytes : 0);
            if (used) umma::bulk_load(B_hi, a.img + (size_t)mat * 2 * sh.b_bytes, 2 * sh.b_bytes, bar);
            last_copy = qq;
        }
    };

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
                    else if (n >= io.n_elements) atomicOr(status, 1);
                }
            }
            src_ids[i] = src;
        }
        __syncthreads();
        // Items are issued LAG_AHEAD = NB - LAG ahead of the MMAs; item s + NB - LAG refills
        // the buffer of item s - LAG, whose MMAs were issued LAG iterations ago (with four
        // buffers the refill never waits for the MMAs just issued).  The first items of
        // the tile go into buffers that are free after the last epilogue.
        const int LAG = NB >= 3 ? 2 : 1, LAG_AHEAD = NB - LAG;
        const int ahead = LAG_AHEAD < sh.W ? LAG_AHEAD : sh.W;
        for (int s0 = 0; s0 < ahead; ++s0) issue(a, tile, s0, q + s0, io.n_elements);
        for (int s = 0; s < sh.W && ok; ++s, ++q) {
            const int buf = q % NB;
            const int nxt = s + LAG_AHEAD;
            if (nxt < sh.W) {
                if (tid == 0 && s >= LAG &&
                    !umma::wait_bounded(&mma_done[(q - LAG) % NB], ((q - LAG) / NB) & 1, a.polls))
                    *fail_flag = 1;
                if (__syncthreads_or(*fail_flag)) {
                    ok = false;
                    break;
                }
                issue(a, tile, nxt, q + LAG_AHEAD, io.n_elements);
            }
            // copy groups issued after item q's: those of items q+1 .. min(q + LAG_AHEAD, last)
            const int later = (sh.W - 1 - s) < LAG_AHEAD ? (sh.W - 1 - s) : LAG_AHEAD;
            if (later >= 3) umma::cp_async_wait<3>();
            else if (later == 2) umma::cp_async_wait<2>();
            else if (later == 1) umma::cp_async_wait<1>();
            else umma::cp_async_wait<0>();
            umma::fence_proxy_async();  // async-proxy reads of what the copies wrote
            __syncthreads();
            if (tid == 0) {
                const int32_t mat = a.tile_mats[tile * sh.W + s];
                const bool used = mat >= 0 && mat < a.n_mats;
                unsigned char *A_hi = ops + (size_t)buf * buf_bytes;
                if (!umma::wait_bounded(&b_full[buf], (q / NB) & 1, a.polls)) {
                    *fail_flag = 1;
                } else {
                    umma::fence_after_sync();
                    const uint32_t a_hi = umma::smem_addr(A_hi), a_lo = a_hi + sh.a_bytes;
                    const uint32_t b_hi = a_lo + sh.a_bytes, b_lo = b_hi + sh.b_bytes;
                    if (used) {
                        for (int ks = 0; ks < ksteps; ++ks) {
                            const int panel = (ks * kstep_bytes) >> 7, within = (ks * kstep_bytes) & 127;
                            const uint32_t oa = panel * (kUmmaTileN * 128) + within;
                            const uint32_t ob = panel * (sh.NP * 128) + within;
                            const uint64_t dah = umma::desc_sw128(a_hi + oa), dal = umma::desc_sw128(a_lo + oa);
                            const uint64_t dbh = umma::desc_sw128(b_hi + ob), dbl = umma::desc_sw128(b_lo + ob);
                            const uint32_t first = (s == 0 && ks == 0) ? 0u : 1u;
                            umma::mma<KIND>(tmem, dah, dbh, idesc, first);
                            umma::mma<KIND>(tmem, dah, dbl, idesc, 1u);
                            umma::mma<KIND>(tmem, dal, dbh, idesc, 1u);
                        }
                    } else if (s == 0) {
                        // a tile whose self slot has no matrix: the gathered rows are zeros
                        const uint64_t dz = umma::desc_sw128(a_hi);
                        umma::mma<KIND>(tmem, dz, dz, idesc, 0u);
                    }
                }
                umma::commit(&mma_done[buf]);
                last_commit = q;
            }
        }
        if (!ok) break;
        // epilogue: the commits arrive in issue order, so the last item's marks them all
        const uint32_t last = q - 1;
        if (tid == 0 && !umma::wait_bounded(&mma_done[last % NB], (last / NB) & 1, a.polls)) *fail_flag = 1;
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
        umma::fence_proxy_async();  // the staging writes above precede the next tile's copies
        __syncthreads();
    }
    if (!ok) {
        // drain what this CTA still has in flight (bounded), then report
        umma::cp_async_wait<0>();
        if (tid == 0) {
            for (int64_t i = last_copy - NB + 1; i <= last_copy; ++i)
                if (i >= 0) umma::wait_bounded(&b_full[i % NB], (uint32_t)(i / NB) & 1, kUmmaPolls);
            if (last_commit >= 0)
                umma::wait_bounded(&mma_done[last_commit % NB], (uint32_t)(last_commit / NB) & 1, kUmmaPolls);
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

template <int KIND>
__global__ void __launch_bounds__(kUmmaThreads, 1)
    linear_umma_stage(const StageIOT<float> io, const UmmaArgs a, const UmmaShape sh) {
    umma_persistent<KIND>(sh, UmmaOneProblem{io, a}, io.status);
}

}  // namespace hgg
