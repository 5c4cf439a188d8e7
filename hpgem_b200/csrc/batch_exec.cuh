// Grouped execution of many independent problems (hgg_batch_*).
//
// Every problem keeps its own handle: its vectors and geometry stay resident
// where hgg_create put them.  A batch groups its problems by kernel class
// (kernel organisation, shape, order, physics, precision, tableau).  One RK
// stage of a class is ONE persistent launch: its CTAs walk the virtual blocks
// of all member problems (a prefix table of per-problem block counts, binary
// searched per virtual block) and run the same per-block code as the
// single-problem kernels, with that problem's stage inputs (its own dt and its
// own current buffer).  Per problem the device holds the buffer parity (which
// of its two solution buffers is current) and the steps still to take; a
// small kernel at the end of every step flips the parity and counts down, so a
// problem stops at exactly its own step count while the others go on.  The
// classes of one step are captured into one CUDA graph as parallel branches
// (fork/join on per-class streams) and the graph is replayed for every step;
// adding or removing a problem rewrites the tables and recaptures.
//
// Kernel tile shapes are chosen per class by a small autotuner: candidate
// launch shapes are timed on the class's own members with a stage-1 launch
// (which writes only the first stage vector, scratch between steps), and the
// fastest is cached per (class, size bucket) for the life of the process.
#pragma once

#include <cstddef>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

namespace hgg {

template <typename KT>
struct alignas(16) DenseItem {
    StageIOT<KT> io[2];  // [parity]: from sol[base] / from sol[1 - base]
    DenseGeom g;
    const int32_t *tiles;  // the wave on tiles of equal operators: the member's tiles (else null)
    int64_t block0;  // first virtual block
    int slot;
};
template <typename KT>
struct alignas(16) TensorItem {
    StageIOT<KT> io[2];
    TensorGeom geo;
    int64_t block0;
    int slot;
};
template <typename KT>
struct alignas(16) SliceItem {
    StageIOT<KT> io[2];
    const double *geo;
    int64_t block0;
    int slot;
};

// stored-matrix tiles on the tensor cores (tcgen05), the mixed forms
struct UmmaItem {
    StageIOT<float> io[2];
    UmmaArgs a;
    int64_t block0;  // first virtual tile
    int slot;
};

template <typename KT>
struct alignas(16) LinearItem {
    StageIOT<KT> io[2];
    LinearGeom g;
    LinearTiles t;
    int64_t block0;  // first virtual block (= tile)
    int slot;
};

// item whose virtual blocks contain vb: binary search of the items' first blocks,
// which the class table keeps as one compact array after the block total (total[1 + m]
// = item m's block0, ascending, total[1] = 0), so the probes stay in a few cache lines
// instead of touching one item record each
__device__ __forceinline__ int find_item(const int64_t *total, int n, int64_t vb) {
    const int64_t *block0 = total + 1;
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (block0[mid] <= vb) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The item of the virtual block in shared memory: the stage bodies read its fields
// (pointers, coefficients, sizes) many times, which from shared memory costs what the
// one-problem kernels pay for their parameters, not an L1 load each.  Ends with a
// barrier; the caller's loop begins with one, so the previous block is done with it.
template <typename Item>
__device__ __forceinline__ const Item &item_to_shared(const Item *items, int i, Item &s_item) {
    static_assert(sizeof(Item) % 16 == 0, "items are copied in 16-byte chunks");
    const int4 *src = reinterpret_cast<const int4 *>(items + i);
    int4 *dst = reinterpret_cast<int4 *>(&s_item);
    for (int k = threadIdx.x; k < (int)(sizeof(Item) / 16); k += blockDim.x) dst[k] = src[k];
    __syncthreads();
    return s_item;
}

template <typename KT, int DIM, int NFL, int WAVE, int NB>
__global__ void __launch_bounds__(256)
    grouped_dense(const DenseItem<KT> *items, const int *n_items, const int64_t *total, const int *parity,
                  const int *remaining) {
    const int n = *n_items;
    const int64_t nb = *total;
    for (int64_t vb = blockIdx.x; vb < nb; vb += gridDim.x) {
        const int i = find_item(total, n, vb);
        const int slot = items[i].slot;
        __syncthreads();  // shared memory of the previous virtual block is free
        if (remaining[slot] <= 0) continue;
        __shared__ DenseItem<KT> s_it;
        const DenseItem<KT> &it = item_to_shared(items, i, s_it);
        dense_any_body<KT, DIM, NFL, WAVE, NB>(it.io[parity[slot]], it.g, vb - it.block0);
    }
}

// the wave on tiles of elements with equal operators (one virtual block per tile)
template <typename KT, int DIM, int NFL, int NB>
__global__ void __launch_bounds__(group_threads(NB), 1024 / group_threads(NB) > 0 ? 1024 / group_threads(NB) : 1)
    grouped_wave_tiles(const DenseItem<KT> *items, const int *n_items, const int64_t *total, const int *parity,
                       const int *remaining) {
    const int n = *n_items;
    const int64_t nb = *total;
    for (int64_t vb = blockIdx.x; vb < nb; vb += gridDim.x) {
        const int i = find_item(total, n, vb);
        const int slot = items[i].slot;
        __syncthreads();
        if (remaining[slot] <= 0) continue;
        __shared__ DenseItem<KT> s_it;
        const DenseItem<KT> &it = item_to_shared(items, i, s_it);
        wave_group_body<KT, DIM, NFL, NB>(it.io[parity[slot]], it.g, it.tiles, vb - it.block0);
    }
}

template <typename KT, int P, int DIM, int EPB>
__global__ void __launch_bounds__(EPB *TensorConsts<P, DIM>::NB)
    grouped_tensor(const TensorItem<KT> *items, const int *n_items, const int64_t *total, const int *parity,
                   const int *remaining, const TensorConsts<P, DIM> tc) {
    const int n = *n_items;
    const int64_t nb = *total;
    for (int64_t vb = blockIdx.x; vb < nb; vb += gridDim.x) {
        const int i = find_item(total, n, vb);
        const int slot = items[i].slot;
        __syncthreads();
        if (remaining[slot] <= 0) continue;
        __shared__ TensorItem<KT> s_it;
        const TensorItem<KT> &it = item_to_shared(items, i, s_it);
        tensor_stage_body<KT, P, DIM, EPB>(it.io[parity[slot]], it.geo, tc, vb - it.block0);
    }
}

template <typename KT, int NIN, int NFIN>
__global__ void __launch_bounds__(SliceShape::THREADS, sizeof(KT) == 4 ? 5 : (NFIN == 0 ? 5 : 4))
    grouped_slice(const SliceItem<KT> *items, const int *n_items, const int64_t *total, const int *parity,
                  const int *remaining, const SliceOps op) {
    const int n = *n_items;
    const int64_t nb = *total;
    for (int64_t vb = blockIdx.x; vb < nb; vb += gridDim.x) {
        const int i = find_item(total, n, vb);
        const int slot = items[i].slot;
        __syncthreads();
        if (remaining[slot] <= 0) continue;
        __shared__ SliceItem<KT> s_it;
        const SliceItem<KT> &it = item_to_shared(items, i, s_it);
        tensor_slice_body<KT, NIN, NFIN>(it.io[parity[slot]], it.geo, op, vb - it.block0);
    }
}

template <typename KT>
__global__ void __launch_bounds__(256)
    grouped_linear(const LinearItem<KT> *items, const int *n_items, const int64_t *total, const int *parity,
                   const int *remaining) {
    const int n = *n_items;
    const int64_t nb = *total;
    for (int64_t vb = blockIdx.x; vb < nb; vb += gridDim.x) {
        const int i = find_item(total, n, vb);
        const int slot = items[i].slot;
        __syncthreads();
        if (remaining[slot] <= 0) continue;
        __shared__ LinearItem<KT> s_it;
        const LinearItem<KT> &it = item_to_shared(items, i, s_it);
        linear_tile_body<KT>(it.io[parity[slot]], it.g, it.t, vb - it.block0);
    }
}

// the tiles of all members of a class, for the persistent tensor-core kernel
struct UmmaGroupedTiles {
    const UmmaItem *items;
    int n;
    int64_t nb;
    const int64_t *totals;  // the block total, then the items' first blocks
    const int *parity, *remaining;
    __device__ int64_t total() const { return nb; }
    __device__ bool get(int64_t vt, StageIOT<float> &io, UmmaArgs &a, int64_t &tile) const {
        const int i = find_item(totals, n, vt);
        const int slot = items[i].slot;
        if (remaining[slot] <= 0) return false;
        io = items[i].io[parity[slot]];
        a = items[i].a;
        tile = vt - items[i].block0;
        return true;
    }
};

template <int KIND>
__global__ void __launch_bounds__(kUmmaThreads, 1)
    grouped_umma(const UmmaItem *items, const int *n_items, const int64_t *total, const int *parity,
                 const int *remaining, const UmmaShape sh, int *status) {
    umma_persistent<KIND>(sh, UmmaGroupedTiles{items, *n_items, *total, total, parity, remaining}, status);
}

// the split stage input of every member (blockIdx.y, then in steps of gridDim.y: member)
template <int KIND, int NIN>
__global__ void __launch_bounds__(256)
    grouped_umma_planes(const UmmaItem *items, const int *n_items, const int *parity, const int *remaining,
                        const UmmaShape sh) {
    constexpr int per16 = KIND == kUmmaTF32 ? 4 : 8;
    const int members = *n_items;
    for (int m = blockIdx.y; m < members; m += gridDim.y) {
        const UmmaItem &it = items[m];
        if (remaining[it.slot] <= 0) continue;
        const StageIOT<float> &io = it.io[parity[it.slot]];
        const int64_t n = io.n_elements * (sh.KP / per16);
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            umma_planes_body<KIND, NIN>(io, const_cast<unsigned char *>(it.a.planes), sh.R, sh.KP, i);
    }
}

// end of one step of every member: flip the current buffer, count the step
__global__ void batch_advance(int *parity, int *remaining, int cap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < cap && remaining[i] > 0) {
        parity[i] ^= 1;
        remaining[i] -= 1;
    }
}

// a member's counters when it joins (kernel arguments are copied at launch, so the
// host issues the change without waiting for the stream)
__global__ void batch_set_slot(int *parity, int *remaining, int slot, int nsteps) {
    parity[slot] = 0;
    remaining[slot] = nsteps;
}

}  // namespace hgg

namespace {

enum BatchKind { KIND_DENSE = 0, KIND_TENSOR = 1, KIND_SLICE = 2, KIND_LINEAR = 3, KIND_UMMA = 4, KIND_WAVE_TILES = 5 };

struct BatchClass {
    // key
    int kind = 0, shape = 0, order = 0, dim = 0, physics = 0, S = 0;
    bool mixed = false;
    int precision = 0, rows = 0, lslots = 0;  // tensor-core tiles: precision, rows and slots per element
    // the reference-element data the launches take (basis size, 1D operators), from the
    // first member: the class launches the same way when it has no members
    HostOperators rep;
    unsigned grid_floor = 0;  // grid of the last capture: a class's grid never shrinks
    std::vector<double> rk_a, rk_b;
    // members and launch shape
    std::vector<int> slots;
    int epb = 1;          // dense: elements per block
    int ctas_per_sm = 2;  // persistent CTAs per SM
    bool tuned = false;
    int tuned_bucket = -1;
    bool table_dirty = true;  // members changed since the tables were uploaded
    // device tables: items [S][cap] (one array per stage), count and block total
    std::vector<void *> d_items;
    size_t item_bytes = 0;
    int *d_n = nullptr;
    int64_t *d_total = nullptr;
    int64_t total_blocks = 0;
    int64_t total_elements = 0;
    // pinned staging of the table uploads, two buffers used in turn: an upload only waits
    // for the copy issued from the same buffer two uploads earlier, never for the stream
    unsigned char *h_up[2] = {nullptr, nullptr};
    cudaEvent_t up_done[2] = {nullptr, nullptr};
    int up_next = 0;
    size_t up_bytes = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
};

struct TuneKey {
    int kind, shape, order, physics, mixed, bucket;
    bool operator<(const TuneKey &o) const {
        return std::tie(kind, shape, order, physics, mixed, bucket) <
               std::tie(o.kind, o.shape, o.order, o.physics, o.mixed, o.bucket);
    }
};
struct TuneChoice {
    int epb, ctas_per_sm;
    float ms;
};
std::mutex g_tune_mutex;
std::map<TuneKey, TuneChoice> g_tune_cache;

thread_local std::string g_batch_create_error = "no error";

}  // namespace

struct hgg_batch {
    int device = 0;
    int cap = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<hgg_handle *> handles;  // by slot, nullptr when free
    std::vector<double> dt;
    std::vector<int> base;               // the handle's current buffer when it was added
    std::vector<int> cls;                // class index of each slot
    std::vector<int> remaining_host;     // as last read back
    std::vector<std::vector<unsigned char>> item_cache;  // per slot: its items of every stage
    std::vector<int> cache_epb;          // elements per block the cached items were formed with
    std::vector<int64_t> slot_blocks;    // virtual blocks of each slot's member
    std::vector<int> parity_host;
    int *d_parity = nullptr, *d_remaining = nullptr, *d_status = nullptr;
    std::vector<BatchClass> classes;
    cudaGraphExec_t graph = nullptr;
    std::vector<int> graph_sig;  // (class, epb, ctas per SM, grid) of the captured step
    bool dirty = true;
    bool autotune = true;
    // launch_class_stage in query mode: the class's kernel is not launched, its resident
    // CTAs per SM are recorded instead (the default persistent grid)
    bool occ_query = false;
    mutable int occ_result = 0;
    int64_t launches = 0;
    std::string err = "no error";
};

namespace {

int bfail(hgg_batch *b, int code, const std::string &msg) {
    if (b) b->err = msg;
    else g_batch_create_error = msg;
    return code;
}

#define HGG_BCUDA(b, call)                                                                    \
    do {                                                                                      \
        cudaError_t _e = (call);                                                              \
        if (_e != cudaSuccess)                                                                \
            return bfail(b, HGG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
    } while (0)

int batch_kind(const hgg_handle *h) {
    if (h->umma_tiles > 0) return KIND_UMMA;
    if (h->linear) return KIND_LINEAR;
    if (h->slice_ok) return KIND_SLICE;
    if (h->op.tensor) return KIND_TENSOR;
    // the same choice as the handle's own dense launch: tiles where the contraction is FP64
    if (group_wave_wanted(h)) return KIND_WAVE_TILES;
    // Above 24 basis functions a batch takes the 16-element tiles on any member that
    // forms them: a class adds its members up, and on the served request mix the class
    // of tetrahedra at p = 4 measured 1.42 ms per step on the tiles against 1.82 ms on
    // the per-row kernel (a single handle takes them from 2^16 elements).  Both kernels
    // do the same arithmetic in the same order, so the result equals the handle's alone.
    if (h->group_tiles > 0 && h->op.nB > kGroupMaxRows && h->variant == 0 && !h->linear && !h->op.tensor)
        return KIND_WAVE_TILES;
    return KIND_DENSE;
}

bool same_class(const BatchClass &c, const hgg_handle *h) {
    return c.kind == batch_kind(h) && c.shape == h->op.shape && c.order == h->op.order && c.dim == h->op.dim &&
           c.physics == h->op.physics && c.mixed == h->mixed && c.S == h->S && c.rk_a == h->rk_a &&
           c.rk_b == h->rk_b &&
           (c.kind != KIND_UMMA || (c.precision == h->precision && c.rows == h->lin_R && c.lslots == h->lin_slots));
}

int dense_R(const hgg_handle *h) { return h->op.V * h->op.nB; }

int tensor_epb(int order, int dim) {
    const int np = order + 1, nb = dim == 2 ? np * np : np * np * np;
    return std::max(1, 256 / nb);
}

int64_t item_blocks(const BatchClass &c, const hgg_handle *h) {
    const int64_t nE = h->op.nE;
    if (c.kind == KIND_LINEAR) return h->lin_tiles;
    if (c.kind == KIND_UMMA) return h->umma_tiles;
    if (c.kind == KIND_WAVE_TILES) return h->group_tiles;
    if (c.kind == KIND_SLICE) return (nE + SliceShape::TE - 1) / SliceShape::TE;
    if (c.kind == KIND_TENSOR) {
        const int epb = tensor_epb(c.order, c.dim);
        return (nE + epb - 1) / epb;
    }
    return (nE + c.epb - 1) / c.epb;
}

size_t class_item_bytes(const BatchClass &c) {
    if (c.kind == KIND_DENSE || c.kind == KIND_WAVE_TILES)
        return c.mixed ? sizeof(DenseItem<float>) : sizeof(DenseItem<double>);
    if (c.kind == KIND_TENSOR) return c.mixed ? sizeof(TensorItem<float>) : sizeof(TensorItem<double>);
    if (c.kind == KIND_LINEAR) return c.mixed ? sizeof(LinearItem<float>) : sizeof(LinearItem<double>);
    if (c.kind == KIND_UMMA) return sizeof(UmmaItem);
    return c.mixed ? sizeof(SliceItem<float>) : sizeof(SliceItem<double>);
}

DenseGeom dense_geom(const hgg_handle *h, int epb) {
    const HostOperators &op = h->op;
    return DenseGeom{h->d_vol, h->d_pairs, h->d_vol_f, h->d_pairs_f, h->d_nbr, h->d_self, h->d_nbrp, h->d_mode,
                     h->d_elem_geo, h->d_face_geo, 1.0 / op.c_inv, upwind_speed(op), op.nB, epb};
}

// the item of one member for one stage (block0: its first virtual block in the class)
template <typename KT>
void fill_member(const hgg_batch *b, const BatchClass &c, int slot, int stage, int64_t block0, unsigned char *dst) {
    const hgg_handle *h = b->handles[slot];
    const int base = b->base[slot];
    if (c.kind == KIND_DENSE || c.kind == KIND_WAVE_TILES) {
        DenseItem<KT> it{};
        for (int par = 0; par < 2; ++par)
            it.io[par] = make_stage_io<KT>(h, par ? 1 - base : base, b->dt[slot], stage, b->d_status);
        it.g = dense_geom(h, c.epb);
        it.tiles = c.kind == KIND_WAVE_TILES ? h->d_group_tiles : nullptr;
        it.block0 = block0;
        it.slot = slot;
        std::memcpy(dst, &it, sizeof(it));
    } else if (c.kind == KIND_UMMA) {
        UmmaItem it{};
        for (int par = 0; par < 2; ++par)
            it.io[par] = make_stage_io<float>(h, par ? 1 - base : base, b->dt[slot], stage, b->d_status);
        it.a = UmmaArgs{h->d_umma_img, h->d_umma_planes, h->d_umma_tile_elems, h->d_umma_tile_mats, h->d_lin_nbr,
                        h->umma_tiles, h->lin_mats, kUmmaPolls};
        it.block0 = block0;
        it.slot = slot;
        std::memcpy(dst, &it, sizeof(it));
    } else if (c.kind == KIND_LINEAR) {
        LinearItem<KT> it{};
        for (int par = 0; par < 2; ++par)
            it.io[par] = make_stage_io<KT>(h, par ? 1 - base : base, b->dt[slot], stage, b->d_status);
        it.g = LinearGeom{h->d_lin_table, h->d_lin_table_rm, h->d_lin_table_f, h->d_lin_self, h->d_lin_nbr,
                          h->d_lin_mat, h->lin_R, h->lin_slots, std::max(1, 256 / h->lin_R), h->lin_mats};
        it.t = LinearTiles{h->d_lin_tile_elems, h->d_lin_tile_mats};
        it.block0 = block0;
        it.slot = slot;
        std::memcpy(dst, &it, sizeof(it));
    } else if (c.kind == KIND_TENSOR) {
        TensorItem<KT> it{};
        for (int par = 0; par < 2; ++par)
            it.io[par] = make_stage_io<KT>(h, par ? 1 - base : base, b->dt[slot], stage, b->d_status);
        it.geo = TensorGeom{h->d_ahat, h->d_tnbr, h->d_tmode, h->d_tsigma};
        it.block0 = block0;
        it.slot = slot;
        std::memcpy(dst, &it, sizeof(it));
    } else {
        SliceItem<KT> it{};
        for (int par = 0; par < 2; ++par)
            it.io[par] = make_stage_io<KT>(h, par ? 1 - base : base, b->dt[slot], stage, b->d_status);
        it.geo = h->d_slice_geo;
        it.block0 = block0;
        it.slot = slot;
        std::memcpy(dst, &it, sizeof(it));
    }
}

// sets the first virtual block of a stored item (every item type ends with block0, slot)
template <typename KT>
void set_block0(const BatchClass &c, unsigned char *dst, int64_t block0) {
    auto put = [&](auto *it) {
        using T = std::remove_pointer_t<decltype(it)>;
        std::memcpy(dst + offsetof(T, block0), &block0, sizeof(block0));
    };
    if (c.kind == KIND_DENSE || c.kind == KIND_WAVE_TILES) put((DenseItem<KT> *)nullptr);
    else if (c.kind == KIND_UMMA) put((UmmaItem *)nullptr);
    else if (c.kind == KIND_LINEAR) put((LinearItem<KT> *)nullptr);
    else if (c.kind == KIND_TENSOR) put((TensorItem<KT> *)nullptr);
    else put((SliceItem<KT> *)nullptr);
}

// host copy of the items of one stage of a class: each member's items are formed once
// when it joins (or when the class's elements per block change) and kept per slot, so
// a table rewrite after a join or a removal copies them and sets their first blocks
template <typename KT>
void fill_items(hgg_batch *b, const BatchClass &c, int stage, std::vector<unsigned char> &buf) {
    buf.resize(c.item_bytes * c.slots.size());
    int64_t block0 = 0;
    for (size_t m = 0; m < c.slots.size(); ++m) {
        const int slot = c.slots[m];
        auto &cache = b->item_cache[slot];
        if (cache.size() != c.item_bytes * c.S || b->cache_epb[slot] != c.epb) {
            cache.assign(c.item_bytes * c.S, 0);
            for (int st = 0; st < c.S; ++st) fill_member<KT>(b, c, slot, st, 0, cache.data() + st * c.item_bytes);
            b->cache_epb[slot] = c.epb;
            b->slot_blocks[slot] = item_blocks(c, b->handles[slot]);
        }
        unsigned char *dst = buf.data() + m * c.item_bytes;
        std::memcpy(dst, cache.data() + stage * c.item_bytes, c.item_bytes);
        set_block0<KT>(c, dst, block0);
        block0 += b->slot_blocks[slot];
    }
}

int upload_class(hgg_batch *b, BatchClass &c) {
    c.total_blocks = 0;
    c.total_elements = 0;
    for (int slot : c.slots) {
        c.total_blocks += item_blocks(c, b->handles[slot]);
        c.total_elements += b->handles[slot]->op.nE;
    }
    // layout of a staging buffer: the S item arrays, then the block total followed by
    // every item's first block, then n
    const size_t items = c.item_bytes * (size_t)b->cap;
    const size_t need = items * c.S + 8 * (size_t)(b->cap + 1) + 16;
    const int u = c.up_next;
    c.up_next ^= 1;
    if (!c.h_up[u] || c.up_bytes < need) {
        HGG_BCUDA(b, cudaStreamSynchronize(b->stream));  // both staging buffers idle before a resize
        for (int i = 0; i < 2; ++i) {
            if (c.h_up[i]) cudaFreeHost(c.h_up[i]);
            c.h_up[i] = nullptr;
            HGG_BCUDA(b, cudaHostAlloc((void **)&c.h_up[i], need, cudaHostAllocDefault));
        }
        c.up_bytes = need;
    } else if (c.up_done[u]) {
        HGG_BCUDA(b, cudaEventSynchronize(c.up_done[u]));  // the copy from this buffer two uploads ago
    }
    if (!c.up_done[u]) HGG_BCUDA(b, cudaEventCreateWithFlags(&c.up_done[u], cudaEventDisableTiming));
    unsigned char *stage = c.h_up[u];
    std::vector<unsigned char> buf;
    for (int st = 0; st < c.S; ++st) {
        if (c.mixed) fill_items<float>(b, c, st, buf);
        else fill_items<double>(b, c, st, buf);
        if (!buf.empty()) {
            std::memcpy(stage + items * st, buf.data(), buf.size());
            HGG_BCUDA(b, cudaMemcpyAsync(c.d_items[st], stage + items * st, buf.size(), cudaMemcpyHostToDevice,
                                         b->stream));
        }
    }
    unsigned char *tail = stage + items * c.S;
    const int n = (int)c.slots.size();
    int64_t *totals = reinterpret_cast<int64_t *>(tail);
    totals[0] = c.total_blocks;
    int64_t first = 0;
    for (int m = 0; m < n; ++m) {
        totals[1 + m] = first;
        first += b->slot_blocks[c.slots[m]];
    }
    unsigned char *ntail = tail + 8 * (size_t)(b->cap + 1);
    std::memcpy(ntail, &n, sizeof(int));
    HGG_BCUDA(b, cudaMemcpyAsync(c.d_total, tail, sizeof(int64_t) * (1 + n), cudaMemcpyHostToDevice, b->stream));
    HGG_BCUDA(b, cudaMemcpyAsync(c.d_n, ntail, sizeof(int), cudaMemcpyHostToDevice, b->stream));
    HGG_BCUDA(b, cudaEventRecord(c.up_done[u], b->stream));
    return 0;
}

// launches a class kernel, or in query mode records how many of its CTAs fit on an SM
template <typename Kern, typename... A>
void class_kernel(const hgg_batch *b, Kern kern, unsigned grid, unsigned threads, size_t smem, cudaStream_t s,
                  A... args) {
    if (b->occ_query) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, (int)threads, smem) == cudaSuccess)
            b->occ_result = n;
        return;
    }
    kern<<<grid, threads, smem, s>>>(args...);
}

template <typename KT, int DIM, int NFL, int WAVE>
void launch_grouped_dense(const hgg_batch *b, const BatchClass &c, int st, unsigned grid, cudaStream_t s) {
    const int nB = c.rep.nB;
    const int threads = dense_threads(DIM, WAVE, nB, c.epb);
    dense_dispatch<DIM, NFL, WAVE>(nB, [&](auto nbc) {
        constexpr int NB = decltype(nbc)::value;
        const size_t smem = dense_smem(DIM, NFL, WAVE, NB, c.epb, sizeof(DenseCT<KT, NB>));
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(grouped_dense<KT, DIM, NFL, WAVE, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        class_kernel(b, grouped_dense<KT, DIM, NFL, WAVE, NB>, grid, threads, smem, s,
                     static_cast<const DenseItem<KT> *>(c.d_items[st]), c.d_n, c.d_total, b->d_parity,
                     b->d_remaining);
    });
}

template <int DIM, int NFL, int WAVE>
void launch_grouped_dense_any(const hgg_batch *b, const BatchClass &c, int st, unsigned grid, cudaStream_t s) {
    if (c.mixed) launch_grouped_dense<float, DIM, NFL, WAVE>(b, c, st, grid, s);
    else launch_grouped_dense<double, DIM, NFL, WAVE>(b, c, st, grid, s);
}

template <typename KT, int DIM, int NFL>
void launch_grouped_wave(const hgg_batch *b, const BatchClass &c, int st, unsigned grid, cudaStream_t s) {
    const int nB = c.rep.nB;
    dense_dispatch<DIM, NFL, 1>(nB, [&](auto nbc) {
        constexpr int NB = decltype(nbc)::value;
        if constexpr (DIM >= 2 && NB <= kGroupMaxBasis) {
            constexpr size_t smem = group_smem<DenseCT<KT, NB>, DIM, NFL, NB>();
            cudaFuncSetAttribute(grouped_wave_tiles<KT, DIM, NFL, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
            class_kernel(b, grouped_wave_tiles<KT, DIM, NFL, NB>, grid, group_threads(NB), smem, s,
                         static_cast<const DenseItem<KT> *>(c.d_items[st]), c.d_n, c.d_total, b->d_parity,
                         b->d_remaining);
        }
    });
}

template <int P, int DIM>
void launch_grouped_tensor(const hgg_batch *b, const BatchClass &c, int st, unsigned grid, cudaStream_t s) {
    constexpr int NB = TensorConsts<P, DIM>::NB;
    constexpr int EPB = (256 / NB) > 0 ? (256 / NB) : 1;
    const TensorConsts<P, DIM> tc = tensor_consts<P, DIM>(c.rep);
    if (c.mixed)
        class_kernel(b, grouped_tensor<float, P, DIM, EPB>, grid, EPB * NB, 0, s,
                     static_cast<const TensorItem<float> *>(c.d_items[st]), c.d_n, c.d_total, b->d_parity,
                     b->d_remaining, tc);
    else
        class_kernel(b, grouped_tensor<double, P, DIM, EPB>, grid, EPB * NB, 0, s,
                     static_cast<const TensorItem<double> *>(c.d_items[st]), c.d_n, c.d_total, b->d_parity,
                     b->d_remaining, tc);
}

template <typename KT>
void launch_grouped_slice(const hgg_batch *b, const BatchClass &c, int st, unsigned grid, cudaStream_t s) {
    SliceOps sops;
    for (int i = 0; i < 16; ++i) sops.D[i] = c.rep.D1[i];
    for (int sd = 0; sd < 2; ++sd)
        for (int a = 0; a < 4; ++a) sops.L[sd][a] = c.rep.lift[sd * 4 + a];
    // the stage's shape is the same for every member (same tableau): its stage-input
    // vectors (nonzero a_ij) and, in the final stage, the earlier vectors of the update
    struct {
        int nin = 0, nfin = 0;
    } io;
    for (int j = 0; j < st; ++j) io.nin += c.rk_a[st * c.S + j] != 0.0;
    const bool fin = st == c.S - 1;
    if (fin)
        for (int j = 0; j < c.S - 1; ++j) io.nfin += c.rk_b[j] != 0.0;
    const auto *items = static_cast<const SliceItem<KT> *>(c.d_items[st]);
    const dim3 g(grid), blk(SliceShape::THREADS);
    if (io.nin == 0 && (!fin || io.nfin == 0))
        class_kernel(b, grouped_slice<KT, 0, 0>, grid, SliceShape::THREADS, 0, s, items, c.d_n, c.d_total,
                     b->d_parity, b->d_remaining, sops);
    else if (io.nin == 1 && (!fin || io.nfin == 0))
        class_kernel(b, grouped_slice<KT, 1, 0>, grid, SliceShape::THREADS, 0, s, items, c.d_n, c.d_total,
                     b->d_parity, b->d_remaining, sops);
    else if (io.nin == 1 && fin && io.nfin == 3)
        class_kernel(b, grouped_slice<KT, 1, 3>, grid, SliceShape::THREADS, 0, s, items, c.d_n, c.d_total,
                     b->d_parity, b->d_remaining, sops);
    else
        class_kernel(b, grouped_slice<KT, -1, -1>, grid, SliceShape::THREADS, 0, s, items, c.d_n, c.d_total,
                     b->d_parity, b->d_remaining, sops);
}

// one stage of one class
// Persistent grid of a class: ctas_per_sm CTAs per SM, or fewer for a class with
// fewer virtual blocks (its block count rounded up to a power of two, and never less
// than the grid it was last captured with), so that the kernels of small classes leave
// SMs to the other classes of the step, which run as parallel branches of the captured
// graph.  A captured grid stays valid while the class's membership changes (the CTAs
// loop over the virtual blocks); the step is captured again only when a class outgrows
// its grid or a class that is not in the graph gains members.
unsigned class_grid(const hgg_batch *b, const BatchClass &c) {
    const int64_t full = (int64_t)c.ctas_per_sm * b->num_sms;
    if (c.total_blocks >= full) return (unsigned)full;
    int64_t g = 1;
    while (g < c.total_blocks) g <<= 1;
    return (unsigned)std::min(std::max(g, (int64_t)c.grid_floor), full);
}

void launch_class_stage(hgg_batch *b, const BatchClass &c, int st, cudaStream_t s) {
    const unsigned grid = class_grid(b, c);
    if (c.kind == KIND_UMMA) {
        const int kind = c.precision == HGG_PRECISION_BF16X3 ? kUmmaBF16 : kUmmaTF32;
        const UmmaShape sh = umma_shape(c.rows, c.lslots, kind);
        int nin = 0;  // stage-input vectors of this stage (the tableau's nonzero a_ij)
        for (int j = 0; j < st; ++j) nin += c.rk_a[st * c.S + j] != 0.0;
        if (!(c.rows % 4 == 0 && nin <= 1)) nin = -1;
        const size_t smem = umma_smem(sh);
        const UmmaItem *it = static_cast<const UmmaItem *>(c.d_items[st]);
        // members along y (a power of two at least their count, looping past it)
        unsigned my = 1;
        while (my < c.slots.size() && my < 1024) my <<= 1;
        const dim3 pgrid((unsigned)(2 * b->num_sms), my);
        auto planes = [&](auto kc, auto nc) {
            constexpr int K = decltype(kc)::value, NIN = decltype(nc)::value;
            if (!b->occ_query)  // the planes kernel's grid is not the class's persistent grid
                grouped_umma_planes<K, NIN><<<pgrid, 256, 0, s>>>(it, c.d_n, b->d_parity, b->d_remaining, sh);
        };
        auto tiles = [&](auto kc) {
            constexpr int K = decltype(kc)::value;
            cudaFuncSetAttribute(grouped_umma<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            class_kernel(b, grouped_umma<K>, grid, kUmmaThreads, smem, s, it, c.d_n, c.d_total, b->d_parity,
                         b->d_remaining, sh, b->d_status);
        };
        using I0 = std::integral_constant<int, 0>;
        using I1 = std::integral_constant<int, 1>;
        using IM = std::integral_constant<int, -1>;
        using KT32 = std::integral_constant<int, kUmmaTF32>;
        using KB16 = std::integral_constant<int, kUmmaBF16>;
        if (kind == kUmmaTF32) {
            if (nin == 0) planes(KT32{}, I0{});
            else if (nin == 1) planes(KT32{}, I1{});
            else planes(KT32{}, IM{});
            tiles(KT32{});
        } else {
            if (nin == 0) planes(KB16{}, I0{});
            else if (nin == 1) planes(KB16{}, I1{});
            else planes(KB16{}, IM{});
            tiles(KB16{});
        }
        if (!b->occ_query) b->launches++;  // the planes launch
    } else if (c.kind == KIND_LINEAR) {
        if (c.mixed)
            class_kernel(b, grouped_linear<float>, grid, 256, 0, s, static_cast<const LinearItem<float> *>(c.d_items[st]),
                         c.d_n, c.d_total, b->d_parity, b->d_remaining);
        else
            class_kernel(b, grouped_linear<double>, grid, 256, 0, s,
                         static_cast<const LinearItem<double> *>(c.d_items[st]), c.d_n, c.d_total, b->d_parity,
                         b->d_remaining);
    } else if (c.kind == KIND_SLICE) {
        if (c.mixed) launch_grouped_slice<float>(b, c, st, grid, s);
        else launch_grouped_slice<double>(b, c, st, grid, s);
    } else if (c.kind == KIND_WAVE_TILES) {
        switch (c.shape) {
            case HGG_SHAPE_TRIANGLE:
                c.mixed ? launch_grouped_wave<float, 2, 3>(b, c, st, grid, s) : launch_grouped_wave<double, 2, 3>(b, c, st, grid, s);
                break;
            case HGG_SHAPE_SQUARE:
                c.mixed ? launch_grouped_wave<float, 2, 4>(b, c, st, grid, s) : launch_grouped_wave<double, 2, 4>(b, c, st, grid, s);
                break;
            case HGG_SHAPE_TETRAHEDRON:
                c.mixed ? launch_grouped_wave<float, 3, 4>(b, c, st, grid, s) : launch_grouped_wave<double, 3, 4>(b, c, st, grid, s);
                break;
            case HGG_SHAPE_CUBE:
                c.mixed ? launch_grouped_wave<float, 3, 6>(b, c, st, grid, s) : launch_grouped_wave<double, 3, 6>(b, c, st, grid, s);
                break;
        }
    } else if (c.kind == KIND_TENSOR) {
#define HGG_GT(P)                                                  \
    case P:                                                        \
        if (c.dim == 2) launch_grouped_tensor<P, 2>(b, c, st, grid, s); \
        else launch_grouped_tensor<P, 3>(b, c, st, grid, s);            \
        break;
        switch (c.order) { HGG_GT(1) HGG_GT(2) HGG_GT(3) HGG_GT(4) HGG_GT(5) }
#undef HGG_GT
    } else {
        const bool wave = c.physics != HGG_PHYSICS_ADVECTION;
        switch (c.shape) {
            case HGG_SHAPE_LINE: wave ? launch_grouped_dense_any<1, 2, 1>(b, c, st, grid, s) : launch_grouped_dense_any<1, 2, 0>(b, c, st, grid, s); break;
            case HGG_SHAPE_TRIANGLE: wave ? launch_grouped_dense_any<2, 3, 1>(b, c, st, grid, s) : launch_grouped_dense_any<2, 3, 0>(b, c, st, grid, s); break;
            case HGG_SHAPE_SQUARE: wave ? launch_grouped_dense_any<2, 4, 1>(b, c, st, grid, s) : launch_grouped_dense_any<2, 4, 0>(b, c, st, grid, s); break;
            case HGG_SHAPE_TETRAHEDRON: wave ? launch_grouped_dense_any<3, 4, 1>(b, c, st, grid, s) : launch_grouped_dense_any<3, 4, 0>(b, c, st, grid, s); break;
            case HGG_SHAPE_CUBE: wave ? launch_grouped_dense_any<3, 6, 1>(b, c, st, grid, s) : launch_grouped_dense_any<3, 6, 0>(b, c, st, grid, s); break;
        }
    }
    if (!b->occ_query) b->launches++;
}

int size_bucket(int64_t elements) {
    int k = 0;
    while (elements > 1 && k < 40) {
        elements >>= 1;
        ++k;
    }
    return k;
}

// Time the candidate launch shapes of a class on its members (stage 1, which
// writes only the first stage vector) and keep the fastest.
int tune_class(hgg_batch *b, BatchClass &c) {
    const TuneKey key{c.kind, c.shape, c.order, c.physics, (int)c.mixed, size_bucket(c.total_elements)};
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            const bool same_epb = c.epb == it->second.epb;
            c.epb = it->second.epb;
            c.ctas_per_sm = it->second.ctas_per_sm;
            c.tuned = true;
            c.tuned_bucket = key.bucket;
            if (!same_epb) return upload_class(b, c);  // dense block counts depend on epb
            return 0;
        }
    }
    if (c.kind == KIND_UMMA) {
        // one resident CTA per SM (its shared memory and tensor memory), or as many as fit
        const int kind = c.precision == HGG_PRECISION_BF16X3 ? kUmmaBF16 : kUmmaTF32;
        const size_t smem = umma_smem(umma_shape(c.rows, c.lslots, kind));
        c.ctas_per_sm = std::max(1, std::min(4, (int)((227 * 1024) / (smem + 1024))));
        c.tuned = true;
        c.tuned_bucket = key.bucket;
        return 0;
    }
    std::vector<std::pair<int, int>> cands;  // (epb, ctas_per_sm)
    const int ctas[] = {2, 4, 8};
    if (c.kind == KIND_DENSE) {
        // elements per block: the largest that fills 256 threads, and half of it
        const hgg_handle *h0 = b->handles[c.slots[0]];
        const int wave = c.physics != HGG_PHYSICS_ADVECTION;
        const int rows = dense_rows(c.dim, wave, h0->op.nB);
        const int nfl = c.shape == HGG_SHAPE_LINE ? 2 : (c.shape == HGG_SHAPE_TRIANGLE ? 3
                        : (c.shape == HGG_SHAPE_SQUARE || c.shape == HGG_SHAPE_TETRAHEDRON ? 4 : 6));
        const int full = std::max(1, 256 / rows);
        for (int epb : {full, std::max(1, full / 2)}) {
            if (dense_smem(c.dim, nfl, wave, h0->op.nB, epb, 8) > 200 * 1024) continue;
            for (int cs : ctas) cands.push_back({epb, cs});
            if (full == 1) break;
        }
    } else {
        for (int cs : ctas) cands.push_back({c.epb, cs});
    }
    if (cands.empty()) return bfail(b, HGG_ERR_UNSUPPORTED, "batch: no launch shape fits this class");
    // the remaining counters must read positive for every member while timing
    cudaEvent_t e0, e1;
    HGG_BCUDA(b, cudaEventCreate(&e0));
    HGG_BCUDA(b, cudaEventCreate(&e1));
    TuneChoice best{c.epb, c.ctas_per_sm, 1e30f};
    for (auto [epb, cs] : cands) {
        if (epb != c.epb) {
            c.epb = epb;
            int rc = upload_class(b, c);
            if (rc) return rc;
        }
        c.ctas_per_sm = cs;
        float tmin = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {
            cudaEventRecord(e0, b->stream);
            launch_class_stage(b, c, 0, b->stream);
            cudaEventRecord(e1, b->stream);
            HGG_BCUDA(b, cudaEventSynchronize(e1));
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            tmin = std::min(tmin, ms);
        }
        HGG_BCUDA(b, cudaGetLastError());
        if (tmin < best.ms) best = TuneChoice{epb, cs, tmin};
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (c.epb != best.epb) {
        c.epb = best.epb;
        int rc = upload_class(b, c);
        if (rc) return rc;
    }
    c.ctas_per_sm = best.ctas_per_sm;
    c.tuned = true;
    c.tuned_bucket = key.bucket;
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = best;
    return 0;
}

// read parity and remaining counters back (after the stream is idle)
int read_counters(hgg_batch *b) {
    HGG_BCUDA(b, cudaMemcpyAsync(b->parity_host.data(), b->d_parity, sizeof(int) * b->cap, cudaMemcpyDeviceToHost,
                                 b->stream));
    HGG_BCUDA(b, cudaMemcpyAsync(b->remaining_host.data(), b->d_remaining, sizeof(int) * b->cap,
                                 cudaMemcpyDeviceToHost, b->stream));
    HGG_BCUDA(b, cudaStreamSynchronize(b->stream));
    return 0;
}

void release_batch_graph(hgg_batch *b) {
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
}

// tables of the classes whose members changed (an emptied class gets n = 0, so a graph
// that still launches it finds no work), autotuning of classes with enough work and no
// tuned shape for their size, and a new capture of one step only when a class with
// members is missing from the captured step or its launch shape changed
int prepare_batch(hgg_batch *b) {
    if (!b->dirty && b->graph) return 0;
    bool counters_read = false;
    for (auto &c : b->classes) {
        if (c.table_dirty) {
            int rc = upload_class(b, c);
            if (rc) return rc;
            c.table_dirty = false;
        }
        if (c.slots.empty()) continue;
        // tuning launches stage 1 of the members (every member must have steps left for it
        // to run); a one-stage tableau's first stage is its final update, so it is not tuned;
        // classes with less than two blocks per SM keep the default shape
        const int bucket = size_bucket(c.total_elements);
        if (b->autotune && c.S > 1 && c.total_blocks >= 2 * b->num_sms && (!c.tuned || c.tuned_bucket != bucket)) {
            if (!counters_read) {
                int rc = read_counters(b);  // the values the tuning below overwrites for a moment
                if (rc) return rc;
                counters_read = true;
            }
            std::vector<int> ones(b->cap, 1);
            HGG_BCUDA(b, cudaMemcpyAsync(b->d_remaining, ones.data(), sizeof(int) * b->cap, cudaMemcpyHostToDevice,
                                         b->stream));
            int rc = tune_class(b, c);
            if (rc) return rc;
            HGG_BCUDA(b, cudaMemcpyAsync(b->d_remaining, b->remaining_host.data(), sizeof(int) * b->cap,
                                         cudaMemcpyHostToDevice, b->stream));
            HGG_BCUDA(b, cudaStreamSynchronize(b->stream));
        }
    }
    // classes of the step: those with members and those already in the graph (a class
    // that empties stays in the captured step with n = 0, so that it can refill without
    // a new capture)
    auto in_graph = [&](int i) {
        for (size_t j = 0; j + 3 < b->graph_sig.size(); j += 4)
            if (b->graph_sig[j] == i) return true;
        return false;
    };
    std::vector<int> sig;
    bool covered = b->graph != nullptr;
    for (size_t i = 0; i < b->classes.size(); ++i) {
        const auto &c = b->classes[i];
        if (c.slots.empty() && !(b->graph && in_graph((int)i))) continue;
        const int grid = (int)class_grid(b, c);
        sig.push_back((int)i);
        sig.push_back(c.epb);
        sig.push_back(c.ctas_per_sm);
        sig.push_back(grid);
        bool found = false;
        for (size_t j = 0; j + 3 < b->graph_sig.size(); j += 4)
            found = found || (b->graph_sig[j] == (int)i && b->graph_sig[j + 1] == c.epb &&
                              b->graph_sig[j + 2] == c.ctas_per_sm && b->graph_sig[j + 3] >= grid);
        covered = covered && found;
    }
    if (covered) {
        b->dirty = false;
        return 0;
    }
    release_batch_graph(b);
    cudaGraph_t g = nullptr;
    HGG_BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int64_t before = b->launches;
    cudaEventRecord(b->fork, b->stream);
    for (size_t j = 0; j + 3 < sig.size(); j += 4) {
        BatchClass &c = b->classes[sig[j]];
        cudaStreamWaitEvent(c.stream, b->fork, 0);
        for (int st = 0; st < c.S; ++st) launch_class_stage(b, c, st, c.stream);
        cudaEventRecord(c.done, c.stream);
        cudaStreamWaitEvent(b->stream, c.done, 0);
        c.grid_floor = (unsigned)sig[j + 3];
    }
    batch_advance<<<(b->cap + 255) / 256, 256, 0, b->stream>>>(b->d_parity, b->d_remaining, b->cap);
    cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    b->launches = before;
    if (ce != cudaSuccess) return bfail(b, HGG_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(ce));
    cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return bfail(b, HGG_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(ie));
    b->graph_sig = sig;
    b->dirty = false;
    return 0;
}

// kernels of one captured step: each class in it launches its S stages (tensor-core
// classes also form the split stage input before each stage), then the counters advance
int launches_per_step(const hgg_batch *b) {
    int n = 1;
    for (size_t j = 0; j < b->graph_sig.size(); j += 4) {
        const BatchClass &c = b->classes[b->graph_sig[j]];
        n += c.kind == KIND_UMMA ? 2 * c.S : c.S;
    }
    return n;
}

void destroy_batch(hgg_batch *b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    release_batch_graph(b);
    for (auto &c : b->classes) {
        if (c.stream) cudaStreamSynchronize(c.stream);
        for (void *p : c.d_items) cudaFreeAsync(p, b->stream);
        for (int i = 0; i < 2; ++i) {
            if (c.h_up[i]) cudaFreeHost(c.h_up[i]);
            if (c.up_done[i]) cudaEventDestroy(c.up_done[i]);
        }
        cudaFreeAsync(c.d_n, b->stream);
        cudaFreeAsync(c.d_total, b->stream);
        if (c.done) cudaEventDestroy(c.done);
        if (c.stream) cudaStreamDestroy(c.stream);
    }
    cudaFree(b->d_parity);
    cudaFree(b->d_remaining);
    cudaFree(b->d_status);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

// takes the member of `slot` out of the batch, given the parity of its buffers after its
// last step: host bookkeeping, and a reset of its counters ordered after the steps already
// issued (no wait for the stream); the tables are rewritten before the next step
int remove_member(hgg_batch *b, int slot, int parity) {
    hgg_handle *h = b->handles[slot];
    h->cur = parity ? 1 - b->base[slot] : b->base[slot];
    BatchClass &c = b->classes[b->cls[slot]];
    c.slots.erase(std::find(c.slots.begin(), c.slots.end(), slot));
    c.table_dirty = true;
    b->handles[slot] = nullptr;
    b->cls[slot] = -1;
    b->remaining_host[slot] = 0;
    b->item_cache[slot].clear();
    batch_set_slot<<<1, 1, 0, b->stream>>>(b->d_parity, b->d_remaining, slot, 0);
    HGG_BCUDA(b, cudaGetLastError());
    b->dirty = true;
    return 0;
}

}  // namespace

extern "C" {

int hgg_batch_create(int32_t capacity, hgg_batch **out) {
    if (!out || capacity < 1 || capacity > (1 << 20)) return bfail(nullptr, HGG_ERR_INVALID, "capacity must be 1..2^20");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return bfail(nullptr, HGG_ERR_NOT_LOADED, "no CUDA device available");
    auto *b = new hgg_batch();
    b->cap = capacity;
    b->handles.assign(capacity, nullptr);
    b->dt.assign(capacity, 0.0);
    b->base.assign(capacity, 0);
    b->cls.assign(capacity, -1);
    b->remaining_host.assign(capacity, 0);
    b->item_cache.assign(capacity, {});
    b->cache_epb.assign(capacity, -1);
    b->slot_blocks.assign(capacity, 0);
    b->parity_host.assign(capacity, 0);
    auto fail_create = [&](cudaError_t e, const char *what) {
        g_batch_create_error = std::string(what) + ": " + cudaGetErrorString(e);
        destroy_batch(b);
        return HGG_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaGetDevice(&b->device)) != cudaSuccess) return fail_create(e, "cudaGetDevice");
    if ((e = cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device)) != cudaSuccess)
        return fail_create(e, "cudaDeviceGetAttribute");
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail_create(e, "cudaStreamCreateWithFlags");
    if ((e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess)
        return fail_create(e, "cudaEventCreate");
    if ((e = cudaMalloc(&b->d_parity, sizeof(int) * capacity)) != cudaSuccess) return fail_create(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->d_remaining, sizeof(int) * capacity)) != cudaSuccess) return fail_create(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->d_status, sizeof(int))) != cudaSuccess) return fail_create(e, "cudaMalloc");
    cudaMemsetAsync(b->d_parity, 0, sizeof(int) * capacity, b->stream);
    cudaMemsetAsync(b->d_remaining, 0, sizeof(int) * capacity, b->stream);
    cudaMemsetAsync(b->d_status, 0, sizeof(int), b->stream);
    if ((e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return fail_create(e, "cudaStreamSynchronize");
    *out = b;
    return 0;
}

int hgg_batch_destroy(hgg_batch *b) {
    destroy_batch(b);
    return 0;
}

const char *hgg_batch_last_error(const hgg_batch *b) { return b ? b->err.c_str() : g_batch_create_error.c_str(); }

int hgg_batch_add(hgg_batch *b, hgg_handle *h, double dt, int32_t nsteps, int32_t *slot) {
    if (!b || !h || !slot) return bfail(b, HGG_ERR_INVALID, "null argument");
    if (nsteps < 0 || !(dt > 0.0)) return bfail(b, HGG_ERR_INVALID, "dt must be positive and nsteps >= 0");
    if (h->device != b->device) return bfail(b, HGG_ERR_INVALID, "handle and batch are on different devices");
    int free_slot = -1;
    for (int i = 0; i < b->cap; ++i) {
        if (b->handles[i] == h) return bfail(b, HGG_ERR_INVALID, "handle is already in the batch");
        if (free_slot < 0 && !b->handles[i]) free_slot = i;
    }
    if (free_slot < 0) return bfail(b, HGG_ERR_INVALID, "batch is full");
    if (h->src) return bfail(b, HGG_ERR_UNSUPPORTED, "handles with source terms are stepped on their own");
    if (h->linear && h->lin_tiles == 0)
        return bfail(b, HGG_ERR_UNSUPPORTED, "stored-matrix handles without tiles are stepped on their own");
    if (!h->slice_ok && !h->op.tensor && dense_R(h) > 256)
        return bfail(b, HGG_ERR_UNSUPPORTED, "dense kernel: more than 256 coefficients per element");
    // the handle's own work must be finished before the batch uses its buffers
    HGG_BCUDA(b, cudaStreamSynchronize(h->stream));
    int ci = -1;
    for (size_t i = 0; i < b->classes.size(); ++i)
        if (same_class(b->classes[i], h)) ci = (int)i;
    if (ci < 0) {
        BatchClass c;
        c.kind = batch_kind(h);
        c.shape = h->op.shape;
        c.order = h->op.order;
        c.dim = h->op.dim;
        c.physics = h->op.physics;
        c.mixed = h->mixed;
        c.S = h->S;
        c.rk_a = h->rk_a;
        c.rk_b = h->rk_b;
        c.precision = h->precision;
        c.rows = h->lin_R;
        c.lslots = h->lin_slots;
        c.rep.shape = h->op.shape;
        c.rep.dim = h->op.dim;
        c.rep.order = h->op.order;
        c.rep.nB = h->op.nB;
        c.rep.V = h->op.V;
        c.rep.physics = h->op.physics;
        c.rep.nfl = h->op.nfl;
        c.rep.np = h->op.np;
        c.rep.D1 = h->op.D1;
        c.rep.lift = h->op.lift;
        c.rep.trace_pos[0] = h->op.trace_pos[0];
        c.rep.trace_pos[1] = h->op.trace_pos[1];
        c.epb = c.kind == KIND_DENSE ? std::max(1, 256 / dense_rows(h->op.dim, h->op.physics != HGG_PHYSICS_ADVECTION, h->op.nB)) : 1;
        c.item_bytes = class_item_bytes(c);
        c.d_items.assign(c.S, nullptr);
        for (int st = 0; st < c.S; ++st)
            HGG_BCUDA(b, cudaMallocAsync(&c.d_items[st], c.item_bytes * (size_t)b->cap, b->stream));
        HGG_BCUDA(b, cudaMallocAsync(&c.d_n, sizeof(int), b->stream));
        HGG_BCUDA(b, cudaMallocAsync(&c.d_total, sizeof(int64_t) * (1 + (size_t)b->cap), b->stream));
        HGG_BCUDA(b, cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
        HGG_BCUDA(b, cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming));
        b->classes.push_back(std::move(c));
        ci = (int)b->classes.size() - 1;
        // default persistent grid: as many CTAs per SM as the class's kernel fits (the
        // autotuner, where on, times the alternatives)
        b->occ_query = true;
        b->occ_result = 0;
        launch_class_stage(b, b->classes[ci], 0, b->stream);
        b->occ_query = false;
        if (b->occ_result > 0) b->classes[ci].ctas_per_sm = std::min(b->occ_result, 8);
    }
    b->classes[ci].slots.push_back(free_slot);
    b->classes[ci].table_dirty = true;
    b->item_cache[free_slot].clear();  // formed at the next table upload
    b->handles[free_slot] = h;
    b->dt[free_slot] = dt;
    b->base[free_slot] = h->cur;
    b->cls[free_slot] = ci;
    b->remaining_host[free_slot] = nsteps;
    b->parity_host[free_slot] = 0;
    // ordered after every step already issued, in which the slot is free or its
    // previous member has no steps left
    batch_set_slot<<<1, 1, 0, b->stream>>>(b->d_parity, b->d_remaining, free_slot, nsteps);
    HGG_BCUDA(b, cudaGetLastError());
    b->dirty = true;
    *slot = free_slot;
    return 0;
}

int hgg_batch_remove(hgg_batch *b, int32_t slot) {
    if (!b || slot < 0 || slot >= b->cap || !b->handles[slot]) return bfail(b, HGG_ERR_INVALID, "bad slot");
    int rc = read_counters(b);
    if (rc) return rc;
    return remove_member(b, slot, b->parity_host[slot]);
}

int hgg_batch_step(hgg_batch *b, int32_t nsteps) {
    if (!b || nsteps < 0) return bfail(b, HGG_ERR_INVALID, "bad argument");
    if (nsteps == 0) return 0;
    bool any = false;
    for (auto &c : b->classes) any = any || !c.slots.empty();
    if (!any) return 0;
    int rc = prepare_batch(b);
    if (rc) return rc;
    for (int s = 0; s < nsteps; ++s) HGG_BCUDA(b, cudaGraphLaunch(b->graph, b->stream));
    b->launches += (int64_t)nsteps * launches_per_step(b);
    return 0;
}

int hgg_batch_synchronize(hgg_batch *b) {
    if (!b) return bfail(b, HGG_ERR_INVALID, "null batch");
    int rc = read_counters(b);
    if (rc) return rc;
    int st = 0;
    HGG_BCUDA(b, cudaMemcpyAsync(&st, b->d_status, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    HGG_BCUDA(b, cudaStreamSynchronize(b->stream));
    if (st) return bfail(b, HGG_ERR_DEVICE, status_message(st));
    // keep each member handle's notion of its current buffer up to date
    for (int i = 0; i < b->cap; ++i)
        if (b->handles[i]) b->handles[i]->cur = b->parity_host[i] ? 1 - b->base[i] : b->base[i];
    return 0;
}

int32_t hgg_batch_remaining(const hgg_batch *b, int32_t slot) {
    if (!b || slot < 0 || slot >= b->cap || !b->handles[slot]) return -1;
    return b->remaining_host[slot];
}

int hgg_batch_set_autotune(hgg_batch *b, int32_t enable) {
    if (!b) return bfail(b, HGG_ERR_INVALID, "null batch");
    b->autotune = enable != 0;
    return 0;
}

int64_t hgg_batch_launch_count(const hgg_batch *b) { return b ? b->launches : -1; }

int32_t hgg_batch_num_classes(const hgg_batch *b) {
    if (!b) return -1;
    int n = 0;
    for (auto &c : b->classes) n += !c.slots.empty();
    return n;
}

void *hgg_batch_stream(const hgg_batch *b) { return b ? (void *)b->stream : nullptr; }

int hgg_batch_class_info(const hgg_batch *b, int32_t i, int64_t *info10) {
    if (!b || !info10) return HGG_ERR_INVALID;
    int k = -1;
    for (size_t j = 0; j < b->classes.size(); ++j) {
        if (b->classes[j].slots.empty()) continue;
        if (++k != i) continue;
        const BatchClass &c = b->classes[j];
        int64_t dofs = 0, elements = 0;
        for (int slot : c.slots) {
            const hgg_handle *h = b->handles[slot];
            dofs += h->N;
            elements += h->op.nE;
        }
        const int64_t v[10] = {c.kind, c.shape, c.dim, c.order, c.physics, c.precision,
                               c.S, (int64_t)c.slots.size(), elements, dofs};
        std::copy(v, v + 10, info10);
        return 0;
    }
    return HGG_ERR_INVALID;
}

int hgg_batch_profile_step(hgg_batch *b, double *ms, int32_t n) {
    if (!b || !ms || n < hgg_batch_num_classes(b)) return bfail(b, HGG_ERR_INVALID, "bad argument");
    int rc = prepare_batch(b);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    HGG_BCUDA(b, cudaEventCreate(&e0));
    HGG_BCUDA(b, cudaEventCreate(&e1));
    int k = 0;
    for (auto &c : b->classes) {
        if (c.slots.empty()) continue;
        cudaEventRecord(e0, b->stream);
        for (int st = 0; st < c.S; ++st) launch_class_stage(b, c, st, b->stream);
        cudaEventRecord(e1, b->stream);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return bfail(b, HGG_ERR_CUDA, std::string("profiled step: ") + cudaGetErrorString(e));
        }
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        ms[k++] = t;
    }
    batch_advance<<<(b->cap + 255) / 256, 256, 0, b->stream>>>(b->d_parity, b->d_remaining, b->cap);
    b->launches++;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    HGG_BCUDA(b, cudaStreamSynchronize(b->stream));
    return 0;
}

}  // extern "C"
