// Stage launches of the sum-factorised kernels: the slice kernel (hexahedra,
// p = 3), the pipelined kernel and the one-shot kernel (other squares and cubes).
#include <algorithm>
#include <type_traits>

#include "handle.cuh"

namespace hgg {

namespace {

template <typename KT>
int launch_slice(hgg_handle *h, const StageIOT<KT> &io) {
    const HostOperators &op = h->op;
    SliceOps sops;
    for (int i = 0; i < 16; ++i) sops.D[i] = op.D1[i];
    for (int sd = 0; sd < 2; ++sd)
        for (int a = 0; a < 4; ++a) sops.L[sd][a] = op.lift[sd * 4 + a];
    const int64_t blocks = (op.nE + SliceShape::TE - 1) / SliceShape::TE;
    const dim3 grid((unsigned)blocks), block(SliceShape::THREADS);
    const bool fin = io.unew != nullptr;
    // each block asks L2 for the inputs of the tile a block of the next resident wave runs
    // (5 blocks per SM resident): measured 4 % faster per RK4 step for the FP32 form and
    // 2-3 % for the FP64 form's first three stages; the FP64 final stage (4 resident
    // blocks, three more input vectors) measured slower with it and goes without
    const int64_t ahead = (sizeof(KT) == 4 || !io.unew) ? (int64_t)h->num_sms * 5 : 0;
    if (io.nin == 0 && (!fin || io.nfin == 0))
        tensor_slice<KT, 0, 0><<<grid, block, 0, h->stream>>>(io, h->d_slice_geo, sops, ahead);
    else if (io.nin == 1 && (!fin || io.nfin == 0))
        tensor_slice<KT, 1, 0><<<grid, block, 0, h->stream>>>(io, h->d_slice_geo, sops, ahead);
    else if (io.nin == 1 && fin && io.nfin == 3)
        tensor_slice<KT, 1, 3><<<grid, block, 0, h->stream>>>(io, h->d_slice_geo, sops, ahead);
    else
        tensor_slice<KT, -1, -1><<<grid, block, 0, h->stream>>>(io, h->d_slice_geo, sops, ahead);
    return 0;
}

// shared memory of the pipelined kernel for a ring of `nbuf` slots of `nv` vectors
template <int P, int DIM>
size_t pipe_smem(int nbuf, int nv) {
    using S = PipeShape<P, DIM>;
    size_t tab_end = (64 + 8 * (S::NP * S::NP + 2 * S::NP + S::NB) + 4 * S::NB + 127) / 128 * 128;
    size_t slot = (size_t)nv * S::TILE_VEC_BYTES + S::TILE_GEO_BYTES;
    size_t tail = 8 * ((size_t)S::TE * S::NB * 3 + (size_t)S::TE * S::NS * S::NF);
    return tab_end + nbuf * slot + tail;
}

template <int P, int DIM>
int launch_tensor(hgg_handle *h, const StageIO &io) {
    using TC = TensorConsts<P, DIM>;
    const HostOperators &op = h->op;
    TC tc = tensor_consts<P, DIM>(op);
    using S = PipeShape<P, DIM>;
    PipeArgs pa;
    pa.nv = 1 + io.nin + (io.unew ? io.nfin : 0);
    pa.slot_bytes = (uint32_t)((size_t)pa.nv * S::TILE_VEC_BYTES + S::TILE_GEO_BYTES);
    // two blocks per SM when a ring of >= 3 slots fits, else one block with up to 8 slots
    const size_t budget = 227 * 1024;
    int per_sm = 2, nbuf = 0;
    for (int b = 8; b >= 3; --b)
        if (2 * (pipe_smem<P, DIM>(b, pa.nv) + 1024) <= budget) { nbuf = b; break; }
    if (!nbuf) {
        per_sm = 1;
        for (int b = 8; b >= 2; --b)
            if (pipe_smem<P, DIM>(b, pa.nv) <= budget) { nbuf = b; break; }
    }
    if (!nbuf && h->variant == 2)
        return fail(h, HGG_ERR_UNSUPPORTED, "pipelined kernel: tile does not fit in shared memory");
    // the one-shot kernel when asked for, or when a stage reads too many vectors for the ring
    if (h->variant == 1 || !nbuf) {
        constexpr int EPB = (256 / TC::NB) > 0 ? (256 / TC::NB) : 1;
        TensorGeom geo{h->d_ahat, h->d_tnbr, h->d_tmode, h->d_tsigma};
        int64_t blocks = (op.nE + EPB - 1) / EPB;
        tensor_stage<double, P, DIM, EPB><<<(unsigned)blocks, EPB * TC::NB, 0, h->stream>>>(io, geo, tc);
        return 0;
    }
    pa.geo = h->d_pgeo;
    pa.n_tiles = (op.nE + S::TE - 1) / S::TE;
    pa.nbuf = nbuf;
    pa.polls = kWaitPolls;
    pa.arm_only = -1;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (h->test_arm_polls && cudaStreamIsCapturing(h->stream, &cap) == cudaSuccess &&
        cap == cudaStreamCaptureStatusNone) {  // hgg_test_arm_without_copy: this launch only
        pa.polls = h->test_arm_polls;
        pa.arm_only = 0;
        h->test_arm_polls = 0;
    }
    size_t smem = pipe_smem<P, DIM>(nbuf, pa.nv);
    cudaFuncSetAttribute(tensor_pipe<P, DIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int64_t grid = std::min<int64_t>(pa.n_tiles, (int64_t)h->num_sms * per_sm);
    tensor_pipe<P, DIM><<<(unsigned)grid, S::THREADS, smem, h->stream>>>(io, pa, tc);
    return 0;
}

}  // namespace

int pipe_tile_elems(int order, int dim) {
#define HGG_TE(P) \
    case P: return dim == 2 ? PipeShape<P, 2>::TE : PipeShape<P, 3>::TE;
    switch (order) { HGG_TE(1) HGG_TE(2) HGG_TE(3) HGG_TE(4) HGG_TE(5) }
#undef HGG_TE
    return 1;
}

int pipe_geo_bytes(int dim) { return dim == 2 ? PipeShape<1, 2>::GEO_BYTES : PipeShape<1, 3>::GEO_BYTES; }

template <int DIM>
int launch_tensor_dim(hgg_handle *h, const StageIO &io) {
    switch (h->op.order) {
        case 1: return launch_tensor<1, DIM>(h, io);
        case 2: return launch_tensor<2, DIM>(h, io);
        case 3: return launch_tensor<3, DIM>(h, io);
        case 4: return launch_tensor<4, DIM>(h, io);
        case 5: return launch_tensor<5, DIM>(h, io);
    }
    return fail(h, HGG_ERR_UNSUPPORTED, "tensor kernel: order out of range");
}

namespace {

template <int DIM>
int launch_tensor_oneshot_f(hgg_handle *h, const StageIOT<float> &io) {
    auto go = [&](auto pc) {
        constexpr int P = decltype(pc)::value;
        using TC = TensorConsts<P, DIM>;
        constexpr int EPB = (256 / TC::NB) > 0 ? (256 / TC::NB) : 1;
        const TC tc = tensor_consts<P, DIM>(h->op);
        TensorGeom geo{h->d_ahat, h->d_tnbr, h->d_tmode, h->d_tsigma};
        const int64_t blocks = (h->op.nE + EPB - 1) / EPB;
        tensor_stage<float, P, DIM, EPB><<<(unsigned)blocks, EPB * TC::NB, 0, h->stream>>>(io, geo, tc);
        return 0;
    };
    switch (h->op.order) {
        case 1: return go(std::integral_constant<int, 1>{});
        case 2: return go(std::integral_constant<int, 2>{});
        case 3: return go(std::integral_constant<int, 3>{});
        case 4: return go(std::integral_constant<int, 4>{});
        case 5: return go(std::integral_constant<int, 5>{});
    }
    return fail(h, HGG_ERR_UNSUPPORTED, "tensor kernel: order out of range");
}

}  // namespace

int launch_stage_tensor(hgg_handle *h, const StageIO &io) {
    if (h->slice_ok) return launch_slice<double>(h, io);
    return h->op.dim == 2 ? launch_tensor_dim<2>(h, io)
                          : (h->op.dim == 3 ? launch_tensor_dim<3>(h, io)
                                            : fail(h, HGG_ERR_UNSUPPORTED, "tensor kernel needs dim 2 or 3"));
}

int launch_stage_tensor(hgg_handle *h, const StageIOT<float> &io) {
    if (h->slice_ok) return launch_slice(h, io);
    return h->op.dim == 2 ? launch_tensor_oneshot_f<2>(h, io)
                          : (h->op.dim == 3 ? launch_tensor_oneshot_f<3>(h, io)
                                            : fail(h, HGG_ERR_UNSUPPORTED, "tensor kernel needs dim 2 or 3"));
}

}  // namespace hgg
