// Stage launches of the dense kernels (simplices, the wave, lines) and of the
// stored-matrix kernels (HpgemAPILinear and folded operators).
#include <algorithm>
#include <type_traits>

#include "handle.cuh"

namespace hgg {

// wave speed factor of the upwind wave flux, 0 for the central flux
double upwind_speed(const HostOperators &op) {
    return op.physics == HGG_PHYSICS_WAVE_UPWIND ? 1.0 / std::sqrt(op.c_inv) : 0.0;
}

namespace {

template <typename KT, int DIM, int NFL, int WAVE>
int launch_dense(hgg_handle *h, const StageIOT<KT> &io) {
    const HostOperators &op = h->op;
    const int V = WAVE ? DIM + 1 : 1;
    const int R = V * op.nB;
    if (R > 256) return fail(h, HGG_ERR_UNSUPPORTED, "dense kernel: more than 256 coefficients per element");
    int epb = std::max(1, 256 / dense_rows(DIM, WAVE, op.nB));
    DenseGeom g{h->d_vol, h->d_pairs, h->d_vol_f, h->d_pairs_f, h->d_nbr, h->d_self, h->d_nbrp, h->d_mode,
                h->d_elem_geo, h->d_face_geo, 1.0 / op.c_inv, upwind_speed(op), op.nB, epb};
    int64_t blocks = (op.nE + epb - 1) / epb;
    const int threads = dense_threads(DIM, WAVE, op.nB, epb);
    const bool ok = dense_dispatch<DIM, NFL, WAVE>(op.nB, [&](auto nbc) {
        constexpr int NB = decltype(nbc)::value;
        // the grouped kernel where it measured faster (group_wave_wanted): the wave with
        // FP64 contractions (32^3 x 5 tetrahedra, p = 2, RK4: 1.12 against 2.01 ms per
        // step upwind when it was introduced), and with FP32 contractions on the meshes
        // and orders listed there; for advection the per-row kernel was as fast (0.38 both)
        if constexpr (DIM >= 2 && NB <= kGroupMaxBasis && WAVE) {
            const bool want = group_wave_wanted(h);
            if (h->group_tiles > 0 && want) {
                constexpr size_t gsmem = group_smem<DenseCT<KT, NB>, DIM, NFL, NB>();
                if (gsmem > 48 * 1024)
                    cudaFuncSetAttribute(dense_group_stage<KT, DIM, NFL, NB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsmem);
                dense_group_stage<KT, DIM, NFL, NB>
                    <<<(unsigned)h->group_tiles, group_threads(NB), gsmem, h->stream>>>(io, g, h->d_group_tiles);
                return;
            }
        }
        const size_t smem = dense_smem(DIM, NFL, WAVE, NB, epb, sizeof(DenseCT<KT, NB>));
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(dense_stage<KT, DIM, NFL, WAVE, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        dense_stage<KT, DIM, NFL, WAVE, NB><<<(unsigned)blocks, threads, smem, h->stream>>>(io, g);
    });
    if (!ok) return fail(h, HGG_ERR_UNSUPPORTED, "dense kernel: no kernel for this basis size");
    return 0;
}

template <typename KT>
int launch_dense_any(hgg_handle *h, const StageIOT<KT> &io) {
    const bool wave = h->op.physics != HGG_PHYSICS_ADVECTION;
    switch (h->op.shape) {
        case HGG_SHAPE_LINE: return wave ? launch_dense<KT, 1, 2, 1>(h, io) : launch_dense<KT, 1, 2, 0>(h, io);
        case HGG_SHAPE_TRIANGLE: return wave ? launch_dense<KT, 2, 3, 1>(h, io) : launch_dense<KT, 2, 3, 0>(h, io);
        case HGG_SHAPE_SQUARE: return wave ? launch_dense<KT, 2, 4, 1>(h, io) : launch_dense<KT, 2, 4, 0>(h, io);
        case HGG_SHAPE_TETRAHEDRON: return wave ? launch_dense<KT, 3, 4, 1>(h, io) : launch_dense<KT, 3, 4, 0>(h, io);
        case HGG_SHAPE_CUBE: return wave ? launch_dense<KT, 3, 6, 1>(h, io) : launch_dense<KT, 3, 6, 0>(h, io);
    }
    return fail(h, HGG_ERR_UNSUPPORTED, "shape");
}

// the mixed forms on the tensor cores: the split stage input (planes), then
// persistent CTAs over the 128-element tiles
int launch_umma(hgg_handle *h, const StageIOT<float> &io) {
    const int kind = h->precision == HGG_PRECISION_BF16X3 ? kUmmaBF16 : kUmmaTF32;
    const UmmaShape sh = umma_shape(h->lin_R, h->lin_slots, kind);
    UmmaArgs a{h->d_umma_img, h->d_umma_planes, h->d_umma_tile_elems, h->d_umma_tile_mats, h->d_lin_nbr,
               h->umma_tiles, h->lin_mats, kUmmaPolls};
    const size_t smem = umma_smem(sh);
    const unsigned grid = (unsigned)std::min<int64_t>(h->umma_tiles, h->num_sms);
    const int64_t chunks = h->op.nE * (sh.KP * sh.es / 16);
    const unsigned pgrid = (unsigned)std::min<int64_t>((chunks + 255) / 256, (int64_t)h->num_sms * 8);
    // vector loads need 16-byte aligned rows (R a multiple of 4) and at most one stage-input vector
    const int nin = (h->lin_R % 4 == 0 && io.nin <= 1) ? io.nin : -1;
    auto planes = [&](auto kc, auto nc) {
        constexpr int K = decltype(kc)::value, NIN = decltype(nc)::value;
        umma_planes<K, NIN><<<pgrid, 256, 0, h->stream>>>(io, h->d_umma_planes, sh.R, sh.KP);
    };
    auto tiles = [&](auto kc) {
        constexpr int K = decltype(kc)::value;
        cudaFuncSetAttribute(linear_umma_stage<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        linear_umma_stage<K><<<grid, kUmmaThreads, smem, h->stream>>>(io, a, sh);
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
    h->launches++;  // the planes launch (the tile launch is counted by the caller)
    return 0;
}

template <typename KT>
int launch_linear(hgg_handle *h, const StageIOT<KT> &io) {
    if constexpr (std::is_same_v<KT, float>) {
        if (h->umma_tiles > 0) return launch_umma(h, io);
    }
    const int R = h->lin_R;
    const int epb = std::max(1, 256 / R);
    LinearGeom g{h->d_lin_table, h->d_lin_table_rm, h->d_lin_table_f, h->d_lin_self, h->d_lin_nbr, h->d_lin_mat,
                 R, h->lin_slots, epb, h->lin_mats};
    if (h->lin_tiles > 0) {
        LinearTiles t{h->d_lin_tile_elems, h->d_lin_tile_mats};
        linear_tile_stage<KT><<<(unsigned)h->lin_tiles, 256, 0, h->stream>>>(io, g, t);
        return 0;
    }
    const unsigned blocks = (unsigned)((h->op.nE + epb - 1) / epb);
    const int threads = linear_threads(R, epb);
    auto go = [&](auto ct) {
        using CT = decltype(ct);
        const size_t smem = linear_smem(R, h->lin_slots, epb, sizeof(CT));
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(linear_stage<KT, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        linear_stage<KT, CT><<<blocks, threads, smem, h->stream>>>(io, g);
    };
    if (std::is_same_v<KT, float> && h->d_lin_table_f) go(float{});
    else go(double{});
    return 0;
}

}  // namespace

int launch_stage_dense(hgg_handle *h, const StageIOT<double> &io) { return launch_dense_any<double>(h, io); }
int launch_stage_dense(hgg_handle *h, const StageIOT<float> &io) { return launch_dense_any<float>(h, io); }
int launch_stage_linear(hgg_handle *h, const StageIOT<double> &io) { return launch_linear<double>(h, io); }
int launch_stage_linear(hgg_handle *h, const StageIOT<float> &io) { return launch_linear<float>(h, io); }

}  // namespace hgg
