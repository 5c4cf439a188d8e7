// C ABI of hpgem_b200 (include/hpgem_b200.h): handle management, device
// buffers, stage launches and CUDA-graph capture of the Runge-Kutta step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <sstream>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "handle.cuh"

using namespace hgg;

namespace {

thread_local std::string g_create_error = "no error";

}  // namespace

namespace hgg {

int fail(hgg_handle *h, int code, const std::string &msg) {
    if (h) h->err = msg;
    else g_create_error = msg;
    return code;
}



int alloc(hgg_handle *h, size_t bytes, void **dst) {
    void *p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, h->stream);
    if (e != cudaSuccess) return fail(h, HGG_ERR_NOMEM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    h->bufs.push_back({p, bytes});
    *dst = p;
    return 0;
}

int solution_to_host(hgg_handle *h, double *staging, double *out) {
    const double *d = h->sol[h->cur];
    const int64_t n = h->tensor_layout ? h->N_alloc : h->N;
    HGG_CUDA(h, cudaMemcpyAsync(staging, d, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    HGG_CUDA(h, cudaStreamSynchronize(h->stream));
    if (!h->tensor_layout) {
        std::memcpy(out, staging, sizeof(double) * h->N);
        return 0;
    }
    const int nb = h->op.nB;
    const int64_t ne = h->N / nb;
    for (int64_t e = 0; e < ne; ++e)
        for (int k = 0; k < nb; ++k)
            out[e * nb + k] = h->op.tsign[k] * staging[device_index(e, (int)h->op.tpos[k], nb, h->tiled)];
    return 0;
}

void release_graphs(hgg_handle *h) {
    for (auto &g : h->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}
// ---- kernel dispatch ---------------------------------------------------------
// The device vectors of a sum-factorised handle are already in tensor order
// with the signs folded in, so the kernels see the identity permutation.

// layout conversion kernels (hpGEM order <-> tensor order, signs folded; tiled:
// 32-element tiles, coefficient-major inside a tile)

template <typename TD>
__global__ void to_tensor_order(const double *src, TD *dst, const int32_t *tpos, const double *tsign,
                                int nb, int64_t n, bool tiled) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = i / nb;
        const int k = (int)(i - e * nb);
        dst[device_index(e, tpos[k], nb, tiled)] = (TD)(tsign[k] * src[i]);
    }
}
template <typename TS>
__global__ void from_tensor_order(const TS *src, double *dst, const int32_t *tpos, const double *tsign,
                                  int nb, int64_t n, bool tiled) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = i / nb;
        const int k = (int)(i - e * nb);
        dst[i] = tsign[k] * (double)src[device_index(e, tpos[k], nb, tiled)];
    }
}
// zeros the coefficients of the padding elements [n_elements, n_pad) of a device vector
__global__ void zero_padding(double *v, int nb, int64_t n_elements, int64_t n_pad, bool tiled) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (n_pad - n_elements) * nb) return;
    const int64_t e = n_elements + i / nb;
    v[device_index(e, (int)(i % nb), nb, tiled)] = 0.0;
}
// plain precision conversion of a vector (FP32-mixed stage vectors without layout change)
__global__ void convert_vector(const double *src, float *dst, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}
__global__ void convert_vector(const float *src, double *dst, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}
int launch_stage(hgg_handle *h, const StageIO &io) {
    int rc;
    if (h->linear) rc = launch_stage_linear(h, io);
    else if (h->slice_ok || h->op.tensor) rc = launch_stage_tensor(h, io);
    else rc = launch_stage_dense(h, io);
    if (rc) return rc;
    h->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(h, HGG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return 0;
}

// FP32-mixed form: the stage kernels that have it
int launch_stage(hgg_handle *h, const StageIOT<float> &io) {
    int rc;
    if (h->linear) rc = launch_stage_linear(h, io);
    else if (h->slice_ok || h->op.tensor) rc = launch_stage_tensor(h, io);
    else rc = launch_stage_dense(h, io);
    if (rc) return rc;
    h->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(h, HGG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return 0;
}

// whether the mixed form has a kernel for this handle's shape and order (all have)
bool mixed_supported(const hgg_handle *h) { return h != nullptr; }

void *vector_ptr(hgg_handle *h, int vec) {
    if (vec == 0) return h->sol[h->cur];
    if (vec >= 1 && vec <= h->S) return h->k[vec - 1];
    return nullptr;
}
bool vector_is_float(const hgg_handle *h, int vec) { return h->mixed && vec >= 1; }


// the stages run the grouped wave kernel (the choice launch_dense makes) and every stage
// input has exactly one earlier vector, the previous one: each stage then forms the next
// stage's input in its output phase (the value the next stage would form itself)
bool group_wave_wanted(const hgg_handle *h) {
    if (h->group_tiles <= 0 || h->linear || h->op.tensor) return false;
    if (h->variant == 2) return true;
    if (h->variant != 0) return false;
    const int nb = h->op.nB;
    // 16-element tiles (above 24 basis functions): faster on large meshes only (RK4 steps:
    // tetrahedra p = 4 on 24^3 x 5 cells 4.21 against 4.65 ms, quadrilaterals p = 4 on
    // 192^2 0.88 against 1.08; equal on 16^3 x 5 tetrahedra and hexahedra p = 2 on 40^3)
    if (nb > kGroupMaxRows) return h->op.nE >= 65536;
    if (!h->mixed || nb > kMixedFp32MaxBasis) return true;  // FP64 contractions
    // FP32 contractions: where the tile kernel measured faster than the per-row one
    // (RK4 steps: tetrahedra p = 1 on 40^3 x 5 cells 0.57 against 0.72 ms, p = 2 on
    // 32^3 x 5 0.83 against 0.92; triangles p = 4 on 256^2 x 2 0.84 against 0.96; meshes
    // below 2^15 elements, e.g. 64^2 x 2 triangles p = 2, 0.035 against 0.045); the
    // per-row kernel elsewhere (tetrahedra p = 3 on 24^3 x 5: 1.06 against 1.24 ms;
    // triangles p <= 3 on large meshes, within 6 %)
    return (h->op.dim == 3 && nb <= 10) || (h->op.dim == 2 && nb >= 15) || h->op.nE < 32768;
}

bool forms_next_input(const hgg_handle *h) {
    if (!h->d_win[0] || h->src || !group_wave_wanted(h)) return false;
    const int S = h->S;
    for (int i = 1; i < S; ++i)
        for (int j = 0; j < i; ++j)
            if ((h->rk_a[i * S + j] != 0.0) != (j == i - 1)) return false;
    return true;
}

template <typename KT>
int enqueue_step_t(hgg_handle *h, int from, double dt) {
    const bool fuse = forms_next_input(h);
    for (int i = 0; i < h->S; ++i) {
        StageIOT<KT> io = make_stage_io<KT>(h, from, dt, i, h->d_status);
        if (fuse) {
            if (i > 0) io.win = h->d_win[(i - 1) & 1];
            if (i < h->S - 1) {
                io.wnext = h->d_win[i & 1];
                io.wcoef = dt * h->rk_a[(i + 1) * h->S + i];
            }
        }
        int rc = launch_stage(h, io);
        if (!rc && h->src) rc = enqueue_source(h, from, i, io.kout, io.unew, io.blast);
        if (rc) return rc;
    }
    return 0;
}

int enqueue_step(hgg_handle *h, int from, double dt) {
    return h->mixed ? enqueue_step_t<float>(h, from, dt) : enqueue_step_t<double>(h, from, dt);
}

uint32_t float_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
float bits_float(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
// BF16 bits of f, rounded to nearest even (f finite)
uint16_t bf16_rn(float f) {
    const uint32_t u = float_bits(f);
    return (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
}

std::string status_message(int st) {
    std::string m = "kernel status word " + std::to_string(st) + ":";
    if (st & 1) m += " bad neighbour index (bit 0);";
    if (st & 2) m += " a bounded wait ran out (bit 1);";
    if (st & 4) m += " bad matrix index (bit 2);";
    if (st & ~7) m += " unknown bits;";
    m.pop_back();
    return m;
}

int check_status(hgg_handle *h) {
    int st = 0;
    HGG_CUDA(h, cudaMemcpyAsync(&st, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    HGG_CUDA(h, cudaStreamSynchronize(h->stream));
    if (st) return fail(h, HGG_ERR_DEVICE, status_message(st));
    return 0;
}

// Butcher tableau and precision shared by both descriptors
int set_tableau(hgg_handle *h, int32_t n_stages, const double *a, const double *b, const double *c,
                int32_t precision) {
    if (n_stages < 1 || n_stages > kMaxStages || !a || !b)
        return fail(h, HGG_ERR_INVALID, "Butcher tableau must have 1..8 stages");
    h->S = n_stages;
    h->rk_a.assign(a, a + h->S * h->S);
    h->rk_b.assign(b, b + h->S);
    h->rk_c = c ? std::vector<double>(c, c + h->S) : std::vector<double>(h->S, 0.0);
    if (precision != HGG_PRECISION_FP64 && precision != HGG_PRECISION_FP32 && precision != HGG_PRECISION_BF16X3)
        return fail(h, HGG_ERR_INVALID,
                    "precision must be HGG_PRECISION_FP64, HGG_PRECISION_FP32 or HGG_PRECISION_BF16X3");
    h->mixed = precision != HGG_PRECISION_FP64;
    h->precision = precision;
    return 0;
}

// device, stream, solution and stage vectors (N_alloc doubles each), status word
int init_device_vectors(hgg_handle *h) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(h, HGG_ERR_NOT_LOADED, "no CUDA device available");
    HGG_CUDA(h, cudaGetDevice(&h->device));
    HGG_CUDA(h, cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    h->stream = h->own_stream;
    // the default pool keeps freed handle memory for the next handles instead of
    // returning it to the driver at every synchronisation (which waits for the device)
    static std::once_flag pool_once;
    std::call_once(pool_once, [&] {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, h->device) == cudaSuccess) {
            uint64_t keep = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    });
    int rc;
    HGG_CUDA(h, cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device));
    for (int i = 0; i < 2; ++i)
        if ((rc = alloc(h, sizeof(double) * h->N_alloc, (void **)&h->sol[i]))) return rc;
    h->k.resize(h->S);
    for (int i = 0; i < h->S; ++i)
        if ((rc = alloc(h, (h->mixed ? sizeof(float) : sizeof(double)) * h->N_alloc, &h->k[i]))) return rc;
    for (int i = 0; i < 2; ++i) HGG_CUDA(h, cudaMemsetAsync(h->sol[i], 0, sizeof(double) * h->N_alloc, h->stream));
    for (int i = 0; i < h->S; ++i)
        HGG_CUDA(h, cudaMemsetAsync(h->k[i], 0, (h->mixed ? sizeof(float) : sizeof(double)) * h->N_alloc, h->stream));
    if ((rc = alloc(h, sizeof(int), (void **)&h->d_status))) return rc;
    HGG_CUDA(h, cudaMemsetAsync(h->d_status, 0, sizeof(int), h->stream));
    return 0;
}

// tiles_only: 0 attach in any case; 1 only when a tile kernel (FP64 tensor-core
// DMMA tiles or the tcgen05 tiles of the mixed forms) will run; 2 only for the
// tcgen05 tiles
int attach_linear(hgg_handle *h, const LinearSystem &sys, int tiles_only = 0);

// linear: the handle will run the stored-matrix kernel (attach_linear), so the
// vectors stay in hpGEM order and the matrix-free operators are not uploaded
int create_from_desc(const hgg_problem_desc *desc, hgg_handle *h, bool linear = false) {
    try {
        h->op = build_operators(*desc, !linear);
    } catch (const std::exception &ex) {
        return fail(h, HGG_ERR_INVALID, ex.what());
    }
    // split-BF16 runs only as folded tiles on the tensor cores: not the sum-factorised kernels
    if (linear || desc->precision == HGG_PRECISION_BF16X3) h->op.tensor = false;
    int rc = set_tableau(h, desc->n_stages, desc->rk_a, desc->rk_b, desc->rk_c, desc->precision);
    if (rc) return rc;
    const HostOperators &op = h->op;
    h->N = op.nE * op.V * op.nB;
    h->tile_elems = op.tensor ? pipe_tile_elems(op.order, op.dim) : 1;
    h->tensor_layout = op.tensor;
    h->slice_ok = op.tensor && op.dim == 3 && op.order == 3 && op.trace_pos[0] == 0 && op.trace_pos[1] == 1;
    h->tiled = h->slice_ok;
    if (h->slice_ok) h->tile_elems = SliceShape::TE;
    if (h->mixed && !mixed_supported(h))
        return fail(h, HGG_ERR_UNSUPPORTED, "the FP32-mixed form has no kernel for this shape and order");
    const int64_t n_pad = (op.nE + h->tile_elems - 1) / h->tile_elems * h->tile_elems;
    h->N_alloc = n_pad * op.V * op.nB;
    if ((rc = init_device_vectors(h))) return rc;
    if (op.tensor) {
        if ((rc = upload(h, op.elem_geo, &h->d_ahat)) || (rc = upload(h, op.t_nbr, &h->d_tnbr)) ||
            (rc = upload(h, op.t_mode, &h->d_tmode)) || (rc = upload(h, op.t_sigma, &h->d_tsigma)))
            return rc;
        // packed geometry records of the pipelined kernel, padded to whole tiles:
        // ahat[dim], sigma[2 dim] (double), nbr[2 dim] (int32), mode[2 dim] (int8)
        const int d = op.dim, ns = 2 * d, gb = pipe_geo_bytes(d);
        std::vector<unsigned char> pg((size_t)n_pad * gb, 0);
        for (int64_t e = 0; e < op.nE; ++e) {
            unsigned char *r = &pg[(size_t)e * gb];
            double *dd = reinterpret_cast<double *>(r);
            for (int c = 0; c < d; ++c) dd[c] = op.elem_geo[e * d + c];
            for (int s2 = 0; s2 < ns; ++s2) dd[d + s2] = op.t_sigma[e * ns + s2];
            int32_t *ni = reinterpret_cast<int32_t *>(r + 8 * (d + ns));
            for (int s2 = 0; s2 < ns; ++s2) ni[s2] = op.t_nbr[e * ns + s2];
            int8_t *mi = reinterpret_cast<int8_t *>(r + 8 * (d + ns) + 4 * ns);
            for (int s2 = 0; s2 < ns; ++s2) mi[s2] = op.t_mode[e * ns + s2];
        }
        if ((rc = upload(h, pg, &h->d_pgeo))) return rc;
        if (h->slice_ok) {
            // slice kernel records, padded to whole tiles: ahat[3], sigma[6] (double),
            // nbr[6] (int32), mode[6] (int8), 2 bytes of padding
            constexpr int GR = SliceShape::GR;
            std::vector<double> rec((size_t)n_pad * GR, 0.0);
            for (int64_t e = 0; e < op.nE; ++e) {
                double *r = &rec[(size_t)e * GR];
                for (int c = 0; c < 3; ++c) r[c] = op.elem_geo[e * 3 + c];
                for (int s2 = 0; s2 < 6; ++s2) r[3 + s2] = op.t_sigma[e * 6 + s2];
                int32_t *ni = reinterpret_cast<int32_t *>(r + 9);
                int8_t *mi = reinterpret_cast<int8_t *>(r + 12);
                for (int s2 = 0; s2 < 6; ++s2) {
                    ni[s2] = op.t_nbr[e * 6 + s2];
                    mi[s2] = op.t_mode[e * 6 + s2];
                }
            }
            if ((rc = upload(h, rec, &h->d_slice_geo))) return rc;
        }
        // layout conversion tables and scratch vector
        std::vector<int32_t> tp(op.tpos.begin(), op.tpos.end());
        if ((rc = upload(h, tp, &h->d_tpos)) || (rc = upload(h, op.tsign, &h->d_tsign))) return rc;
        if ((rc = alloc(h, sizeof(double) * h->N_alloc, (void **)&h->d_scratch))) return rc;
    } else {
        if (h->mixed && (rc = alloc(h, sizeof(double) * h->N_alloc, (void **)&h->d_scratch))) return rc;
        if (linear) {
            HGG_CUDA(h, cudaStreamSynchronize(h->stream));
            return 0;
        }
        // Folded operator: for advection on triangles of order >= 4 (>= 5 in the
        // mixed form) the element's whole stage is one small dense operator per
        // matrix slot (the reference's integrands assembled once, the mass inverse
        // folded in: the same operator as the matrix-free kernel to rounding), and
        // the grouped FP64 tensor-core kernel of the stored-matrix path applies it
        // faster than the per-row dense kernel (256^2 cells, RK4: 0.39 against 0.46
        // ms per step at p = 4, 0.48 against 0.87 at p = 5; in the mixed form p = 4
        // measured 0.33 against 0.29 and stays on the dense kernel).  Only when the
        // mesh forms tiles (structured meshes); otherwise the dense kernel runs.
        // Split-BF16 runs folded tiles on the tensor cores (tcgen05) where the mesh forms
        // them (it has no other kernel); the FP32 form folds advection on triangles at
        // p = 5 onto the FP64 DMMA tiles (FP32 stage vectors).  The FP32 form of the wave stays matrix-free: on the served request mix
        // its dense kernel measured 2-5x the DoF-updates/s of the TF32 tiles (triangles
        // at p = 1: 8.1e9 against 2.0e9; tetrahedra at p = 2: 5.2e9 against 3.5e9).
        const bool fold_tri = op.physics == HGG_PHYSICS_ADVECTION && op.shape == HGG_SHAPE_TRIANGLE &&
                              (op.nB >= 21 || (op.nB >= 15 && !h->mixed));
        const bool fold_tc = h->precision == HGG_PRECISION_BF16X3;
        if (fold_tri || fold_tc) {
            LinearSystem sys;
            bool assembled = true;
            try {
                sys = assemble_linear(*desc);
            } catch (const std::exception &) {
                assembled = false;
            }
            if (assembled) {
                h->lin_min_rows = 1;
                if ((rc = attach_linear(h, sys, fold_tri ? 1 : 2))) return rc;
                if (h->linear) return 0;
            }
            if (h->precision == HGG_PRECISION_BF16X3)
                return fail(h, HGG_ERR_UNSUPPORTED,
                            "split-BF16 runs on tiles of elements with identical matrices: this mesh forms none");
        }
        // the dense kernel reads its operators transposed ([..][j][i]): coalesced across rows i
        auto transposed = [&](const std::vector<double> &m) {
            std::vector<double> t(m.size());
            const size_t nb = (size_t)op.nB, blocks = nb ? m.size() / (nb * nb) : 0;
            for (size_t q = 0; q < blocks; ++q)
                for (size_t i = 0; i < nb; ++i)
                    for (size_t j = 0; j < nb; ++j) t[(q * nb + j) * nb + i] = m[(q * nb + i) * nb + j];
            return t;
        };
        if (h->mixed) {
            auto to_float = [](const std::vector<double> &m) { return std::vector<float>(m.begin(), m.end()); };
            if ((rc = upload(h, to_float(transposed(op.vol)), &h->d_vol_f)) ||
                (rc = upload(h, to_float(transposed(op.pairs)), &h->d_pairs_f)))
                return rc;
        }
        // tiles of the grouped kernel (the wave): elements ordered by their operator
        // signature (pair operators of every face), group_tile_elems(nB) per tile within a
        // group; used when the tiles are at least half full on average
        if (group_rows(op.dim, op.physics != HGG_PHYSICS_ADVECTION, op.nB) > 0) {
            const int TE = group_tile_elems(op.nB);
            const int nf = op.nfl;
            auto sig_less = [&](int64_t x, int64_t y) {
                for (int f = 0; f < nf; ++f) {
                    const size_t a = (size_t)x * nf + f, b = (size_t)y * nf + f;
                    if (op.self_pair[a] != op.self_pair[b]) return op.self_pair[a] < op.self_pair[b];
                    if (op.nbr_pair[a] != op.nbr_pair[b]) return op.nbr_pair[a] < op.nbr_pair[b];
                    if (op.mode[a] != op.mode[b]) return op.mode[a] < op.mode[b];
                }
                return false;
            };
            std::vector<int64_t> order(op.nE);
            for (int64_t e = 0; e < op.nE; ++e) order[e] = e;
            std::stable_sort(order.begin(), order.end(), sig_less);
            std::vector<int32_t> tiles;
            int fill = TE;
            for (size_t i = 0; i < order.size(); ++i) {
                const bool same = i > 0 && !sig_less(order[i - 1], order[i]) && !sig_less(order[i], order[i - 1]);
                if (!same || fill == TE) {
                    tiles.insert(tiles.end(), TE, -1);
                    fill = 0;
                }
                tiles[tiles.size() - TE + fill++] = (int32_t)order[i];
            }
            const int64_t n_tiles = (int64_t)(tiles.size() / TE);
            // run the tiles in the order of their first element, not group by group:
            // the neighbours a tile gathers then belong to tiles of the other groups
            // that run at about the same time, while they are still in L2
            std::vector<int64_t> torder(n_tiles);
            for (int64_t t = 0; t < n_tiles; ++t) torder[t] = t;
            std::stable_sort(torder.begin(), torder.end(), [&](int64_t x, int64_t y) {
                return tiles[x * TE] < tiles[y * TE];
            });
            std::vector<int32_t> sorted(tiles.size());
            for (int64_t t = 0; t < n_tiles; ++t)
                std::copy(tiles.begin() + torder[t] * TE, tiles.begin() + (torder[t] + 1) * TE,
                          sorted.begin() + t * TE);
            tiles.swap(sorted);
            if (n_tiles * TE <= 2 * op.nE) {
                if ((rc = upload(h, tiles, &h->d_group_tiles))) return rc;
                h->group_tiles = n_tiles;
                for (int i = 0; i < 2; ++i)
                    if ((rc = alloc(h, sizeof(double) * h->N_alloc, (void **)&h->d_win[i]))) return rc;
            }
        }
        if ((rc = upload(h, transposed(op.vol), &h->d_vol)) || (rc = upload(h, transposed(op.pairs), &h->d_pairs)) ||
            (rc = upload(h, op.nbr, &h->d_nbr)) || (rc = upload(h, op.self_pair, &h->d_self)) ||
            (rc = upload(h, op.nbr_pair, &h->d_nbrp)) || (rc = upload(h, op.mode, &h->d_mode)) ||
            (rc = upload(h, op.elem_geo, &h->d_elem_geo)) || (rc = upload(h, op.face_geo, &h->d_face_geo)))
            return rc;
    }
    HGG_CUDA(h, cudaStreamSynchronize(h->stream));
    return 0;
}

// Folds the stored matrices (fold_linear) and uploads them: the handle's
// stages then run the stored-matrix kernel.  With tiles_only, nothing is
// attached (and 0 returned) unless the grouped tensor-core kernel will run.
int attach_linear(hgg_handle *h, const LinearSystem &sys, int tiles_only) {
    LinearOperators lo;
    try {
        lo = fold_linear(sys);
    } catch (const std::exception &ex) {
        return fail(h, HGG_ERR_INVALID, ex.what());
    }
    const int R = lo.R;
    const size_t RR = (size_t)R * R;
    int rc;
    // Tiles of the grouped kernel: elements ordered by their matrix tuple (self,
    // slot 1, ..., slot S), cut into tiles of kLinTileN within each group.  Used
    // when the tiles are at least half full on average (few distinct tuples, as
    // on structured meshes) and an element has at least kLinTileMinRows rows
    // (below that the padding of the 8-row fragments and the per-chunk
    // synchronisation cost more than the row kernel: measured on quadrilaterals
    // at p = 2, 9 rows, 0.82 ms per RK4 step against 0.46 ms on 512^2 cells;
    // on 256^2 triangles the tiles won from 15 rows: 0.39 against 0.46 ms).
    // tiles of `tile_n` elements with identical matrices, in the order of their first element
    auto make_tiles = [&](int tile_n, std::vector<int32_t> &tel, std::vector<int32_t> &tmat) -> int64_t {
        const int S = lo.slots, W = S + 1;
        auto tuple = [&](int64_t e, int k) { return k == 0 ? lo.self_mat[e] : lo.nbr_mat[(size_t)e * S + k - 1]; };
        std::vector<int64_t> order(lo.E);
        for (int64_t e = 0; e < lo.E; ++e) order[e] = e;
        std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
            for (int k = 0; k < W; ++k)
                if (tuple(x, k) != tuple(y, k)) return tuple(x, k) < tuple(y, k);
            return false;
        });
        int fill = tile_n;
        for (size_t i = 0; i < order.size(); ++i) {
            const int64_t e = order[i];
            const bool same = i > 0 && [&] {
                for (int k = 0; k < W; ++k)
                    if (tuple(e, k) != tuple(order[i - 1], k)) return false;
                return true;
            }();
            if (!same || fill == tile_n) {
                tel.insert(tel.end(), tile_n, -1);
                for (int k = 0; k < W; ++k) tmat.push_back(tuple(e, k));
                fill = 0;
            }
            tel[tel.size() - tile_n + fill++] = (int32_t)e;
        }
        const int64_t n_tiles = (int64_t)(tel.size() / tile_n);
        // tiles in the order of their first element (see the grouped dense kernel)
        std::vector<int64_t> torder(n_tiles);
        for (int64_t t2 = 0; t2 < n_tiles; ++t2) torder[t2] = t2;
        std::stable_sort(torder.begin(), torder.end(),
                         [&](int64_t x, int64_t y) { return tel[x * tile_n] < tel[y * tile_n]; });
        std::vector<int32_t> el2(tel.size()), mat2(tmat.size());
        for (int64_t t2 = 0; t2 < n_tiles; ++t2) {
            std::copy(tel.begin() + torder[t2] * tile_n, tel.begin() + (torder[t2] + 1) * tile_n,
                      el2.begin() + t2 * tile_n);
            std::copy(tmat.begin() + torder[t2] * W, tmat.begin() + (torder[t2] + 1) * W, mat2.begin() + t2 * W);
        }
        tel.swap(el2);
        tmat.swap(mat2);
        return n_tiles;
    };
    std::vector<int32_t> tel, tmat;
    const int64_t n_tiles = make_tiles(kLinTileN, tel, tmat);
    const bool use_tiles = n_tiles * kLinTileN <= 2 * lo.E && R >= h->lin_min_rows;
    // the mixed forms run the tiles on the tensor cores (tcgen05), 128 elements per tile,
    // where the operands fit the shared memory of one CTA
    std::vector<int32_t> utel, utmat;
    int64_t u_tiles = 0;
    const int ukind = h->precision == HGG_PRECISION_BF16X3 ? kUmmaBF16 : kUmmaTF32;
    const UmmaShape ush = umma_shape(R, lo.slots, ukind);
    // (plane rows of at most 512 bytes: a thread's copies of one item stay in registers)
    // (the FP32 form of a folded matrix-free operator keeps the FP64 DMMA tiles: on the
    // batched triangles at p = 5 they took 1.06 ms per step against 1.34 ms on TF32 x 3)
    const bool umma_wanted = h->precision == HGG_PRECISION_BF16X3 || (h->mixed && tiles_only != 1);
    if (umma_wanted && umma_smem(ush) <= 227 * 1024 && ush.NP <= 256 && ush.KP * ush.es <= 512) {
        u_tiles = make_tiles(kUmmaTileN, utel, utmat);
        if (!(u_tiles * kUmmaTileN <= 2 * lo.E)) u_tiles = 0;
    }
    if (h->precision == HGG_PRECISION_BF16X3 && u_tiles == 0) {
        if (tiles_only) return 0;
        return fail(h, HGG_ERR_UNSUPPORTED,
                    "split-BF16 runs on tiles of elements with identical matrices: this mesh forms none");
    }
    if (tiles_only == 1 && !use_tiles && u_tiles == 0) return 0;
    if (tiles_only == 2 && u_tiles == 0) return 0;
    std::vector<double> t(lo.table.size());
    for (int m = 0; m < lo.n_mats(); ++m)
        for (int i = 0; i < R; ++i)
            for (int j = 0; j < R; ++j) t[m * RR + (size_t)j * R + i] = lo.table[m * RR + (size_t)i * R + j];
    if ((rc = upload(h, t, &h->d_lin_table)) || (rc = upload(h, lo.self_mat, &h->d_lin_self))) return rc;
    if (lo.slots > 0 && ((rc = upload(h, lo.nbr, &h->d_lin_nbr)) || (rc = upload(h, lo.nbr_mat, &h->d_lin_mat))))
        return rc;
    if (h->mixed && R <= kMixedFp32MaxBasis) {
        std::vector<float> tf(t.begin(), t.end());
        if ((rc = upload(h, tf, &h->d_lin_table_f))) return rc;
    }
    if (use_tiles) {
        std::vector<double> rm(lo.table);
        if ((rc = upload(h, rm, &h->d_lin_table_rm)) || (rc = upload(h, tel, &h->d_lin_tile_elems)) ||
            (rc = upload(h, tmat, &h->d_lin_tile_mats)))
            return rc;
        h->lin_tiles = n_tiles;
    }
    if (u_tiles > 0) {
        // operand images of every distinct matrix: hi part then lo part, each NP x KP in the
        // swizzled layout the kernel's shared memory holds (umma_offset)
        const size_t part = ush.b_bytes, mats = (size_t)lo.n_mats();
        std::vector<unsigned char> img(mats * 2 * part, 0);
        for (size_t m = 0; m < mats; ++m)
            for (int n = 0; n < R; ++n)
                for (int k = 0; k < R; ++k) {
                    const double x = lo.table[m * RR + (size_t)n * R + k];
                    unsigned char *dst = img.data() + m * 2 * part + umma_offset(n, k, ush.NP, ush.es);
                    if (ukind == kUmmaTF32) {
                        const uint32_t hb = float_bits((float)x) & 0xFFFFE000u;
                        const uint32_t lb = float_bits((float)(x - (double)bits_float(hb)));
                        std::memcpy(dst, &hb, 4);
                        std::memcpy(dst + part, &lb, 4);
                    } else {
                        const uint16_t hb = bf16_rn((float)x);
                        const uint16_t lb = bf16_rn((float)(x - (double)bits_float((uint32_t)hb << 16)));
                        std::memcpy(dst, &hb, 2);
                        std::memcpy(dst + part, &lb, 2);
                    }
                }
        if ((rc = upload(h, img, &h->d_umma_img)) || (rc = upload(h, utel, &h->d_umma_tile_elems)) ||
            (rc = upload(h, utmat, &h->d_umma_tile_mats)))
            return rc;
        if (!h->d_lin_nbr && lo.slots > 0 && (rc = upload(h, lo.nbr, &h->d_lin_nbr))) return rc;
        if ((rc = alloc(h, 2 * (size_t)lo.E * ush.KP * ush.es, (void **)&h->d_umma_planes))) return rc;
        HGG_CUDA(h, cudaMemsetAsync(h->d_umma_planes, 0, 2 * (size_t)lo.E * ush.KP * ush.es, h->stream));
        h->umma_tiles = u_tiles;
    }
    h->lin_R = R;
    h->lin_slots = lo.slots;
    h->lin_mats = lo.n_mats();
    h->linear = true;
    HGG_CUDA(h, cudaStreamSynchronize(h->stream));
    return 0;
}

void destroy_handle(hgg_handle *h) {
    if (!h) return;
    release_graphs(h);
    destroy_sources(h);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->own_stream) cudaStreamSynchronize(h->own_stream);
    for (auto &b : h->bufs) cudaFreeAsync(b.p, h->stream);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    delete h;
}

}  // namespace hgg

extern "C" {

int hgg_create(const hgg_problem_desc *desc, hgg_handle **out) {
    if (!desc || !out) return fail(nullptr, HGG_ERR_INVALID, "null argument");
    *out = nullptr;
    hgg_handle *h = new (std::nothrow) hgg_handle();
    if (!h) return fail(nullptr, HGG_ERR_NOMEM, "host allocation failed");
    int rc = create_from_desc(desc, h);
    if (rc) {
        g_create_error = h->err;
        destroy_handle(h);
        return rc;
    }
    *out = h;
    return 0;
}

int hgg_destroy(hgg_handle *h) {
    destroy_handle(h);
    return 0;
}

const char *hgg_last_error(const hgg_handle *h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int hgg_set_state(hgg_handle *h, int32_t vec, const double *host) {
    if (!h || !host) return fail(h, HGG_ERR_INVALID, "null argument");
    void *d = vector_ptr(h, vec);
    if (!d) return fail(h, HGG_ERR_INVALID, "vector id out of range");
    const bool f = vector_is_float(h, vec);
    const unsigned grid = 4 * h->num_sms;
    if (h->tensor_layout || f) {
        HGG_CUDA(h, cudaMemcpyAsync(h->d_scratch, host, sizeof(double) * h->N, cudaMemcpyHostToDevice, h->stream));
        if (h->tensor_layout && f)
            to_tensor_order<float><<<grid, 256, 0, h->stream>>>(h->d_scratch, static_cast<float *>(d), h->d_tpos,
                                                                 h->d_tsign, h->op.nB, h->N, h->tiled);
        else if (h->tensor_layout)
            to_tensor_order<double><<<grid, 256, 0, h->stream>>>(h->d_scratch, static_cast<double *>(d), h->d_tpos,
                                                                  h->d_tsign, h->op.nB, h->N, h->tiled);
        else
            convert_vector<<<grid, 256, 0, h->stream>>>(h->d_scratch, static_cast<float *>(d), h->N);
        h->launches++;
        HGG_CUDA(h, cudaGetLastError());
    } else {
        HGG_CUDA(h, cudaMemcpyAsync(d, host, sizeof(double) * h->N, cudaMemcpyHostToDevice, h->stream));
    }
    HGG_CUDA(h, cudaStreamSynchronize(h->stream));
    return 0;
}

int hgg_get_state(hgg_handle *h, int32_t vec, double *host) {
    if (!h || !host) return fail(h, HGG_ERR_INVALID, "null argument");
    void *d = vector_ptr(h, vec);
    if (!d) return fail(h, HGG_ERR_INVALID, "vector id out of range");
    const bool f = vector_is_float(h, vec);
    const unsigned grid = 4 * h->num_sms;
    const double *src = static_cast<const double *>(d);
    if (h->tensor_layout || f) {
        if (h->tensor_layout && f)
            from_tensor_order<float><<<grid, 256, 0, h->stream>>>(static_cast<const float *>(d), h->d_scratch,
                                                                   h->d_tpos, h->d_tsign, h->op.nB, h->N, h->tiled);
        else if (h->tensor_layout)
            from_tensor_order<double><<<grid, 256, 0, h->stream>>>(static_cast<const double *>(d), h->d_scratch,
                                                                    h->d_tpos, h->d_tsign, h->op.nB, h->N, h->tiled);
        else
            convert_vector<<<grid, 256, 0, h->stream>>>(static_cast<const float *>(d), h->d_scratch, h->N);
        h->launches++;
        HGG_CUDA(h, cudaGetLastError());
        src = h->d_scratch;
    }
    HGG_CUDA(h, cudaMemcpyAsync(host, src, sizeof(double) * h->N, cudaMemcpyDeviceToHost, h->stream));
    HGG_CUDA(h, cudaStreamSynchronize(h->stream));
    return 0;
}

int hgg_step(hgg_handle *h, double *time, double dt, int32_t nsteps) {
    if (!h || nsteps < 0) return fail(h, HGG_ERR_INVALID, "bad argument");
    if (nsteps == 0) return 0;
    if (!(dt == h->graph_dt && h->store_last == h->graph_store_last && h->graph[0] && h->graph[1])) {
        release_graphs(h);
        for (int from = 0; from < 2; ++from) {
            cudaGraph_t g = nullptr;
            HGG_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
            int64_t before = h->launches;
            int rc = enqueue_step(h, from, dt);
            cudaError_t ce = cudaStreamEndCapture(h->stream, &g);
            h->graph_launches = h->launches - before;  // kernels of one captured step
            h->launches = before;                      // capture does not launch
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (ce != cudaSuccess) return fail(h, HGG_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
            cudaError_t ie = cudaGraphInstantiate(&h->graph[from], g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) return fail(h, HGG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
        }
        h->graph_dt = dt;
        h->graph_store_last = h->store_last;
    }
    if (h->src && !time) return fail(h, HGG_ERR_INVALID, "source terms need the time: pass a time");
    for (int s = 0; s < nsteps; ++s) {
        if (h->src) {  // the source values of this step's stage times
            int rc = fill_sources(h, h->cur, *time, dt);
            if (rc) return rc;
        }
        HGG_CUDA(h, cudaGraphLaunch(h->graph[h->cur], h->stream));
        h->launches += h->graph_launches;
        h->cur = 1 - h->cur;
        if (time) *time += dt;
    }
    return 0;
}

int hgg_time_derivative(hgg_handle *h, int32_t in_vec, int32_t out_vec) {
    return time_derivative_impl(h, in_vec, out_vec, nullptr);
}

}  // extern "C"

int hgg::time_derivative_impl(hgg_handle *h, int32_t in_vec, int32_t out_vec, const double *time) {
    if (!h) return fail(h, HGG_ERR_INVALID, "null handle");
    void *in = vector_ptr(h, in_vec), *outp = vector_ptr(h, out_vec);
    if (!in || !outp || in == outp) return fail(h, HGG_ERR_INVALID, "bad vector ids");
    if (h->src && !time)
        return fail(h, HGG_ERR_INVALID, "the handle has source terms: use hgg_time_derivative_at with a time");
    int rc;
    if (h->src && (rc = fill_source_values(h, 2, time, 1))) return rc;
    if (h->mixed) {
        // FP32-mixed form: FP64 input (the solution), FP32 stage vector output
        if (vector_is_float(h, in_vec) || !vector_is_float(h, out_vec))
            return fail(h, HGG_ERR_INVALID, "the FP32-mixed form maps the solution (vector 0) to a stage vector");
        StageIOT<float> io{};
        io.u = static_cast<const double *>(in);
        io.kout = static_cast<float *>(outp);
        io.n_elements = h->op.nE;
        io.status = h->d_status;
        rc = launch_stage(h, io);
        if (!rc && h->src) rc = enqueue_source(h, 2, 0, io.kout, nullptr, 0.0);
    } else {
        StageIO io{};
        io.u = static_cast<const double *>(in);
        io.kout = static_cast<double *>(outp);
        io.n_elements = h->op.nE;
        io.status = h->d_status;
        rc = launch_stage(h, io);
        if (!rc && h->src) rc = enqueue_source(h, 2, 0, io.kout, nullptr, 0.0);
    }
    if (rc) return rc;
    return check_status(h);
}

extern "C" {

int hgg_synchronize(hgg_handle *h) {
    if (!h) return fail(h, HGG_ERR_INVALID, "null handle");
    HGG_CUDA(h, cudaStreamSynchronize(h->stream));
    return check_status(h);
}

int64_t hgg_vector_length(const hgg_handle *h) { return h ? h->N : -1; }

int hgg_kernel_kind(const hgg_handle *h) {
    return h ? (h->umma_tiles > 0 ? 3 : (h->linear ? 2 : (h->op.tensor ? 1 : 0))) : -1;
}

int hgg_set_store_last_stage(hgg_handle *h, int32_t enable) {
    if (!h) return fail(h, HGG_ERR_INVALID, "null handle");
    h->store_last = enable != 0;
    return 0;
}

int hgg_set_stream(hgg_handle *h, void *stream) {
    if (!h) return fail(h, HGG_ERR_INVALID, "null handle");
    HGG_CUDA(h, cudaStreamSynchronize(h->stream));
    cudaStream_t s = stream ? (cudaStream_t)stream : h->own_stream;
    if (s != h->stream) {
        release_graphs(h);  // captured on the previous stream
        h->stream = s;
    }
    return 0;
}

int64_t hgg_launch_count(const hgg_handle *h) { return h ? h->launches : -1; }

int hgg_set_kernel_variant(hgg_handle *h, int32_t variant) {
    if (!h || variant < 0 || variant > 2) return fail(h, HGG_ERR_INVALID, "variant must be 0..2");
    if (variant != 0 && h->slice_ok)
        return fail(h, HGG_ERR_UNSUPPORTED, "hexahedra of order 3 have one kernel organisation (the slice kernel)");
    if (variant != h->variant) {
        release_graphs(h);
        h->variant = variant;
    }
    return 0;
}

int hgg_test_arm_without_copy(hgg_handle *h, int32_t polls) {
    if (!h || polls < 1) return fail(h, HGG_ERR_INVALID, "polls must be positive");
    if (h->linear || h->slice_ok || !h->op.tensor || h->variant != 2)
        return fail(h, HGG_ERR_UNSUPPORTED, "only the pipelined kernel (kernel variant 2) waits on mbarriers");
    h->test_arm_polls = (uint32_t)polls;
    return 0;
}

// ---- right-hand side without allocation ---------------------------------------
// The sum-factorised handles keep their vectors in tensor order on the device,
// so a right-hand side of caller-owned vectors in hpGEM order needs two
// vectors of scratch (the input in device order, the output in device order).
// This entry point takes them from one file-scope device array instead of the
// allocator.  Every process that loads the library holds the array on every
// GPU it uses until exit; all calls on a device share it.

namespace {
constexpr int64_t kStaticScratchDoubles = int64_t(1) << 22;  // 32 MiB
constexpr int kMaxStaticDevices = 64;
static __device__ __align__(256) double g_static_scratch[kStaticScratchDoubles];
std::mutex g_static_mutex;
double *g_static_ptr[kMaxStaticDevices] = {};
}  // namespace

int hgg_time_derivative_static(hgg_handle *h, const double *u, double *k) {
    if (!h) return fail(h, HGG_ERR_INVALID, "null handle");
    if (!u || !k || u == k) return fail(h, HGG_ERR_INVALID, "u and k must be distinct device vectors");
    int dev = -1;
    HGG_CUDA(h, cudaGetDevice(&dev));
    if (dev != h->device) return fail(h, HGG_ERR_INVALID, "call with the handle's device current");
    if (h->mixed) return fail(h, HGG_ERR_UNSUPPORTED, "the FP32-mixed form has no static-scratch right-hand side");
    if (h->src) return fail(h, HGG_ERR_UNSUPPORTED, "source terms need a time: use hgg_time_derivative_at");
    StageIO io{};
    io.n_elements = h->op.nE;
    io.status = h->d_status;
    if (!h->tensor_layout) {  // the dense kernels read and write hpGEM order: no scratch
        io.u = u;
        io.kout = k;
        int rc = launch_stage(h, io);
        if (rc) return rc;
        return check_status(h);
    }
    if (2 * h->N_alloc > kStaticScratchDoubles)
        return fail(h, HGG_ERR_UNSUPPORTED,
                    "problem needs " + std::to_string(2 * h->N_alloc) + " doubles of scratch; the static scratch holds " +
                        std::to_string(kStaticScratchDoubles) + " (" + std::to_string(kStaticScratchDoubles / 2) +
                        " per vector, padded to whole tiles)");
    double *base = nullptr;
    {
        // first call on a device: look the array up, with that device current
        std::lock_guard<std::mutex> lock(g_static_mutex);
        if (dev < 0 || dev >= kMaxStaticDevices) return fail(h, HGG_ERR_UNSUPPORTED, "device ordinal too large");
        if (!g_static_ptr[dev]) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
            if (e != cudaSuccess)
                return fail(h, HGG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_static_ptr[dev] = static_cast<double *>(p);
        }
        base = g_static_ptr[dev];
    }
    double *su = base, *sk = base + h->N_alloc;
    // The stage kernels read the padding elements of the last tile (they mask
    // their results); clear them, wherever the layout puts them (tiled layout:
    // interleaved with the tile's real elements), so that they read zeros
    // rather than the previous call's values.
    const int nbv = h->op.V * h->op.nB;
    const int64_t n_pad = h->N_alloc / nbv;
    if (n_pad > h->op.nE) {
        zero_padding<<<(unsigned)(((n_pad - h->op.nE) * nbv + 255) / 256), 256, 0, h->stream>>>(
            su, nbv, h->op.nE, n_pad, h->tiled);
        h->launches++;
    }
    to_tensor_order<double><<<4 * h->num_sms, 256, 0, h->stream>>>(u, su, h->d_tpos, h->d_tsign, h->op.nB, h->N,
                                                                    h->tiled);
    h->launches++;
    HGG_CUDA(h, cudaGetLastError());
    io.u = su;
    io.kout = sk;
    int rc = launch_stage(h, io);
    if (rc) return rc;
    from_tensor_order<double><<<4 * h->num_sms, 256, 0, h->stream>>>(sk, k, h->d_tpos, h->d_tsign, h->op.nB, h->N,
                                                                      h->tiled);
    h->launches++;
    HGG_CUDA(h, cudaGetLastError());
    return check_status(h);
}

}  // extern "C"

// ---- adaptive time step -------------------------------------------------------
// computeErrorAndNormOfUpdate (HpgemAPISimplified_Impl.h:719-749) per element:
// the deviation sum_i (k_i dt) err_i of the element's coefficients, its squared
// Euclidean norm, and the Euclidean norm of the element's (updated) solution.
// The layout is the device's (tensor order, tiled or not): a permutation with
// sign flips inside each element, which leaves both norms unchanged.
template <typename KT>
__global__ void element_error_norm(const double *u, ErrStages<KT> ks, int nb, int64_t n_elements, bool tiled,
                                   double *err2, double *norm) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n_elements) return;
    double s2 = 0.0, n2 = 0.0;
    for (int pos = 0; pos < nb; ++pos) {
        const int64_t idx = device_index(e, pos, nb, tiled);
        double dev = 0.0;
        for (int i = 0; i < ks.n; ++i) dev += ((double)ks.k[i][idx] * ks.dt) * ks.err[i];
        s2 += dev * dev;
        n2 += u[idx] * u[idx];
    }
    err2[e] = s2;
    norm[e] = sqrt(n2);
}

// deterministic sums of two arrays: block partials in a fixed order, then the partials
constexpr int kSumThreads = 256;
__global__ void sum_pairs(const double *a, const double *b, int64_t n, double *pa, double *pb) {
    __shared__ double sa[kSumThreads], sb[kSumThreads];
    double x = 0.0, y = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)kSumThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kSumThreads) {
        x += a[i];
        y += b[i];
    }
    sa[threadIdx.x] = x;
    sb[threadIdx.x] = y;
    __syncthreads();
    for (int w = kSumThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sa[threadIdx.x] += sa[threadIdx.x + w];
            sb[threadIdx.x] += sb[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        pa[blockIdx.x] = sa[0];
        pb[blockIdx.x] = sb[0];
    }
}

// undo a rejected step: u -= dt b_j k_j for j = 0..S-1, one update after the other as
// the reference's scaleAndAddVector calls do (HpgemAPISimplified_Impl.h:843-848)
template <typename KT>
__global__ void rewind_update(double *u, ErrStages<KT> ks, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double v = u[i];
        for (int j = 0; j < ks.n; ++j) v += (-ks.dt * ks.err[j]) * (double)ks.k[j][i];
        u[i] = v;
    }
}

namespace {

template <typename KT>
ErrStages<KT> err_stages(const hgg_handle *h, double dt, const std::vector<double> &coef) {
    ErrStages<KT> ks{};
    ks.n = h->S;
    ks.dt = dt;
    for (int i = 0; i < h->S; ++i) {
        ks.k[i] = static_cast<const KT *>(h->k[i]);
        ks.err[i] = coef[i];
    }
    return ks;
}

// error and solution norm of the step just taken (sol[cur] is the updated solution)
int error_and_norm(hgg_handle *h, double dt, double *error, double *norm) {
    const int64_t nE = h->op.nE;
    const int nb = h->op.V * h->op.nB;
    double *err2 = h->d_reduce, *nrm = h->d_reduce + nE;
    const unsigned eb = (unsigned)((nE + 255) / 256);
    if (h->mixed)
        element_error_norm<float><<<eb, 256, 0, h->stream>>>(h->sol[h->cur], err_stages<float>(h, dt, h->rk_err), nb,
                                                             nE, h->tiled, err2, nrm);
    else
        element_error_norm<double><<<eb, 256, 0, h->stream>>>(h->sol[h->cur], err_stages<double>(h, dt, h->rk_err),
                                                              nb, nE, h->tiled, err2, nrm);
    const int parts = 256;
    double *pa = h->d_reduce + 2 * nE, *pb = pa + parts;
    sum_pairs<<<parts, kSumThreads, 0, h->stream>>>(err2, nrm, nE, pa, pb);
    sum_pairs<<<1, kSumThreads, 0, h->stream>>>(pa, pb, parts, pa + 2 * parts, pb + 2 * parts);
    h->launches += 3;
    HGG_CUDA(h, cudaGetLastError());
    double out[2];
    HGG_CUDA(h, cudaMemcpyAsync(&out[0], pa + 2 * parts, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    HGG_CUDA(h, cudaMemcpyAsync(&out[1], pb + 2 * parts, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    HGG_CUDA(h, cudaStreamSynchronize(h->stream));
    *error = std::sqrt(out[0]);
    *norm = out[1];
    return 0;
}

}  // namespace

extern "C" {

int hgg_set_error_estimate(hgg_handle *h, const double *error_coefficients, int32_t order) {
    if (!h || !error_coefficients || order < 1) return fail(h, HGG_ERR_INVALID, "error coefficients and order >= 1");
    h->rk_err.assign(error_coefficients, error_coefficients + h->S);
    h->rk_order = order;
    return 0;
}

int hgg_step_adaptive(hgg_handle *h, double *time, double max_relative_error, double dt_max, double *dt_estimate,
                      double *dt_taken, int32_t *rejections) {
    if (!h || !time || !dt_estimate) return fail(h, HGG_ERR_INVALID, "null argument");
    if (h->rk_err.empty()) return fail(h, HGG_ERR_INVALID, "the tableau has no error estimate (embedded pair)");
    if (!(max_relative_error > 0.0) || !(dt_max > 0.0) || !(*dt_estimate > 0.0))
        return fail(h, HGG_ERR_INVALID, "maximum relative error, dt_max and the dt estimate must be positive");
    if (!h->d_reduce) {  // per-element error and norm, then the partial sums
        int rc = alloc(h, sizeof(double) * (size_t)(2 * h->op.nE + 1024), (void **)&h->d_reduce);
        if (rc) return rc;
    }
    // the error estimate needs the last stage vector
    const bool keep = h->store_last;
    h->store_last = true;
    double dt = std::min(*dt_estimate, dt_max);
    double error = std::numeric_limits<double>::infinity(), norm = 0.0;
    int rej = 0;
    int rc = 0;
    while (max_relative_error * norm < error || std::isinf(error)) {
        const int from = h->cur;
        if (h->src) rc = fill_sources(h, from, *time, dt);
        if (!rc) rc = enqueue_step(h, from, dt);
        if (rc) break;
        h->cur = 1 - from;
        rc = error_and_norm(h, dt, &error, &norm);
        if (rc) break;
        if (max_relative_error * norm < error || std::isinf(error)) {
            const unsigned grid = 4 * h->num_sms;
            if (h->mixed)
                rewind_update<float><<<grid, 256, 0, h->stream>>>(h->sol[h->cur], err_stages<float>(h, dt, h->rk_b),
                                                                  h->N_alloc);
            else
                rewind_update<double><<<grid, 256, 0, h->stream>>>(h->sol[h->cur], err_stages<double>(h, dt, h->rk_b),
                                                                   h->N_alloc);
            h->launches++;
            dt = 0.8 * dt * std::pow(max_relative_error / error * norm, 1. / h->rk_order);
            ++rej;
            if (rej > 1000) {
                rc = fail(h, HGG_ERR_DEVICE, "adaptive step: no accepted step after 1000 tries");
                break;
            }
        }
    }
    h->store_last = keep;
    if (rc) return rc;
    *dt_estimate = 0.9 * dt * std::pow(max_relative_error / error * norm, 1. / h->rk_order);
    *time += dt;
    if (dt_taken) *dt_taken = dt;
    if (rejections) *rejections = rej;
    return check_status(h);
}

}  // extern "C"

extern "C" {

// ---- stand-alone set-up ------------------------------------------------------

namespace {
void fill_descriptor(const StructuredProblem &P, int32_t precision, hgg_problem_desc &d) {
    d = hgg_problem_desc{};
    d.dim = P.mesh.dim;
    d.shape = P.mesh.shape;
    d.order = P.order;
    d.n_vars = P.n_vars;
    d.physics = P.physics;
    d.precision = precision;
    for (int i = 0; i < 3; ++i) d.advection[i] = P.advection[i];
    d.c_inv = P.c_inv;
    d.n_elements = P.mesh.n_elements;
    d.n_basis = P.n_basis;
    d.n_quad = P.rule.size();
    d.quad_weights = P.rule.weights.data();
    d.basis_values = P.basis_values.data();
    d.basis_grads = P.basis_grads.data();
    d.n_face_quad = P.face_rule.size();
    d.face_weights = P.face_rule.weights.data();
    d.n_face_tabs = P.n_face_tabs;
    d.face_tabs = P.face_tabs.data();
    d.jacobians = P.jacobians.data();
    d.n_faces = P.mesh.n_faces();
    d.face_elements = P.mesh.face_elements.data();
    d.face_local = P.mesh.face_local.data();
    d.face_tab_index = P.face_tab_index.data();
    d.face_normals = P.normals.data();
    d.n_stages = P.n_stages;
    d.rk_a = P.rk_a.data();
    d.rk_b = P.rk_b.data();
    d.rk_c = P.rk_c.data();
}
}  // namespace

int hgg_structured_descriptor(const char *description, int32_t order, int32_t physics, const double *params,
                              const char *tableau, int32_t precision, hgg_problem_desc *out, void **owner) {
    if (!description || !tableau || !out || !owner) return fail(nullptr, HGG_ERR_INVALID, "null argument");
    *owner = nullptr;
    StructuredProblem *sp = new (std::nothrow) StructuredProblem();
    if (!sp) return fail(nullptr, HGG_ERR_NOMEM, "host allocation failed");
    try {
        *sp = build_structured(description, order, physics, params, tableau);
    } catch (const std::exception &ex) {
        delete sp;
        return fail(nullptr, HGG_ERR_INVALID, ex.what());
    }
    fill_descriptor(*sp, precision, *out);
    *owner = sp;
    return 0;
}

void hgg_free_descriptor(void *owner) { delete static_cast<StructuredProblem *>(owner); }

}  // extern "C"

namespace {
// the problem of a mesh file (text read here, parsed by read_mesh2)
int mesh_file_problem(const char *path, int32_t order, int32_t physics, const double *params, const char *tableau,
                      StructuredProblem &P, bool boundary_faces = false) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return fail(nullptr, HGG_ERR_INVALID, std::string("cannot open mesh file ") + path);
    std::stringstream text;
    text << in.rdbuf();
    try {
        P = build_problem(read_mesh2(text.str()), order, physics, params, tableau, boundary_faces);
    } catch (const std::exception &ex) {
        return fail(nullptr, HGG_ERR_INVALID, ex.what());
    }
    return 0;
}
}  // namespace

extern "C" {

int hgg_mesh_file_descriptor(const char *path, int32_t order, int32_t physics, const double *params,
                             const char *tableau, int32_t precision, hgg_problem_desc *out, void **owner) {
    if (!path || !tableau || !out || !owner) return fail(nullptr, HGG_ERR_INVALID, "null argument");
    *owner = nullptr;
    std::unique_ptr<StructuredProblem> sp(new (std::nothrow) StructuredProblem());
    if (!sp) return fail(nullptr, HGG_ERR_NOMEM, "host allocation failed");
    int rc = mesh_file_problem(path, order, physics, params, tableau, *sp);
    if (rc) return rc;
    fill_descriptor(*sp, precision, *out);
    *owner = sp.release();
    return 0;
}

int hgg_create_mesh_file(const char *path, int32_t order, int32_t physics, const double *params,
                         const char *tableau, int32_t precision, hgg_handle **out) {
    if (!path || !out || !tableau) return fail(nullptr, HGG_ERR_INVALID, "null argument");
    *out = nullptr;
    std::unique_ptr<StructuredProblem> sp(new StructuredProblem());
    int rc = mesh_file_problem(path, order, physics, params, tableau, *sp);
    if (rc) return rc;
    hgg_problem_desc d;
    fill_descriptor(*sp, precision, d);
    hgg_handle *h = nullptr;
    rc = hgg_create(&d, &h);
    if (rc) return rc;
    h->sp = std::move(sp);
    butcher_error_estimate(tableau, h->rk_err, h->rk_order);
    *out = h;
    return 0;
}

int hgg_create_structured(const char *description, int32_t order, int32_t physics, const double *params,
                          const char *tableau, int32_t precision, hgg_handle **out) {
    if (!description || !out || !tableau) return fail(nullptr, HGG_ERR_INVALID, "null argument");
    *out = nullptr;
    std::unique_ptr<StructuredProblem> sp(new StructuredProblem());
    try {
        *sp = build_structured(description, order, physics, params, tableau);
    } catch (const std::exception &ex) {
        return fail(nullptr, HGG_ERR_INVALID, ex.what());
    }
    hgg_problem_desc d;
    fill_descriptor(*sp, precision, d);
    hgg_handle *h = nullptr;
    int rc = hgg_create(&d, &h);
    if (rc) return rc;
    h->sp = std::move(sp);
    butcher_error_estimate(tableau, h->rk_err, h->rk_order);
    *out = h;
    return 0;
}

}  // extern "C"

namespace {
// HpgemAPILinear's matrices of a structured mesh or a mesh file (host), with the
// problem they came from
int linear_structured_system(const char *description, int32_t order, int32_t physics, const double *params,
                             const char *tableau, StructuredProblem &P, LinearSystem &sys,
                             const char *mesh_file = nullptr) {
    if (physics != HGG_PHYSICS_ADVECTION && physics != HGG_PHYSICS_WAVE && physics != HGG_PHYSICS_WAVE_UPWIND)
        return fail(nullptr, HGG_ERR_UNSUPPORTED,
                    "the stored-matrix form has the reference's linear advection and wave (central or upwind flux)");
    if (mesh_file) {
        int rc = mesh_file_problem(mesh_file, order, physics, params, tableau, P, true);
        if (rc) return rc;
    }
    try {
        // the stored-matrix path takes meshes with boundary faces (non-periodic directions)
        if (!mesh_file) P = build_structured(description, order, physics, params, tableau, true);
        hgg_problem_desc d;
        fill_descriptor(P, HGG_PRECISION_FP64, d);
        sys = assemble_linear(d);
    } catch (const std::exception &ex) {
        return fail(nullptr, HGG_ERR_INVALID, ex.what());
    }
    return 0;
}

// arrays behind an hgg_linear_desc from hgg_linear_descriptor
struct LinearDescOwner {
    std::vector<double> mass, stiffness, faces, rk_a, rk_b, rk_c;
    std::vector<int64_t> face_elements;
};
}  // namespace

extern "C" {

int hgg_create_linear(const hgg_linear_desc *desc, hgg_handle **out) {
    if (!desc || !out) return fail(nullptr, HGG_ERR_INVALID, "null argument");
    *out = nullptr;
    LinearSystem sys;
    try {
        sys = linear_from_desc(*desc);
    } catch (const std::exception &ex) {
        return fail(nullptr, HGG_ERR_INVALID, ex.what());
    }
    hgg_handle *h = new (std::nothrow) hgg_handle();
    if (!h) return fail(nullptr, HGG_ERR_NOMEM, "host allocation failed");
    auto bail = [&](int rc) {
        g_create_error = h->err;
        destroy_handle(h);
        return rc;
    };
    int rc = set_tableau(h, desc->n_stages, desc->rk_a, desc->rk_b, desc->rk_c, desc->precision);
    if (rc) return bail(rc);
    // one "variable" of R coefficients per element: the layout is hpGEM's either way
    h->op.nE = desc->n_elements;
    h->op.V = 1;
    h->op.nB = desc->n_rows;
    h->N = h->N_alloc = desc->n_elements * desc->n_rows;
    if ((rc = init_device_vectors(h))) return bail(rc);
    if (h->mixed && (rc = alloc(h, sizeof(double) * h->N_alloc, (void **)&h->d_scratch))) return bail(rc);
    if ((rc = attach_linear(h, sys))) return bail(rc);
    *out = h;
    return 0;
}

int hgg_linear_descriptor(const char *description, int32_t order, int32_t physics, const double *params,
                          const char *tableau, int32_t precision, hgg_linear_desc *out, void **owner) {
    if (!description || !tableau || !out || !owner) return fail(nullptr, HGG_ERR_INVALID, "null argument");
    *owner = nullptr;
    StructuredProblem P;
    LinearSystem sys;
    int rc = linear_structured_system(description, order, physics, params, tableau, P, sys);
    if (rc) return rc;
    std::unique_ptr<LinearDescOwner> o(new (std::nothrow) LinearDescOwner());
    if (!o) return fail(nullptr, HGG_ERR_NOMEM, "host allocation failed");
    const size_t RR = (size_t)sys.R * sys.R;
    try {
        o->mass.resize(sys.E * RR);
        o->stiffness.resize(sys.E * RR);
        o->faces.assign(sys.F * 4 * RR, 0.0);
    } catch (const std::bad_alloc &) {
        return fail(nullptr, HGG_ERR_NOMEM, "host allocation failed");
    }
    for (int64_t e = 0; e < sys.E; ++e) {
        std::memcpy(&o->mass[e * RR], sys.pool.get(sys.mass_id[e]), RR * sizeof(double));
        std::memcpy(&o->stiffness[e * RR], sys.pool.get(sys.stiffness_id[e]), RR * sizeof(double));
    }
    for (int64_t f = 0; f < sys.F; ++f)
        for (int b = 0; b < 4; ++b)
            if (sys.face_id[4 * f + b] >= 0)
                std::memcpy(&o->faces[(4 * f + b) * RR], sys.pool.get(sys.face_id[4 * f + b]), RR * sizeof(double));
    o->face_elements = sys.face_elements;
    o->rk_a = P.rk_a;
    o->rk_b = P.rk_b;
    o->rk_c = P.rk_c;
    *out = hgg_linear_desc{};
    out->n_rows = sys.R;
    out->precision = precision;
    out->n_elements = sys.E;
    out->mass = o->mass.data();
    out->element_stiffness = o->stiffness.data();
    out->n_faces = sys.F;
    out->face_elements = o->face_elements.data();
    out->face_stiffness = o->faces.data();
    out->n_stages = P.n_stages;
    out->rk_a = o->rk_a.data();
    out->rk_b = o->rk_b.data();
    out->rk_c = o->rk_c.data();
    *owner = o.release();
    return 0;
}

void hgg_free_linear_descriptor(void *owner) { delete static_cast<LinearDescOwner *>(owner); }

}  // extern "C"

namespace {
int create_linear_from(const char *description, const char *mesh_file, int32_t order, int32_t physics,
                       const double *params, const char *tableau, int32_t precision, hgg_handle **out) {
    *out = nullptr;
    std::unique_ptr<StructuredProblem> sp(new StructuredProblem());
    LinearSystem sys;
    int rc = linear_structured_system(description, order, physics, params, tableau, *sp, sys, mesh_file);
    if (rc) return rc;
    hgg_problem_desc d;
    fill_descriptor(*sp, precision, d);
    hgg_handle *h = new (std::nothrow) hgg_handle();
    if (!h) return fail(nullptr, HGG_ERR_NOMEM, "host allocation failed");
    if ((rc = create_from_desc(&d, h, true)) || (rc = attach_linear(h, sys))) {
        g_create_error = h->err;
        destroy_handle(h);
        return rc;
    }
    // the distinct mass matrices, for the source terms' lifts
    {
        std::map<int32_t, int32_t> compact;
        const size_t RR = (size_t)sys.R * sys.R;
        h->lin_mass_of.resize(sys.E);
        for (int64_t e = 0; e < sys.E; ++e) {
            auto it = compact.find(sys.mass_id[e]);
            if (it == compact.end()) {
                it = compact.emplace(sys.mass_id[e], (int32_t)compact.size()).first;
                const double *m = sys.pool.get(sys.mass_id[e]);
                h->lin_mass.insert(h->lin_mass.end(), m, m + RR);
            }
            h->lin_mass_of[e] = it->second;
        }
    }
    h->linear_api = true;
    h->sp = std::move(sp);
    butcher_error_estimate(tableau, h->rk_err, h->rk_order);
    *out = h;
    return 0;
}
}  // namespace

extern "C" {

int hgg_create_linear_structured(const char *description, int32_t order, int32_t physics, const double *params,
                                 const char *tableau, int32_t precision, hgg_handle **out) {
    if (!description || !out || !tableau) return fail(nullptr, HGG_ERR_INVALID, "null argument");
    return create_linear_from(description, nullptr, order, physics, params, tableau, precision, out);
}

int hgg_create_linear_mesh_file(const char *path, int32_t order, int32_t physics, const double *params,
                                const char *tableau, int32_t precision, hgg_handle **out) {
    if (!path || !out || !tableau) return fail(nullptr, HGG_ERR_INVALID, "null argument");
    return create_linear_from(nullptr, path, order, physics, params, tableau, precision, out);
}

int32_t hgg_num_quadrature_points(const hgg_handle *h) { return h && h->sp ? h->sp->rule.size() : -1; }

int hgg_quadrature_points(const hgg_handle *h, double *xyz) {
    if (!h || !xyz) return HGG_ERR_INVALID;
    if (!h->sp) return fail(const_cast<hgg_handle *>(h), HGG_ERR_UNSUPPORTED, "handle not built from a structured mesh");
    const StructuredProblem &P = *h->sp;
    const int d = P.mesh.dim, nQ = P.rule.size();
    for (int64_t e = 0; e < P.mesh.n_elements; ++e)
        for (int q = 0; q < nQ; ++q) reference_to_physical(P.mesh, e, &P.rule.points[q * d], xyz + (e * nQ + q) * d);
    return 0;
}

int32_t hgg_num_error_points(const hgg_handle *h) { return h && h->sp ? h->sp->error_rule.size() : -1; }

int hgg_error_points(const hgg_handle *h, double *xyz) {
    if (!h || !xyz) return HGG_ERR_INVALID;
    if (!h->sp) return fail(const_cast<hgg_handle *>(h), HGG_ERR_UNSUPPORTED, "handle not built from a structured mesh");
    const StructuredProblem &P = *h->sp;
    const int d = P.mesh.dim, nQ = P.error_rule.size();
    for (int64_t e = 0; e < P.mesh.n_elements; ++e)
        for (int q = 0; q < nQ; ++q)
            reference_to_physical(P.mesh, e, &P.error_rule.points[q * d], xyz + (e * nQ + q) * d);
    return 0;
}

int hgg_project(hgg_handle *h, const double *values, int32_t vec) {
    if (!h || !values) return fail(h, HGG_ERR_INVALID, "null argument");
    if (!h->sp) return fail(h, HGG_ERR_UNSUPPORTED, "projection needs a handle built from a structured mesh");
    const StructuredProblem &P = *h->sp;
    const HostOperators &op = h->op;
    const int nB = op.nB, V = op.V, nQ = P.rule.size();
    // M^{-1} int phi u0 = Mhat^{-1} sum_q w_q phi u0(x_q): |J| and cInv cancel on affine elements
    std::vector<double> out((size_t)h->N), rhs(nB);
    for (int64_t e = 0; e < op.nE; ++e)
        for (int v = 0; v < V; ++v) {
            std::fill(rhs.begin(), rhs.end(), 0.0);
            for (int q = 0; q < nQ; ++q) {
                double val = P.rule.weights[q] * values[(e * nQ + q) * V + v];
                for (int i = 0; i < nB; ++i) rhs[i] += val * P.basis_values[q * nB + i];
            }
            double *o = &out[(e * V + v) * nB];
            for (int i = 0; i < nB; ++i) {
                double s = 0.0;
                for (int j = 0; j < nB; ++j) s += op.mass_inv[i * nB + j] * rhs[j];
                o[i] = s;
            }
        }
    return hgg_set_state(h, vec, out.data());
}

}  // extern "C"

// ---- error norms on the device -------------------------------------------------
// computeTotalError (HpgemAPISimplified_Impl.h:370-401, rule of order 2p+2) and
// computeMaxError (:499-530, the element rule): the caller gives the exact
// solution's values at the points (hgg_error_points / hgg_quadrature_points); one
// thread per element evaluates the discrete solution there and accumulates, then
// the elements' results are summed in a fixed order (L2) or maximised (max).

// per element: sum_q w_q |J_e| sum_v (exact - u_h)^2, the host loop's order
__global__ void element_l2_error(const double *u, const double *exact, const double *basis, const double *w,
                                 const double *absdet, int nq, int nb, int V, int64_t n_elements, double *out) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n_elements) return;
    double loc = 0.0;
    for (int q = 0; q < nq; ++q) {
        double s = 0.0;
        for (int v = 0; v < V; ++v) {
            double uh = 0.0;
            for (int j = 0; j < nb; ++j) uh += basis[q * nb + j] * u[(e * V + v) * nb + j];
            const double diff = exact[(e * nq + q) * V + v] - uh;
            s += diff * diff;
        }
        loc += w[q] * absdet[e] * s;
    }
    out[e] = loc;
}

// per element and variable: max_q |u_h - exact| at the element rule's points
__global__ void element_max_error(const double *u, const double *exact, const double *basis, int nq, int nb, int V,
                                  int64_t n_elements, double *out) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n_elements) return;
    for (int v = 0; v < V; ++v) {
        double m = 0.0;
        for (int q = 0; q < nq; ++q) {
            double uh = 0.0;
            for (int j = 0; j < nb; ++j) uh += u[(e * V + v) * nb + j] * basis[q * nb + j];
            const double d = fabs(uh - exact[(e * nq + q) * V + v]);
            if (d > m) m = d;
        }
        out[v * n_elements + e] = m;
    }
}

// out[v] = max over rows of a[v][:], one block per variable
__global__ void max_per_row(const double *a, int64_t n, double *out) {
    __shared__ double sm[kSumThreads];
    const double *row = a + blockIdx.x * n;
    double m = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += kSumThreads) m = fmax(m, row[i]);
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int w = kSumThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = sm[0];
}

namespace {

// a device view of vector `vec` in hpGEM order (element-major, FP64): the vector itself
// when it is stored that way, else its conversion in the scratch vector
int hpgem_order_view(hgg_handle *h, int vec, const double **view) {
    void *d = vector_ptr(h, vec);
    if (!d) return fail(h, HGG_ERR_INVALID, "vector id out of range");
    const bool f = vector_is_float(h, vec);
    if (!h->tensor_layout && !f) {
        *view = static_cast<const double *>(d);
        return 0;
    }
    const unsigned grid = 4 * h->num_sms;
    if (h->tensor_layout && f)
        from_tensor_order<float><<<grid, 256, 0, h->stream>>>(static_cast<const float *>(d), h->d_scratch, h->d_tpos,
                                                               h->d_tsign, h->op.nB, h->N, h->tiled);
    else if (h->tensor_layout)
        from_tensor_order<double><<<grid, 256, 0, h->stream>>>(static_cast<const double *>(d), h->d_scratch,
                                                                h->d_tpos, h->d_tsign, h->op.nB, h->N, h->tiled);
    else
        convert_vector<<<grid, 256, 0, h->stream>>>(static_cast<const float *>(d), h->d_scratch, h->N);
    h->launches++;
    HGG_CUDA(h, cudaGetLastError());
    *view = h->d_scratch;
    return 0;
}

// device copy of the caller's exact values (kept for the next call of the same size)
int exact_on_device(hgg_handle *h, const double *exact, size_t count, const double **out) {
    if (count > h->exact_cap) {
        if (h->d_exact) {
            for (auto it = h->bufs.begin(); it != h->bufs.end(); ++it)
                if (it->p == h->d_exact) {
                    cudaFreeAsync(it->p, h->stream);
                    h->bufs.erase(it);
                    break;
                }
            h->d_exact = nullptr;
        }
        int rc = alloc(h, sizeof(double) * count, (void **)&h->d_exact);
        if (rc) return rc;
        h->exact_cap = count;
    }
    HGG_CUDA(h, cudaMemcpyAsync(h->d_exact, exact, sizeof(double) * count, cudaMemcpyHostToDevice, h->stream));
    *out = h->d_exact;
    return 0;
}

int error_tables(hgg_handle *h) {
    if (h->d_err_basis) return 0;
    const StructuredProblem &P = *h->sp;
    int rc;
    if ((rc = upload(h, P.error_basis, &h->d_err_basis)) || (rc = upload(h, P.error_rule.weights, &h->d_err_w)) ||
        (rc = upload(h, P.basis_values, &h->d_elem_basis)) || (rc = upload(h, h->op.abs_det, &h->d_absdet)))
        return rc;
    if (!h->d_reduce) {
        rc = alloc(h, sizeof(double) * (size_t)(2 * h->op.nE + 1024), (void **)&h->d_reduce);
        if (rc) return rc;
    }
    return 0;
}

}  // namespace

extern "C" {

int hgg_l2_error(hgg_handle *h, int32_t vec, const double *exact, double *error) {
    if (!h || !exact || !error) return fail(h, HGG_ERR_INVALID, "null argument");
    if (!h->sp) return fail(h, HGG_ERR_UNSUPPORTED, "error norms need a handle built from a structured mesh");
    if (h->sp->error_rule.size() == 0)
        return fail(h, HGG_ERR_UNSUPPORTED, "no quadrature rule of order 2p+2 for this shape");
    int rc = error_tables(h);
    const double *u = nullptr, *ex = nullptr;
    const HostOperators &op = h->op;
    const int nQ = h->sp->error_rule.size();
    if (rc || (rc = hpgem_order_view(h, vec, &u)) ||
        (rc = exact_on_device(h, exact, (size_t)op.nE * nQ * op.V, &ex)))
        return rc;
    double *per = h->d_reduce, *pa = h->d_reduce + 2 * op.nE, *pb = pa + 256;
    element_l2_error<<<(unsigned)((op.nE + 255) / 256), 256, 0, h->stream>>>(u, ex, h->d_err_basis, h->d_err_w,
                                                                            h->d_absdet, nQ, op.nB, op.V, op.nE, per);
    sum_pairs<<<256, kSumThreads, 0, h->stream>>>(per, per, op.nE, pa, pb);
    sum_pairs<<<1, kSumThreads, 0, h->stream>>>(pa, pa, 256, pa + 512, pb + 512);
    h->launches += 3;
    HGG_CUDA(h, cudaGetLastError());
    double total = 0.0;
    HGG_CUDA(h, cudaMemcpyAsync(&total, pa + 512, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    HGG_CUDA(h, cudaStreamSynchronize(h->stream));
    *error = std::sqrt(std::fabs(total));
    return 0;
}

int hgg_max_error(hgg_handle *h, int32_t vec, const double *exact, double *max_error) {
    if (!h || !exact || !max_error) return fail(h, HGG_ERR_INVALID, "null argument");
    if (!h->sp) return fail(h, HGG_ERR_UNSUPPORTED, "error norms need a handle built from a structured mesh");
    int rc = error_tables(h);
    const double *u = nullptr, *ex = nullptr;
    const HostOperators &op = h->op;
    const int nQ = h->sp->rule.size();
    if (rc || (rc = hpgem_order_view(h, vec, &u)) ||
        (rc = exact_on_device(h, exact, (size_t)op.nE * nQ * op.V, &ex)))
        return rc;
    if (!h->d_maxbuf) {  // per element and variable, then per variable
        rc = alloc(h, sizeof(double) * ((size_t)op.V * op.nE + op.V), (void **)&h->d_maxbuf);
        if (rc) return rc;
    }
    double *per = h->d_maxbuf, *res = h->d_maxbuf + (int64_t)op.V * op.nE;
    element_max_error<<<(unsigned)((op.nE + 255) / 256), 256, 0, h->stream>>>(u, ex, h->d_elem_basis, nQ, op.nB,
                                                                             op.V, op.nE, per);
    max_per_row<<<op.V, kSumThreads, 0, h->stream>>>(per, op.nE, res);
    h->launches += 2;
    HGG_CUDA(h, cudaGetLastError());
    HGG_CUDA(h, cudaMemcpyAsync(max_error, res, sizeof(double) * op.V, cudaMemcpyDeviceToHost, h->stream));
    HGG_CUDA(h, cudaStreamSynchronize(h->stream));
    return 0;
}

}  // extern "C"
