// The device problem behind an hgg_handle, shared by the translation units of
// the library: the entry points (capi.cu), the stage launchers
// (stage_tensor.cu, stage_dense.cu) and the batch and serving loop (batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/hpgem_b200.h"
#include "dg_kernels.cuh"
#include "linear_stage.cuh"
#include "linear_umma.cuh"
#include "tensor_pipe.cuh"
#include "tensor_slice.cuh"
#include "host/linear.h"
#include "host/operators.h"
#include "host/setup.h"

namespace hgg {
struct SourceState;  // sources.cu
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};
}  // namespace hgg

struct hgg_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    hgg::HostOperators op;
    std::unique_ptr<hgg::StructuredProblem> sp;  // set when built from a structured description
    int S = 0;
    std::vector<double> rk_a, rk_b, rk_c;
    std::vector<double> rk_err;   // error coefficients of an embedded tableau (empty: none)
    int rk_order = 0;
    int64_t N = 0;                 // doubles per vector
    int64_t N_alloc = 0;           // doubles allocated per vector (whole tiles)
    double *sol[2] = {nullptr, nullptr};
    int cur = 0;                   // which sol[] holds the solution
    std::vector<void *> k;         // S stage vectors (double, or float in the FP32-mixed form)
    bool mixed = false;            // FP32-mixed form: float stage vectors and contractions
    std::vector<hgg::DevBuf> bufs;      // every device allocation
    // device operator / geometry arrays
    double *d_vol = nullptr, *d_pairs = nullptr, *d_elem_geo = nullptr, *d_face_geo = nullptr;
    float *d_vol_f = nullptr, *d_pairs_f = nullptr;  // FP32-mixed form: the dense operators in FP32
    int32_t *d_nbr = nullptr, *d_self = nullptr, *d_nbrp = nullptr;
    int8_t *d_mode = nullptr;
    double *d_ahat = nullptr, *d_tsigma = nullptr;
    int32_t *d_tnbr = nullptr;
    int8_t *d_tmode = nullptr;
    unsigned char *d_pgeo = nullptr;  // packed per-element geometry of the pipelined kernel
    int tile_elems = 1;               // elements per tile (common multiple of the tensor kernels' tiles)
    int variant = 0;                  // 0: automatic, 1: one-shot, 2: pipelined kernel
    bool tensor_layout = false;       // device vectors in tensor order (signs folded)
    bool tiled = false;               // ... and in tiles of 32 elements, coefficient-major (slice kernel)
    double *d_scratch = nullptr;      // one vector, for layout conversion of set/get_state
    double *d_reduce = nullptr;       // adaptive steps and error norms: per-element values, partial sums
    double *d_exact = nullptr;        // error norms: the caller's exact values on the device
    size_t exact_cap = 0;
    double *d_maxbuf = nullptr;
    double *d_err_basis = nullptr, *d_err_w = nullptr, *d_elem_basis = nullptr, *d_absdet = nullptr;
    int32_t *d_tpos = nullptr;        // hpGEM index -> tensor position
    double *d_tsign = nullptr;
    // slice kernel (hexahedra, p = 3): per-element records of SliceShape::GR doubles
    bool slice_ok = false;
    double *d_slice_geo = nullptr;
    // stored-matrix form (HpgemAPILinear): distinct folded matrices, transposed
    bool linear = false;
    int lin_R = 0, lin_slots = 0, lin_mats = 0;
    double *d_lin_table = nullptr;
    float *d_lin_table_f = nullptr;  // FP32-mixed form with FP32 contractions (R <= kMixedFp32MaxBasis)
    int32_t *d_lin_self = nullptr, *d_lin_nbr = nullptr, *d_lin_mat = nullptr;
    // grouped DMMA kernel: tiles of elements with identical matrices (0 tiles: not used)
    double *d_lin_table_rm = nullptr;
    int32_t *d_lin_tile_elems = nullptr, *d_lin_tile_mats = nullptr;
    int64_t lin_tiles = 0;
    int lin_min_rows = hgg::kLinTileMinRows;  // fewer rows per element: the row kernel
    // mixed forms on the tensor cores (tcgen05): tiles of 128 elements with identical
    // matrices, matrix operand images split into hi / lo parts
    int precision = 0;                     // enum hgg_precision
    int64_t umma_tiles = 0;                // 0: not used
    int32_t *d_umma_tile_elems = nullptr, *d_umma_tile_mats = nullptr;
    unsigned char *d_umma_img = nullptr;
    unsigned char *d_umma_planes = nullptr;  // split stage input, two planes [E][KP]
    // grouped dense kernel: tiles of group_tile_elems(nB) elements with the same operator signature
    int32_t *d_group_tiles = nullptr;
    double *d_win[2] = {nullptr, nullptr};  // stage inputs formed ahead (grouped wave kernel)
    int64_t group_tiles = 0;
    int num_sms = 148;
    int *d_status = nullptr;
    uint32_t test_arm_polls = 0;  // hgg_test_arm_without_copy: poll limit of the next pipelined launch
    // HpgemAPILinear source terms (sources.cu)
    bool linear_api = false;            // HpgemAPILinear built from a structured mesh or a mesh file
    std::vector<double> lin_mass;       // its distinct element mass matrices [n][R][R]
    std::vector<int32_t> lin_mass_of;   // [E]
    hgg::SourceState *src = nullptr;    // set: every stage adds the caller's source terms
    bool store_last = true;
    int64_t launches = 0;
    int64_t graph_launches = 0;  // kernels in one captured step
    // graph of one full step, per starting buffer, valid for (dt, store_last)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    double graph_dt = 0.0;
    bool graph_store_last = true;
    std::string err = "no error";
};

namespace hgg {

// records msg as the handle's last error (or the last create error) and returns code
int fail(hgg_handle *h, int code, const std::string &msg);

#define HGG_CUDA(h, call)                                                                    \
    do {                                                                                     \
        cudaError_t _e = (call);                                                             \
        if (_e != cudaSuccess)                                                               \
            return fail(h, HGG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
    } while (0)

// Device memory of a handle is stream-ordered (cudaMallocAsync / cudaFreeAsync on the
// handle's stream, from the device's default pool): freeing a handle never waits for
// work of other streams, so a solve that finishes inside a batch or a server is freed
// while the other members keep stepping.

// device copy of a host vector, owned by the handle
template <typename T>
int upload(hgg_handle *h, const std::vector<T> &v, T **dst) {
    *dst = nullptr;
    if (v.empty()) return 0;
    void *p = nullptr;
    size_t bytes = v.size() * sizeof(T);
    cudaError_t e = cudaMallocAsync(&p, bytes, h->stream);
    if (e != cudaSuccess) return fail(h, HGG_ERR_NOMEM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    h->bufs.push_back({p, bytes});
    e = cudaMemcpyAsync(p, v.data(), bytes, cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) return fail(h, HGG_ERR_CUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
    *dst = (T *)p;
    return 0;
}

int alloc(hgg_handle *h, size_t bytes, void **dst);
// the wave runs the grouped tile kernel (alone and in a batch): kernel variant 2, or
// the automatic choice where it measured faster than the per-row kernel
bool group_wave_wanted(const hgg_handle *h);
void release_graphs(hgg_handle *h);
// the current solution in hpGEM order with no kernel on the device: one copy of the
// device vector into `staging` (pinned, h->N_alloc doubles), the layout change on the host
int solution_to_host(hgg_handle *h, double *staging, double *out);

template <int P, int DIM>
TensorConsts<P, DIM> tensor_consts(const HostOperators &op) {
    using TC = TensorConsts<P, DIM>;
    TC tc;
    for (int i = 0; i < TC::NP * TC::NP; ++i) tc.D1[i] = op.D1[i];
    for (int i = 0; i < 2 * TC::NP; ++i) tc.lift[i] = op.lift[i];
    tc.trace_pos[0] = op.trace_pos[0];
    tc.trace_pos[1] = op.trace_pos[1];
    for (int i = 0; i < TC::NB; ++i) {
        tc.tpos[i] = (short)i;
        tc.tinv[i] = (short)i;
        tc.tsign[i] = 1.0;
    }
    return tc;
}

// layout conversion index (hpGEM order <-> tensor order, signs folded; tiled:
// 32-element tiles, coefficient-major inside a tile)
__host__ __device__ __forceinline__ int64_t device_index(int64_t e, int pos, int nb, bool tiled) {
    return tiled ? (e >> 5) * ((int64_t)nb << 5) + (int64_t)pos * 32 + (e & 31) : e * nb + pos;
}
// stage vectors and per-stage coefficients of the error estimate and the rewind
template <typename KT>
struct ErrStages {
    const KT *k[kMaxStages];
    double err[kMaxStages];
    double dt;
    int n;
};

// elements per tile of the pipelined kernel for (order, dim); bytes of its packed geometry
int pipe_tile_elems(int order, int dim);
int pipe_geo_bytes(int dim);
// wave speed factor of the upwind wave flux, 0 for the central flux
double upwind_speed(const HostOperators &op);

// one stage launch of the handle's kernel (stage_tensor.cu: slice and
// sum-factorised kernels; stage_dense.cu: dense and stored-matrix kernels)
int launch_stage_tensor(hgg_handle *h, const StageIOT<double> &io);
int launch_stage_tensor(hgg_handle *h, const StageIOT<float> &io);
int launch_stage_dense(hgg_handle *h, const StageIOT<double> &io);
int launch_stage_dense(hgg_handle *h, const StageIOT<float> &io);
int launch_stage_linear(hgg_handle *h, const StageIOT<double> &io);
int launch_stage_linear(hgg_handle *h, const StageIOT<float> &io);
// the handle's stage kernel, counted, with the launch error checked
int launch_stage(hgg_handle *h, const StageIO &io);
int launch_stage(hgg_handle *h, const StageIOT<float> &io);

void *vector_ptr(hgg_handle *h, int vec);
bool vector_is_float(const hgg_handle *h, int vec);

// Inputs and outputs of stage i of one Runge-Kutta step from sol[from] into
// sol[1 - from] (stages as in HpgemAPISimplified_Impl.h:788-820; zero tableau
// entries are skipped).
template <typename KT>
StageIOT<KT> make_stage_io(const hgg_handle *h, int from, double dt, int i, int *status) {
    const int S = h->S;
    auto kv = [&](int j) { return static_cast<KT *>(h->k[j]); };
    StageIOT<KT> io{};
    io.u = h->sol[from];
    io.n_elements = h->op.nE;
    io.status = status;
    for (int j = 0; j < i; ++j) {
        double c = dt * h->rk_a[i * S + j];
        if (c != 0.0) {
            io.kin[io.nin] = kv(j);
            io.cin[io.nin] = c;
            io.nin++;
        }
    }
    const bool last = i == S - 1;
    io.kout = (!last || h->store_last) ? kv(i) : nullptr;
    if (last) {
        io.unew = h->sol[1 - from];
        for (int j = 0; j < S - 1; ++j) {
            double b = dt * h->rk_b[j];
            if (b != 0.0) {
                io.kfin[io.nfin] = kv(j);
                io.bfin[io.nfin] = b;
                io.nfin++;
            }
        }
        io.blast = dt * h->rk_b[S - 1];
    }
    return io;
}

// source terms (sources.cu): the caller's functions evaluated at the stage times
// t + c_i dt of one step (buf 0 / 1: the step from sol[0] / sol[1]) or at
// `times` (buf 2) and copied to the device; the lift of stage `stage` added to
// kout (and blast times it to unew) after the stage kernel
int fill_sources(hgg_handle *h, int buf, double t, double dt);
int fill_source_values(hgg_handle *h, int buf, const double *times, int n);
int enqueue_source(hgg_handle *h, int buf, int stage, double *kout, double *unew, double blast);
int enqueue_source(hgg_handle *h, int buf, int stage, float *kout, double *unew, double blast);
void destroy_sources(hgg_handle *h);
// hgg_time_derivative (time null) and hgg_time_derivative_at
int time_derivative_impl(hgg_handle *h, int32_t in_vec, int32_t out_vec, const double *time);

// the failures a device status word records (bit 0: bad neighbour index, bit 1:
// a bounded wait ran out, bit 2: bad matrix index)
std::string status_message(int st);
// reads the device status word (synchronises the handle's stream)
int check_status(hgg_handle *h);

}  // namespace hgg
