// Source terms of HpgemAPILinear on the device: hgg_set_element_source,
// hgg_set_boundary_source, hgg_time_derivative_at.
//
// The reference adds, in every stage after the stiffness multiply and before
// the mass solve, the integrals of the application's source integrands
// (addSourceTerm, addSourceTermAtBoundary, kernel/Base/HpgemAPILinear_Impl.h:
// 437-469, called from computeRightHandSide, :471-498).  Here the caller's
// functions are evaluated on the host at the stage times of a step (all stages
// of the step at once, into a pinned buffer, while the GPU runs the previous
// step), copied to the device, and one small kernel per stage adds their lift
// L g (the mass inverse folded into L, host/sources.h) to the stage's
// derivative and, in the final stage, dt b_S L g to the new solution (the
// fused update already holds dt b_S k_S without the source).
#include <algorithm>
#include <string>
#include <vector>

#include "handle.cuh"
#include "host/sources.h"

namespace hgg {

struct SourceState {
    hgg_source_fn elem_fn = nullptr, face_fn = nullptr;
    void *elem_user = nullptr, *face_user = nullptr;
    SourcePlan plan;
    int64_t stride = 0;  // values per evaluation time
    double *d_table = nullptr;
    int64_t *d_table_off = nullptr, *d_off = nullptr;
    int32_t *d_cols = nullptr, *d_elem = nullptr, *d_ptr = nullptr, *d_lift = nullptr;
    // [0], [1]: the stage values of a step from sol[0] / sol[1]; [2]: one time
    double *d_vals[3] = {nullptr, nullptr, nullptr};
    double *h_vals[3] = {nullptr, nullptr, nullptr};  // pinned
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};  // the copy out of h_vals[i] is done
    std::vector<void *> dev;
};

namespace {

struct SourceArgs {
    const double *table;
    const int64_t *table_off;
    const int32_t *cols;
    const int32_t *elem, *ptr, *lift;
    const int64_t *off;
    int R;
};

// one block per element with a source; thread r: row r of the element's
// increment sum over its entries of L g (entries in the reference's order)
template <typename KT>
__global__ void __launch_bounds__(256)
    add_sources(const SourceArgs a, const double *g, KT *k, double *unew, double blast) {
    const int b = blockIdx.x;
    const int64_t e = a.elem[b];
    const int i0 = a.ptr[b], i1 = a.ptr[b + 1];
    for (int r = threadIdx.x; r < a.R; r += blockDim.x) {
        double acc = 0.0;
        for (int i = i0; i < i1; ++i) {
            const int l = a.lift[i];
            const double *L = a.table + a.table_off[l];
            const double *gv = g + a.off[i];
            const int cols = a.cols[l];
            for (int c = 0; c < cols; ++c) acc += L[(int64_t)c * a.R + r] * gv[c];
        }
        const int64_t idx = e * a.R + r;
        if (k) k[idx] = (KT)((double)k[idx] + acc);
        if (unew) unew[idx] += blast * acc;
    }
}

void free_state(SourceState *s) {
    if (!s) return;
    for (void *p : s->dev) cudaFree(p);
    for (int i = 0; i < 3; ++i) {
        if (s->h_vals[i]) cudaFreeHost(s->h_vals[i]);
        if (s->ev[i]) cudaEventDestroy(s->ev[i]);
    }
    delete s;
}

template <typename T>
int dev_copy(hgg_handle *h, SourceState *s, const std::vector<T> &v, T **out) {
    *out = nullptr;
    const size_t bytes = std::max<size_t>(1, v.size()) * sizeof(T);
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) return fail(h, HGG_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    s->dev.push_back(p);
    if (!v.empty()) HGG_CUDA(h, cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, h->stream));
    *out = static_cast<T *>(p);
    return 0;
}

// (re)builds the plan and the device tables for the functions now set
int rebuild(hgg_handle *h, hgg_source_fn efn, void *euser, hgg_source_fn ffn, void *fuser) {
    HGG_CUDA(h, cudaStreamSynchronize(h->stream));
    release_graphs(h);
    free_state(h->src);
    h->src = nullptr;
    if (!efn && !ffn) return 0;
    SourceState *s = new (std::nothrow) SourceState();
    if (!s) return fail(h, HGG_ERR_NOMEM, "host allocation failed");
    s->elem_fn = efn;
    s->elem_user = euser;
    s->face_fn = ffn;
    s->face_user = fuser;
    auto bail = [&](int rc) {
        cudaStreamSynchronize(h->stream);
        free_state(s);
        return rc;
    };
    try {
        s->plan = plan_sources(*h->sp, h->lin_mass, h->lin_mass_of, efn != nullptr, ffn != nullptr);
    } catch (const std::exception &ex) {
        return bail(fail(h, HGG_ERR_INVALID, ex.what()));
    }
    const SourcePlan &p = s->plan;
    s->stride = std::max<int64_t>(1, p.values);
    int rc;
    if ((rc = dev_copy(h, s, p.table, &s->d_table)) || (rc = dev_copy(h, s, p.table_off, &s->d_table_off)) ||
        (rc = dev_copy(h, s, p.table_cols, &s->d_cols)) || (rc = dev_copy(h, s, p.elem, &s->d_elem)) ||
        (rc = dev_copy(h, s, p.ptr, &s->d_ptr)) || (rc = dev_copy(h, s, p.lift, &s->d_lift)) ||
        (rc = dev_copy(h, s, p.off, &s->d_off)))
        return bail(rc);
    for (int i = 0; i < 3; ++i) {
        const size_t n = (size_t)s->stride * (i < 2 ? h->S : 1);
        if ((rc = dev_copy(h, s, std::vector<double>(n, 0.0), &s->d_vals[i]))) return bail(rc);
        cudaError_t e = cudaMallocHost((void **)&s->h_vals[i], n * sizeof(double));
        if (e != cudaSuccess) return bail(fail(h, HGG_ERR_NOMEM, std::string("cudaMallocHost: ") + cudaGetErrorString(e)));
        e = cudaEventCreateWithFlags(&s->ev[i], cudaEventDisableTiming);
        if (e != cudaSuccess) return bail(fail(h, HGG_ERR_CUDA, std::string("cudaEventCreate: ") + cudaGetErrorString(e)));
    }
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return bail(fail(h, HGG_ERR_CUDA, std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e)));
    h->src = s;
    return 0;
}

int set_source(hgg_handle *h, bool boundary, hgg_source_fn fn, void *user) {
    if (!h) return fail(h, HGG_ERR_INVALID, "null handle");
    if (!h->linear_api || !h->sp)
        return fail(h, HGG_ERR_UNSUPPORTED,
                    "source terms need an HpgemAPILinear handle built from a structured mesh or a mesh file "
                    "(hgg_create_linear_structured, hgg_create_linear_mesh_file)");
    hgg_source_fn efn = h->src ? h->src->elem_fn : nullptr, ffn = h->src ? h->src->face_fn : nullptr;
    void *eu = h->src ? h->src->elem_user : nullptr, *fu = h->src ? h->src->face_user : nullptr;
    if (boundary) {
        ffn = fn;
        fu = user;
    } else {
        efn = fn;
        eu = user;
    }
    return rebuild(h, efn, eu, ffn, fu);
}

template <typename KT>
int enqueue_source_t(hgg_handle *h, int buf, int stage, KT *kout, double *unew, double blast) {
    SourceState *s = h->src;
    if (!s || s->plan.elem.empty() || (!kout && !unew)) return 0;
    const SourceArgs a{s->d_table, s->d_table_off, s->d_cols, s->d_elem, s->d_ptr, s->d_lift, s->d_off, s->plan.R};
    const int threads = std::min(256, (s->plan.R + 31) / 32 * 32);
    add_sources<KT><<<(unsigned)s->plan.elem.size(), threads, 0, h->stream>>>(a, s->d_vals[buf] + stage * s->stride,
                                                                              kout, unew, blast);
    h->launches++;
    HGG_CUDA(h, cudaGetLastError());
    return 0;
}

}  // namespace

int fill_source_values(hgg_handle *h, int buf, const double *times, int n) {
    SourceState *s = h->src;
    if (!s) return 0;
    HGG_CUDA(h, cudaEventSynchronize(s->ev[buf]));  // the last copy out of this host buffer is done
    const SourcePlan &p = s->plan;
    for (int i = 0; i < n; ++i) {
        double *vals = s->h_vals[buf] + (size_t)i * s->stride;
        if (s->elem_fn && p.n_elem_points)
            s->elem_fn(p.elem_xyz.data(), nullptr, p.n_elem_points, p.dim, times[i], vals, s->elem_user);
        if (s->face_fn && p.n_face_points)
            s->face_fn(p.face_xyz.data(), p.face_normals.data(), p.n_face_points, p.dim, times[i],
                       vals + p.n_elem_points * p.V, s->face_user);
    }
    HGG_CUDA(h, cudaMemcpyAsync(s->d_vals[buf], s->h_vals[buf], sizeof(double) * n * s->stride,
                                cudaMemcpyHostToDevice, h->stream));
    HGG_CUDA(h, cudaEventRecord(s->ev[buf], h->stream));
    return 0;
}

int fill_sources(hgg_handle *h, int buf, double t, double dt) {
    std::vector<double> times(h->S);
    for (int i = 0; i < h->S; ++i) times[i] = t + h->rk_c[i] * dt;
    return fill_source_values(h, buf, times.data(), h->S);
}

int enqueue_source(hgg_handle *h, int buf, int stage, double *kout, double *unew, double blast) {
    return enqueue_source_t<double>(h, buf, stage, kout, unew, blast);
}
int enqueue_source(hgg_handle *h, int buf, int stage, float *kout, double *unew, double blast) {
    return enqueue_source_t<float>(h, buf, stage, kout, unew, blast);
}

void destroy_sources(hgg_handle *h) {
    if (!h || !h->src) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_state(h->src);
    h->src = nullptr;
}

}  // namespace hgg

using namespace hgg;

extern "C" {

int hgg_set_element_source(hgg_handle *h, hgg_source_fn fn, void *user) { return set_source(h, false, fn, user); }

int hgg_set_boundary_source(hgg_handle *h, hgg_source_fn fn, void *user) { return set_source(h, true, fn, user); }

int hgg_time_derivative_at(hgg_handle *h, int32_t in_vec, int32_t out_vec, double time) {
    return time_derivative_impl(h, in_vec, out_vec, &time);
}

}  // extern "C"
