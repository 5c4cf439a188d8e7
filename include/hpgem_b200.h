/*
 * hpgem_b200: B200 (sm_100a) explicit discontinuous-Galerkin time stepping,
 * a drop-in for hpGEM's HpgemAPISimplified<DIM> time loop.
 *
 * The library advances the element coefficient vectors of one (or many)
 * meshes through explicit Runge-Kutta steps on the GPU.  The physics is
 * selected by an enum instead of hpGEM's virtual integrands:
 *   HGG_PHYSICS_ADVECTION  linear advection, weak form, upwind flux
 *                          (tests/self/Basic/090Advection_SelfTest.cpp:92-220)
 *   HGG_PHYSICS_WAVE       linear acoustic wave, first-order system,
 *                          strong form, central flux
 *                          (applications/ExampleMultipleVariableProblem/
 *                           AcousticWave_Impl.h:102-373)
 *   HGG_PHYSICS_WAVE_UPWIND  the same system with the upwind (Riemann) flux:
 *                          the central flux plus the jump penalty
 *                          (1/2) |A_n| [[U]], which for v_t = div s,
 *                          c_inv s_t = grad v is c |n| [[v]] / 2 in the
 *                          first equation and c c_inv n (n . [[s]]) / (2 |n|)
 *                          in the others, c = 1 / sqrt(c_inv).  The
 *                          reference has the central flux only; this flux
 *                          is the one its wave benchmark names.
 *
 * Conventions shared by every entry point:
 *   - Return value 0 on success, a negative HGG_ERR_* code otherwise; the
 *     message is available from hgg_last_error().  No C++ exception crosses
 *     this boundary.
 *   - Coefficient vectors are FP64, element-major, and inside an element
 *     variable-major: index (e * n_vars + v) * n_basis + i, exactly hpGEM's
 *     ElementData::convertToSingleIndex layout (kernel/Base/ElementData.h:209-225)
 *     concatenated over elements in element-id order.
 *   - Vector ids follow hpGEM's time-integration vectors: 0 is the solution,
 *     1..S are the Runge-Kutta stage derivatives
 *     (kernel/Base/HpgemAPISimplified_Impl.h:93-99).
 *   - A handle is used by one host thread at a time; all device work of a
 *     handle runs on its own CUDA stream.
 */
#ifndef HPGEM_B200_H
#define HPGEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum hgg_shape {
    HGG_SHAPE_LINE = 1,
    HGG_SHAPE_SQUARE = 2,
    HGG_SHAPE_TRIANGLE = 3,
    HGG_SHAPE_CUBE = 4,
    HGG_SHAPE_TETRAHEDRON = 5
};

enum hgg_physics { HGG_PHYSICS_ADVECTION = 0, HGG_PHYSICS_WAVE = 1, HGG_PHYSICS_WAVE_UPWIND = 2 };

enum hgg_precision {
    HGG_PRECISION_FP64 = 0,  /* everything in FP64 (parity form) */
    HGG_PRECISION_FP32 = 1,  /* FP32-mixed: FP32 stage vectors and contractions; geometry, mass
                                inverse, stage input and RK sums in FP64.  Where the stage is
                                a dense product (stored-matrix tiles, folded operators) the
                                contractions run on the tensor cores as three TF32 products
                                (hi*hi + hi*lo + lo*hi of split operands), FP32-accurate */
    HGG_PRECISION_BF16X3 = 2 /* split-BF16: as FP32 but every contraction on the tensor cores as
                                three BF16 products of split operands with FP32 accumulation
                                (about 2^-17 of each product); only handles whose stage runs as
                                tiles of dense products (stored matrices, folded operators on
                                structured meshes), else HGG_ERR_UNSUPPORTED */
};

enum hgg_error {
    HGG_OK = 0,
    HGG_ERR_INVALID = -1,      /* bad argument or descriptor */
    HGG_ERR_UNSUPPORTED = -2,  /* valid hpGEM input outside what this library implements */
    HGG_ERR_CUDA = -3,         /* a CUDA call failed */
    HGG_ERR_NOMEM = -4,        /* host or device allocation failed */
    HGG_ERR_DEVICE = -5,       /* a kernel reported an error through its status word */
    HGG_ERR_NOT_LOADED = -6    /* no CUDA device / kernels not loadable */
};

typedef struct hgg_handle hgg_handle;

/*
 * Everything hpGEM knows about one mesh that the time loop needs, taken
 * from its own objects (an hpGEM-side subclass fills it from the mesh's
 * elements and faces, the quadrature rules and the Butcher tableau):
 *   - basis values and reference gradients at the element quadrature points
 *     (PhysicalElement::basisFunction / basisFunctionDeriv before the
 *     J^{-T} transform; GaussQuadratureRule::eval caches),
 *   - basis values at face quadrature points mapped into the element through
 *     a local face and a face-to-face orientation (PhysicalFace::basisFunction
 *     on the LEFT and RIGHT side; FaceGeometry::mapRefFaceToRefElemL/R),
 *   - the element Jacobians (ElementGeometry::calcJacobian; the elements must
 *     be affine, which every structured Preprocessor mesh is),
 *   - per face, the normal of FaceGeometry::getNormalVector (outward from the
 *     left element, length = physical / reference face measure),
 *   - the Butcher tableau (TimeIntegration::ButcherTableau).
 * All arrays are copied during hgg_create; the caller may free them after.
 */
typedef struct hgg_problem_desc {
    int32_t dim;            /* 1, 2 or 3 */
    int32_t shape;          /* enum hgg_shape of every element */
    int32_t order;          /* polynomial order p of hpGEM's default DG basis */
    int32_t n_vars;         /* 1 for advection, dim + 1 for the wave system */
    int32_t physics;        /* enum hgg_physics */
    int32_t precision;      /* enum hgg_precision */
    double advection[3];    /* advection velocity a (first dim entries used) */
    double c_inv;           /* wave material parameter cInv = 1/c^2 (AcousticWave::cInv_) */

    int64_t n_elements;
    int32_t n_basis;        /* basis functions per element and variable */

    int32_t n_quad;                /* element quadrature points */
    const double *quad_weights;    /* [n_quad] reference weights */
    const double *basis_values;    /* [n_quad][n_basis] */
    const double *basis_grads;     /* [n_quad][n_basis][dim] reference gradients */

    int32_t n_face_quad;           /* face quadrature points */
    const double *face_weights;    /* [n_face_quad] reference-face weights */
    int32_t n_face_tabs;           /* number of distinct face tabulations */
    const double *face_tabs;       /* [n_face_tabs][n_face_quad][n_basis] */

    const double *jacobians;       /* [n_elements][dim][dim], J[r][c] = dx_r / dxi_c */

    int64_t n_faces;
    const int64_t *face_elements;  /* [n_faces][2]: left, right element (right >= 0) */
    const int32_t *face_local;     /* [n_faces][2]: local face number on left, right */
    const int32_t *face_tab_index; /* [n_faces][2]: tabulation index of the left, right side */
    const double *face_normals;    /* [n_faces][dim] */

    int32_t n_stages;              /* S */
    const double *rk_a;            /* [S][S], row i holds a_ij for j < i */
    const double *rk_b;            /* [S] */
    const double *rk_c;            /* [S] */
} hgg_problem_desc;

/* ---- drop-in boundary: what hpGEM's HpgemAPISimplified<DIM> calls ------- */

/* Builds the device problem.  Replaces the host set-up hpGEM does before its
 * time loop (HpgemAPISimplified::readMesh + tasksBeforeSolving,
 * kernel/Base/HpgemAPISimplified_Impl.h:139-160).  Device: current device. */
int hgg_create(const hgg_problem_desc *desc, hgg_handle **out);

/* Frees the handle and all its device memory. */
int hgg_destroy(hgg_handle *h);

/* Message of the last failure on this handle (or of the last failed create
 * when h is NULL).  Never NULL. */
const char *hgg_last_error(const hgg_handle *h);

/* Host -> device copy of time-integration vector `vec` (0..S).
 * Replaces writing Element::getTimeIntegrationVector(vec) element by element. */
int hgg_set_state(hgg_handle *h, int32_t vec, const double *host);

/* Device -> host copy of time-integration vector `vec`.  Replaces reading
 * Element::getTimeIntegrationVector(vec) (output frames, error norms). */
int hgg_get_state(hgg_handle *h, int32_t vec, double *host);

/* `nsteps` explicit Runge-Kutta steps of size dt; *time advances by dt each.
 * Replaces HpgemAPISimplified::computeOneTimeStep(double&, double)
 * (kernel/Base/HpgemAPISimplified_Impl.h:788-820) called nsteps times.
 * Stage vectors 1..S hold the last step's stage derivatives afterwards. */
int hgg_step(hgg_handle *h, double *time, double dt, int32_t nsteps);

/* out = M^{-1} R(in): replaces HpgemAPISimplified::computeTimeDerivative(in,
 * out, t) (kernel/Base/HpgemAPISimplified_Impl.h:764-770), i.e.
 * computeRightHandSide + solveMassMatrixEquations for one vector. */
int hgg_time_derivative(hgg_handle *h, int32_t in_vec, int32_t out_vec);

/* Blocks until all device work of the handle is done. */
int hgg_synchronize(hgg_handle *h);

/* Number of coefficients of one vector (n_elements * n_vars * n_basis). */
int64_t hgg_vector_length(const hgg_handle *h);

/* 1 when the sum-factorised tensor-product kernel drives this handle,
 * 0 when the dense reference-operator kernel does, 2 for the stored-matrix
 * kernels: handles from hgg_create_linear*, and matrix-free handles whose
 * operator the library folded into per-element matrices because the grouped
 * tensor-core kernel applies them faster (advection on triangles, p >= 4);
 * 3 for the same stored-matrix tiles on the fifth-generation tensor cores
 * (tcgen05: the FP32-mixed form as three TF32 products, the split-BF16 form as
 * three BF16 products, 128-element tiles). */
int hgg_kernel_kind(const hgg_handle *h);

/* When enabled (default), the last stage derivative k_S is stored like the
 * other stages; disabling it saves one vector write per step when no caller
 * reads vector S after a step. */
int hgg_set_store_last_stage(hgg_handle *h, int32_t enable);

/* Runs the handle's device work on `stream` (a cudaStream_t of the handle's
 * device; NULL restores the handle's own stream). */
int hgg_set_stream(hgg_handle *h, void *stream);

/* Selects the kernel organisation: 0 (default) automatic; on the
 * sum-factorised path 1 is one block per small group of elements and 2 the
 * pipelined kernel; on the dense path 1 runs one thread per element row and 2
 * the grouped kernel (tiles of elements with equal operators) wherever the
 * mesh has such tiles, whatever the contraction type (automatic takes it for
 * the wave with FP64 contractions).  All compute the same result; the choice
 * exists for comparison and profiling.
 * Hexahedra of order 3 keep their vectors in a tiled layout that only their
 * slice kernel reads: any variant but 0 returns HGG_ERR_UNSUPPORTED there. */
int hgg_set_kernel_variant(hgg_handle *h, int32_t variant);

/* Right-hand side k = M^{-1} R(u) of caller-owned DEVICE vectors u and k, both
 * in hpGEM order (length hgg_vector_length), without any allocation: no
 * cudaMalloc, cudaFree or allocating library call.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory while
 * they step (a serving loop that admits work by a fixed HBM budget, a host
 * application whose memory manager owns the device, code running where an
 * allocation's implicit device synchronisation would stall co-scheduled
 * work).  The sum-factorised handles need two vectors of scratch; they come
 * from one file-scope device array of 2^22 doubles (32 MiB) that every GPU
 * using the library holds until the process exits, so one device vector may
 * hold at most 2^21 doubles, else HGG_ERR_UNSUPPORTED.  A device vector is
 * hgg_vector_length padded with the elements that complete the kernel's last
 * tile (of 7 to 128 elements, by shape and order), which adds fewer than 2048
 * doubles, so every problem with hgg_vector_length <= 2^21 - 2048 fits (32^3
 * hexahedra at p = 3 is the largest cube mesh of that order).  The first call
 * on a device looks the array up (with the handle's device current, which
 * every call requires); make that first call before any stream capture.  All
 * calls on a device share the array and it keeps the last call's contents:
 * each call clears the padding elements of its input (the stage kernels read
 * them and discard what they compute from them); calls that overlap on the
 * GPU, from different streams or handles, race.  Runs on the handle's stream
 * and returns after it (like hgg_time_derivative, whose result it
 * reproduces). */
int hgg_time_derivative_static(hgg_handle *h, const double *u, double *k);

/* computeOneTimeStep(time, maximumRelativeError, dtMax)
 * (HpgemAPISimplified_Impl.h:822-861): one accepted step of an embedded tableau
 * (DormandPrince, BogackiShampine) with the reference's error control.  A trial
 * step of dt = min(*dt_estimate, dt_max) is taken; with error = the Euclidean
 * norm of sum_i dt err_i k_i over all coefficients and norm = the sum over
 * elements of the Euclidean norms of the updated solution
 * (computeErrorAndNormOfUpdate, :719-749), it is undone (u -= dt b_j k_j) and
 * retried with dt = 0.8 dt (max_relative_error norm / error)^(1/order) while
 * max_relative_error * norm < error.  On return *time has advanced by the
 * accepted dt (*dt_taken), *dt_estimate holds the next estimate
 * 0.9 dt (max_relative_error norm / error)^(1/order) (the reference keeps it in
 * a static variable), *rejections counts the undone tries.  dt_taken and
 * rejections may be null.  HGG_ERR_INVALID if the tableau has no error
 * estimate. */
int hgg_step_adaptive(hgg_handle *h, double *time, double max_relative_error, double dt_max, double *dt_estimate,
                      double *dt_taken, int32_t *rejections);

/* Error coefficients (b_i - b*_i, one per stage) and order of the handle's
 * embedded tableau (ButcherTableau::getErrorCoefficient / getOrder,
 * ButcherTableau.h:58-72), for handles made by hgg_create from a descriptor;
 * hgg_create_structured sets them for DormandPrince and BogackiShampine. */
int hgg_set_error_estimate(hgg_handle *h, const double *error_coefficients, int32_t order);

/* Number of kernel launches the library issued on this handle so far. */
int64_t hgg_launch_count(const hgg_handle *h);

/* Test of the device-side failure path; no counterpart in the reference.  The
 * next stage launch of the pipelined kernel (kernel variant 2 on a
 * sum-factorised handle, outside stream capture) arms the mbarrier of every
 * block's first tile with the tile's byte count but issues no copy, and gives
 * up waiting on any mbarrier after `polls` polls: every block then waits
 * (bounded) for the copies it did issue, sets bit 1 of the handle's status
 * word and returns, so the call that launched it (hgg_time_derivative,
 * hgg_synchronize) returns HGG_ERR_DEVICE while the CUDA context stays
 * usable.  The status word stays set: the handle is then only destroyed.
 * HGG_ERR_UNSUPPORTED on handles of other kernels. */
int hgg_test_arm_without_copy(hgg_handle *h, int32_t polls);

/* ---- stand-alone set-up: hpGEM's host side, restated ------------------- */

/* Builds the descriptor hpGEM would build from a Preprocessor "structured"
 * mesh description (applications/Preprocessor/lib/hpgem.cpp:55-265), its
 * default DG basis of order p, the Gauss rules of order 2p+1 and the named
 * Butcher tableau ("RK4_4", "DormandPrince", "ForwardEuler", "MidPoint",
 * "RK2TVD", "RK3TVD", "BogackiShampine"), and creates the handle from it.
 * params: advection velocity (dim values) for advection, {c_inv} for the wave. */
int hgg_create_structured(const char *description, int32_t order, int32_t physics,
                          const double *params, const char *tableau, int32_t precision,
                          hgg_handle **out);

/* The same descriptor, built on the host only (no device needed): fills *out
 * with arrays owned by *owner, valid until hgg_free_descriptor(*owner). */
int hgg_structured_descriptor(const char *description, int32_t order, int32_t physics,
                              const double *params, const char *tableau, int32_t precision,
                              hgg_problem_desc *out, void **owner);
void hgg_free_descriptor(void *owner);

/* readMesh(fileName) (kernel/Base/MeshManipulator_Impl.h:1505-) for a
 * Preprocessor "mesh 2" file (applications/Preprocessor/lib/hpgem.cpp writes
 * it; version 1 files are rejected), then the same set-up as
 * hgg_create_structured: the mesh goes from the file straight to the
 * descriptor's arrays (no per-element objects).  Element
 * shapes must be uniform and every face must have two elements (periodic
 * meshes); the element order and vertex order are the file's. */
int hgg_create_mesh_file(const char *path, int32_t order, int32_t physics, const double *params,
                         const char *tableau, int32_t precision, hgg_handle **out);

/* The same descriptor, host only (like hgg_structured_descriptor). */
int hgg_mesh_file_descriptor(const char *path, int32_t order, int32_t physics, const double *params,
                             const char *tableau, int32_t precision, hgg_problem_desc *out, void **owner);

/* Element quadrature points in physical coordinates, [n_elements][n_quad][dim]
 * (PhysicalElement::getPointPhysical at each point of the element rule). */
int hgg_quadrature_points(const hgg_handle *h, double *xyz);
int32_t hgg_num_quadrature_points(const hgg_handle *h);

/* setInitialSolution (HpgemAPISimplified_Impl.h:751-758): L2 projection of
 * the initial condition, given at the element quadrature points as
 * values[n_elements][n_quad][n_vars], into vector `vec`. */
int hgg_project(hgg_handle *h, const double *values, int32_t vec);

/* computeTotalError (HpgemAPISimplified_Impl.h:370-401): the L2 error of
 * vector `vec` against exact values given at the error-rule points
 * (rule of order 2p+2, :354-361) returned by hgg_error_points. */
int32_t hgg_num_error_points(const hgg_handle *h);
int hgg_error_points(const hgg_handle *h, double *xyz);
int hgg_l2_error(hgg_handle *h, int32_t vec, const double *exact, double *error);

/* computeMaxError (HpgemAPISimplified_Impl.h:499-530 with :406-463): per
 * variable, the largest |u_h - exact| over every element's quadrature points
 * (the element rule of hgg_quadrature_points), exact values given there as
 * exact[n_elements][n_quad][n_vars]; max_error receives n_vars values.  Both
 * norms are evaluated on the device; only the exact values cross to it. */
int hgg_max_error(hgg_handle *h, int32_t vec, const double *exact, double *max_error);

/* ---- HpgemAPILinear: stored element and face matrices ---------------------
 * HpgemAPILinear<DIM> (kernel/Base/HpgemAPILinear_Impl.h) builds, before its
 * time loop, per element a mass matrix (createMassMatrices, :131-139) and a
 * stiffness matrix, and per face the four blocks of a face stiffness matrix
 * (createStiffnessMatrices, :250-288).  Every stage it multiplies them with
 * the stage input (multiplyStiffnessMatrices, :291-434) and solves with the
 * stored mass matrix (solveMassMatrixEquations, :143-156).  The library takes
 * those matrices as hpGEM built them, so any linear application's integrands
 * run unchanged; on the device each element's stage is
 *   k_e = D_e w_e + sum_s N_{e,s} w_{n(e,s)},
 *   D_e = M_e^{-1} (K_e + its own-side face blocks),
 *   N_{e,s} = M_e^{-1} (the block coupling to neighbour n(e,s)),
 * with every distinct matrix stored once (structured meshes repeat a few).
 * Rows and columns use hpGEM's element index iV * n_basis + iB. */
typedef struct hgg_linear_desc {
    int32_t n_rows;                   /* R: coefficients per element (n_vars * n_basis) */
    int32_t precision;                /* enum hgg_precision */
    int64_t n_elements;
    const double *mass;               /* [n_elements][R][R], row-major */
    const double *element_stiffness;  /* [n_elements][R][R] */
    int64_t n_faces;
    const int64_t *face_elements;     /* [n_faces][2]: left, right element; right = -1 on a boundary face */
    const double *face_stiffness;     /* [n_faces][4][R][R]: FaceMatrix::getElementMatrix(iSide, jSide)
                                         for (LEFT,LEFT), (LEFT,RIGHT), (RIGHT,LEFT), (RIGHT,RIGHT);
                                         on a boundary face only (LEFT,LEFT) is read */
    int32_t n_stages;                 /* Butcher tableau, as in hgg_problem_desc */
    const double *rk_a;
    const double *rk_b;
    const double *rk_c;
} hgg_linear_desc;

/* HpgemAPILinear::readMesh + tasksBeforeSolving: a handle whose stages apply
 * the stored matrices.  Every time-loop entry point (hgg_set_state,
 * hgg_step, hgg_time_derivative, hgg_step_adaptive after
 * hgg_set_error_estimate, hgg_get_state, ...) works on it unchanged; at most
 * 256 rows per element. */
int hgg_create_linear(const hgg_linear_desc *desc, hgg_handle **out);

/* The matrices of the reference's two linear applications on a structured
 * mesh: physics HGG_PHYSICS_ADVECTION assembles the integrands of
 * tests/self/Basic/080AdvectionLinear_SelfTest.cpp:108-168 (weak form, upwind
 * flux), HGG_PHYSICS_WAVE those of applications/ExampleMultipleVariableProblem/
 * AcousticWaveLinear_Impl.h:98-284 (strong form, central flux).  Host only:
 * fills *out with arrays owned by *owner (hgg_free_linear_descriptor). */
int hgg_linear_descriptor(const char *description, int32_t order, int32_t physics, const double *params,
                          const char *tableau, int32_t precision, hgg_linear_desc *out, void **owner);
void hgg_free_linear_descriptor(void *owner);

/* The same matrices, assembled without the per-element arrays (identical
 * matrices kept once) and handed to the device; the handle also has the
 * structured mesh's projection, quadrature points and error norms. */
int hgg_create_linear_structured(const char *description, int32_t order, int32_t physics,
                                 const double *params, const char *tableau, int32_t precision,
                                 hgg_handle **out);

/* The same from a Preprocessor "mesh 2" file (HpgemAPILinear::readMesh(fileName),
 * HpgemAPILinear_Impl.h:107-129; the file as for hgg_create_mesh_file). */
int hgg_create_linear_mesh_file(const char *path, int32_t order, int32_t physics, const double *params,
                                const char *tableau, int32_t precision, hgg_handle **out);

/* Both stored-matrix constructors above take meshes with boundary faces
 * (non-periodic directions): a boundary face contributes its (LEFT, LEFT)
 * block, with the application's boundary integrand (advection: the upwind
 * outflow term, nothing on inflow faces; wave: -n_d phi_j phi_i in the
 * (p, s_d) block, AcousticWaveLinear_Impl.h:254-272). */

/* Source terms of HpgemAPILinear: useSourceTerm / useSourceTermAtBoundary with
 * addSourceTerm and addSourceTermAtBoundary (HpgemAPILinear_Impl.h:437-469),
 * which computeRightHandSide (:471-498) calls after the stiffness multiply and
 * before the mass solve, in every stage at the stage time t + c_i dt.  The
 * integrand is phi_i(x) g_v(x, t) for basis function i of variable v, as in
 * computeIntegrandSourceTermAtElement (:201-229) and in the face integrands
 * of the reference's applications (080AdvectionLinear_SelfTest.cpp:72-88:
 * g = -u_exact(x, t) (a . n) on inflow faces, 0 elsewhere); the library
 * integrates it with the element rule times |J| (ElementIntegral) and the
 * face rule times |n| (FaceIntegral).  The caller's function writes
 * values[n_points][n_vars] = g(xyz[k], t) for every point: the element
 * quadrature points of every element for the element source (normals null),
 * and the face quadrature points of every boundary face, face by face, with
 * the unit normal out of its element, for the boundary source.  It is called
 * on the thread that steps the handle, once per stage time of each step
 * (hgg_step evaluates a step's stage times while the GPU runs the previous
 * step), never from a CUDA callback.  fn = NULL removes the term.  Only for
 * handles from hgg_create_linear_structured / hgg_create_linear_mesh_file
 * (they know the mesh), else HGG_ERR_UNSUPPORTED.  A handle with source terms
 * needs the time: hgg_step with a non-null time, hgg_time_derivative_at
 * (hgg_time_derivative and hgg_time_derivative_static return an error), and
 * is not taken by batches. */
typedef void (*hgg_source_fn)(const double *xyz, const double *normals, int64_t n_points, int32_t dim, double time,
                              double *values, void *user);
int hgg_set_element_source(hgg_handle *h, hgg_source_fn fn, void *user);
int hgg_set_boundary_source(hgg_handle *h, hgg_source_fn fn, void *user);

/* computeTimeDerivative(in, out, time) (HpgemAPISimplified_Impl.h:764-770)
 * with the time the source terms are evaluated at; the same as
 * hgg_time_derivative for handles without source terms. */
int hgg_time_derivative_at(hgg_handle *h, int32_t in_vec, int32_t out_vec, double time);

/* ---- many problems at once ------------------------------------------------
 * No counterpart in the reference (hpGEM advances one mesh per process).  A
 * batch advances many independent problems, each an existing handle with its
 * own mesh, order, physics, dt and step count, together: every RK stage of all
 * members of one kernel class (organisation, shape, order, physics,
 * precision, tableau) is one persistent launch over all their element blocks,
 * the classes of a step run as parallel branches of one CUDA graph, and each
 * problem stops at exactly its own step count.  Launch shapes per class are
 * picked by timing candidates on the members (autotuner, cached per class and
 * size for the process).  A handle in a batch must not be stepped, read or
 * destroyed through its own entry points until hgg_batch_synchronize (read)
 * or hgg_batch_remove (anything) has returned. */
typedef struct hgg_batch hgg_batch;

/* A batch with room for `capacity` problems on the current device. */
int hgg_batch_create(int32_t capacity, hgg_batch **out);
int hgg_batch_destroy(hgg_batch *b);
const char *hgg_batch_last_error(const hgg_batch *b);

/* Adds handle h, to advance `nsteps` steps of `dt` from its current solution;
 * *slot receives its slot number. */
int hgg_batch_add(hgg_batch *b, hgg_handle *h, double dt, int32_t nsteps, int32_t *slot);

/* Takes the problem out of the batch (waits for the batch's work); the handle's
 * solution is then its state after the steps it took. */
int hgg_batch_remove(hgg_batch *b, int32_t slot);

/* Enqueues nsteps steps of every member that still has steps to take (asynchronous). */
int hgg_batch_step(hgg_batch *b, int32_t nsteps);

/* Waits for the batch, reads every member's remaining step count and the
 * device status word (HGG_ERR_DEVICE on a bad neighbour index). */
int hgg_batch_synchronize(hgg_batch *b);

/* Steps the member in `slot` still has to take, as of the last synchronize;
 * -1 for an empty slot. */
int32_t hgg_batch_remaining(const hgg_batch *b, int32_t slot);

/* 1 (default): time candidate launch shapes per kernel class; 0: fixed defaults. */
int hgg_batch_set_autotune(hgg_batch *b, int32_t enable);

/* Kernel launches the batch enqueued so far; kernel classes with members. */
int64_t hgg_batch_launch_count(const hgg_batch *b);
int32_t hgg_batch_num_classes(const hgg_batch *b);

/* The batch's own CUDA stream (every step is enqueued on it): for timing with
 * CUDA events.  No counterpart in the reference. */
void *hgg_batch_stream(const hgg_batch *b);

/* Kernel class i (0 .. hgg_batch_num_classes - 1, classes with members):
 * info10 = kind (0 matrix-free dense, 1 sum-factorised, 2 sum-factorised slices,
 * 3 stored-matrix tiles, 4 tensor-core tiles), shape, dim, order, physics,
 * precision (0 FP64, 1 FP32-mixed, 2 split-BF16), stages, members, elements,
 * coefficients. */
int hgg_batch_class_info(const hgg_batch *b, int32_t i, int64_t *info10);

/* One step of every member with steps left, class after class on the batch
 * stream, each class's stages timed with CUDA events: ms[i] for class i (the
 * order of hgg_batch_class_info).  Synchronous; for profiling the mix. */
int hgg_batch_profile_step(hgg_batch *b, double *ms, int32_t n);

/* ---- serving loop ------------------------------------------------------------
 * No counterpart in the reference.  A server admits solves (a Preprocessor
 * structured description, order, physics, parameters, tableau, precision,
 * initial condition, dt, step count) in arrival order while their device
 * footprint fits a byte budget, keeps their state on the device, and advances
 * all running solves together through one batch of the kind above (every RK stage of all
 * running solves of a kernel class is one launch); solves that arrive while
 * others run join at the next chunk boundary, and a finished solve's memory
 * admits the next.  Set-up (host descriptor, handle, projection) runs on
 * `setup_threads` threads beside the GPU thread; the GPU thread keeps two chunks
 * of steps in flight, and a retire thread copies finished solutions back and
 * frees their memory.  submit/poll/release/times/stats are thread-safe. */
typedef struct hgg_server hgg_server;

/* Initial condition callback: values[n_points][n_vars] at points xyz[n_points][dim]
 * (the element quadrature points; the server projects the values). */
typedef void (*hgg_initial_fn)(const double *xyz, int64_t n_points, int32_t dim, double *values, void *user);

/* Starts a server on the current device: budget_bytes of device memory for the
 * solves' state, at most max_chunk steps between admissions, `capacity`
 * solves running at once. */
int hgg_server_start(int64_t budget_bytes, int32_t max_chunk, int32_t setup_threads, int32_t capacity,
                     hgg_server **out);

/* Queues one solve; the initial condition is either n_u0 coefficients in hpGEM
 * order (u0) or a callback (init_fn, user; called on a set-up thread). */
int hgg_server_submit(hgg_server *s, const char *description, int32_t order, int32_t physics, const double *params,
                      int32_t n_params, const char *tableau, int32_t precision, const double *u0, int64_t n_u0,
                      hgg_initial_fn init_fn, void *user, double dt, int32_t nsteps, int64_t *id);

/* 1 when the solve is done (its solution copied into out[n_out] unless out is
 * null; *latency_s = done - submit), 0 while it is queued or running, < 0 if it
 * failed (message via hgg_server_last_error).  wait != 0 blocks until done. */
int hgg_server_poll(hgg_server *s, int64_t id, int32_t wait, double *out, int64_t n_out, double *latency_s);

/* Coefficients in a finished solve's solution (0 while not finished). */
int64_t hgg_server_result_length(hgg_server *s, int64_t id);

/* Forgets a finished solve. */
int hgg_server_release(hgg_server *s, int64_t id);

/* Steady-clock times in seconds of submit, set-up done, first step, done. */
int hgg_server_times(hgg_server *s, int64_t id, double *t4);

/* Completed solves, their DoF-updates, chunks stepped, device bytes reserved now. */
int hgg_server_stats(hgg_server *s, int64_t *stats4);

/* Seconds so far: [0] the GPU thread stepping (issuing the chunks' graph launches,
 * which block while the device's launch queue is full, and waiting for chunks),
 * [1] the GPU thread's membership work (joins, removals, table uploads, graph
 * captures), [2] the GPU thread waiting for work, [3] the retire thread
 * (solutions copied back, device memory freed), [4] device time of the chunks
 * (CUDA events on the batch stream); parts of [1]: [5] joins, [6] table uploads
 * and graph captures; part of [3]: [7] copies back. */
int hgg_server_timing(hgg_server *s, double *t8);

const char *hgg_server_last_error(hgg_server *s);

/* Waits for every submitted solve, stops the threads, frees the server. */
int hgg_server_stop(hgg_server *s);

#ifdef __cplusplus
}
#endif

#endif /* HPGEM_B200_H */
