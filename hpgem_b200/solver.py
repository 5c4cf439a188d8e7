"""Python face of the library, shaped like hpGEM's HpgemAPISimplified<DIM>.

The method names follow the reference (kernel/Base/HpgemAPISimplified.h:
readMesh, setInitialSolution, computeOneTimeStep, computeTimeDerivative,
solve, computeTotalError, getTimeIntegrationVector) so that a caller of the
reference's stepping loop finds the same calls.  All work runs in the native
library through the C ABI; there is no Python or CPU fallback.
"""
import ctypes
import math

import numpy as np

from . import _native


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class Handle:
    """Owns one hgg_handle."""

    def __init__(self, raw):
        self._raw = raw
        self._lib = _native.load()

    @classmethod
    def from_descriptor(cls, desc: _native.ProblemDesc):
        lib = _native.load()
        h = ctypes.c_void_p()
        _native.check(lib.hgg_create(ctypes.byref(desc), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def structured(cls, description, order, physics, params, tableau="RK4_4",
                   precision=_native.PRECISION_FP64):
        lib = _native.load()
        h = ctypes.c_void_p()
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        _native.check(lib.hgg_create_structured(description.encode(), int(order), int(physics),
                                                _ptr(p), tableau.encode(), int(precision),
                                                ctypes.byref(h)))
        return cls(h)

    @classmethod
    def mesh_file(cls, path, order, physics, params, tableau="RK4_4", precision=_native.PRECISION_FP64):
        lib = _native.load()
        h = ctypes.c_void_p()
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        _native.check(lib.hgg_create_mesh_file(str(path).encode(), int(order), int(physics), _ptr(p),
                                               tableau.encode(), int(precision), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def linear_structured(cls, description, order, physics, params, tableau="RK4_4",
                          precision=_native.PRECISION_FP64):
        """HpgemAPILinear on a structured mesh: the stored matrices of the reference's
        linear advection / central-flux wave applications (hgg_create_linear_structured)."""
        lib = _native.load()
        h = ctypes.c_void_p()
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        _native.check(lib.hgg_create_linear_structured(description.encode(), int(order), int(physics),
                                                       _ptr(p), tableau.encode(), int(precision),
                                                       ctypes.byref(h)))
        return cls(h)

    @classmethod
    def linear_mesh_file(cls, path, order, physics, params, tableau="RK4_4", precision=_native.PRECISION_FP64):
        """HpgemAPILinear on a Preprocessor "mesh 2" file (hgg_create_linear_mesh_file)."""
        lib = _native.load()
        h = ctypes.c_void_p()
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        _native.check(lib.hgg_create_linear_mesh_file(str(path).encode(), int(order), int(physics), _ptr(p),
                                                      tableau.encode(), int(precision), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def linear(cls, mass, element_stiffness, face_elements, face_stiffness, rk_a, rk_b, rk_c=None,
               precision=_native.PRECISION_FP64):
        """HpgemAPILinear from the matrices hpGEM stored (hgg_create_linear): mass and
        element stiffness [E][R][R], face_elements [F][2] (right -1 on a boundary face),
        face_stiffness [F][4][R][R] (LL, LR, RL, RR blocks), Butcher tableau arrays."""
        lib = _native.load()
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        E, R = mass.shape[0], mass.shape[1]
        K = np.ascontiguousarray(element_stiffness, dtype=np.float64).reshape(E, R, R)
        fe = np.ascontiguousarray(face_elements, dtype=np.int64).reshape(-1, 2)
        fs = np.ascontiguousarray(face_stiffness, dtype=np.float64).reshape(len(fe), 4, R, R)
        a = np.ascontiguousarray(rk_a, dtype=np.float64)
        b = np.ascontiguousarray(rk_b, dtype=np.float64)
        c = np.ascontiguousarray(rk_c if rk_c is not None else np.zeros(len(b)), dtype=np.float64)
        d = _native.LinearDesc(n_rows=R, precision=int(precision), n_elements=E, mass=mass.ctypes.data,
                               element_stiffness=K.ctypes.data, n_faces=len(fe), face_elements=fe.ctypes.data,
                               face_stiffness=fs.ctypes.data, n_stages=len(b), rk_a=a.ctypes.data,
                               rk_b=b.ctypes.data, rk_c=c.ctypes.data)
        h = ctypes.c_void_p()
        _native.check(lib.hgg_create_linear(ctypes.byref(d), ctypes.byref(h)))
        return cls(h)

    def close(self):
        if self._raw is not None and self._raw.value:
            self._lib.hgg_destroy(self._raw)
        self._raw = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, code):
        return _native.check(code, self._raw)

    @property
    def vector_length(self):
        return int(self._lib.hgg_vector_length(self._raw))

    @property
    def kernel_kind(self):
        return {1: "tensor", 2: "linear", 3: "linear_tc"}.get(self._lib.hgg_kernel_kind(self._raw), "dense")

    @property
    def launch_count(self):
        return int(self._lib.hgg_launch_count(self._raw))

    def set_state(self, vec, values):
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        if a.size != self.vector_length:
            raise ValueError("vector has %d entries, expected %d" % (a.size, self.vector_length))
        self._check(self._lib.hgg_set_state(self._raw, int(vec), _ptr(a)))

    def set_state_ptr(self, vec, host_ptr):
        self._check(self._lib.hgg_set_state(self._raw, int(vec), ctypes.c_void_p(host_ptr)))

    def get_state(self, vec, out=None):
        if out is None:
            out = np.empty(self.vector_length)
        self._check(self._lib.hgg_get_state(self._raw, int(vec), _ptr(out)))
        return out

    def get_state_ptr(self, vec, host_ptr):
        self._check(self._lib.hgg_get_state(self._raw, int(vec), ctypes.c_void_p(host_ptr)))

    def step(self, time, dt, nsteps):
        t = ctypes.c_double(time)
        self._check(self._lib.hgg_step(self._raw, ctypes.byref(t), float(dt), int(nsteps)))
        return t.value

    def step_adaptive(self, time, max_relative_error, dt_max, dt_estimate):
        """One accepted adaptive step; returns (time, next dt estimate, dt taken, rejections)."""
        t = ctypes.c_double(time)
        est = ctypes.c_double(dt_estimate)
        taken = ctypes.c_double()
        rej = ctypes.c_int32()
        self._check(self._lib.hgg_step_adaptive(self._raw, ctypes.byref(t), float(max_relative_error),
                                                float(dt_max), ctypes.byref(est), ctypes.byref(taken),
                                                ctypes.byref(rej)))
        return t.value, est.value, taken.value, rej.value

    def set_error_estimate(self, error_coefficients, order):
        e = np.ascontiguousarray(np.asarray(error_coefficients, dtype=np.float64))
        self._check(self._lib.hgg_set_error_estimate(self._raw, _ptr(e), int(order)))

    def time_derivative(self, in_vec, out_vec, time=None):
        if time is None:
            self._check(self._lib.hgg_time_derivative(self._raw, int(in_vec), int(out_vec)))
        else:
            self._check(self._lib.hgg_time_derivative_at(self._raw, int(in_vec), int(out_vec), float(time)))

    def set_source(self, boundary, fn, n_vars):
        """hgg_set_boundary_source / hgg_set_element_source with a Python function:
        boundary: fn(x [n, dim], unit normals [n, dim], t); element: fn(x [n, dim], t);
        either returns g [n] or [n, n_vars].  None removes the term."""
        if fn is None:
            cb = None
        else:
            def cb_py(xyz, normals, n, dim, t, values, user):
                x = np.ctypeslib.as_array(xyz, shape=(n, dim))
                out = np.ctypeslib.as_array(values, shape=(n, n_vars))
                if boundary:
                    nn = np.ctypeslib.as_array(normals, shape=(n, dim))
                    g = fn(x, nn, t)
                else:
                    g = fn(x, t)
                out[:] = np.asarray(g, dtype=float).reshape(n, n_vars)
            cb = _native.SOURCE_FN(cb_py)
        setter = self._lib.hgg_set_boundary_source if boundary else self._lib.hgg_set_element_source
        self._check(setter(self._raw, ctypes.cast(cb, ctypes.c_void_p) if cb else None, None))
        # the library calls the function until it is replaced: keep it alive
        if not hasattr(self, "_sources"):
            self._sources = {}
        self._sources[boundary] = cb

    def synchronize(self):
        self._check(self._lib.hgg_synchronize(self._raw))

    def set_stream(self, stream_ptr):
        self._check(self._lib.hgg_set_stream(self._raw, ctypes.c_void_p(stream_ptr or None)))

    def set_kernel_variant(self, variant):
        self._check(self._lib.hgg_set_kernel_variant(self._raw, int(variant)))

    def set_store_last_stage(self, enable):
        self._check(self._lib.hgg_set_store_last_stage(self._raw, 1 if enable else 0))

    def quadrature_points(self, n_elements, dim):
        n = self._lib.hgg_num_quadrature_points(self._raw)
        if n < 0:
            raise _native.NativeError(-2, "no quadrature points for this handle")
        out = np.empty(n_elements * n * dim)
        self._check(self._lib.hgg_quadrature_points(self._raw, _ptr(out)))
        return out.reshape(n_elements, n, dim)

    def project(self, values, vec=0):
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        self._check(self._lib.hgg_project(self._raw, _ptr(a), int(vec)))

    def error_points(self, n_elements, dim):
        n = self._lib.hgg_num_error_points(self._raw)
        out = np.empty(n_elements * n * dim)
        self._check(self._lib.hgg_error_points(self._raw, _ptr(out)))
        return out.reshape(n_elements, n, dim)

    def max_error(self, vec, exact_values, n_vars):
        """Per variable, max |u_h - exact| at the element quadrature points (exact given there)."""
        a = np.ascontiguousarray(np.asarray(exact_values, dtype=np.float64).reshape(-1))
        out = np.zeros(int(n_vars), dtype=np.float64)
        self._check(self._lib.hgg_max_error(self._raw, int(vec), _ptr(a), _ptr(out)))
        return out

    def l2_error(self, vec, exact_values):
        a = np.ascontiguousarray(exact_values, dtype=np.float64).reshape(-1)
        err = ctypes.c_double()
        self._check(self._lib.hgg_l2_error(self._raw, int(vec), _ptr(a), ctypes.byref(err)))
        return err.value


class HpgemAPISimplified:
    """Explicit DG solver for one mesh, driven through the GPU library.

    ``physics`` is "advection" (linear advection, weak form, upwind flux,
    tests/self/Basic/090Advection_SelfTest.cpp) or "wave" (linear acoustic
    wave, strong form, central flux, applications/ExampleMultipleVariableProblem/
    AcousticWave_Impl.h).  ``tableau`` names one of hpGEM's Butcher tableaux;
    the reference's default for HpgemAPISimplified is Dormand-Prince
    (HpgemAPISimplified.h:150-155).
    """

    def __init__(self, dim, order, physics="advection", advection=None, c_inv=1.0,
                 tableau="DormandPrince", precision=_native.PRECISION_FP64):
        self.dim = int(dim)
        self.polynomialOrder = int(order)
        self.physics = physics
        self.tableau = tableau
        self.precision = precision
        if physics == "advection":
            self.numberOfVariables = 1
            a = np.zeros(3)
            if advection is not None:
                a[:self.dim] = np.asarray(advection, dtype=float)[:self.dim]
            self.params = a[:self.dim]
            self._physics_code = _native.PHYSICS_ADVECTION
        elif physics in ("wave", "wave_upwind"):
            self.numberOfVariables = self.dim + 1
            self.params = np.array([float(c_inv)])
            self._physics_code = _native.PHYSICS_WAVE if physics == "wave" else _native.PHYSICS_WAVE_UPWIND
        else:
            raise ValueError("physics must be 'advection', 'wave' or 'wave_upwind'")
        self.handle = None
        self.n_elements = 0
        self.dtEstimate = math.inf

    # -- set-up -------------------------------------------------------------
    def readMesh(self, description):
        """Creates the device problem from a Preprocessor 'structured' description."""
        self.handle = Handle.structured(description, self.polynomialOrder, self._physics_code,
                                        self.params, self.tableau, self.precision)
        self._description = description
        self._mass = None
        self.n_basis = _basis_count(self.dim, description, self.polynomialOrder)
        self.n_elements = self.handle.vector_length // (self.numberOfVariables * self.n_basis)
        return self

    def readMeshFile(self, path):
        """readMesh(fileName): creates the device problem from a Preprocessor "mesh 2" file."""
        from .descriptor import mesh_file_descriptor
        D = mesh_file_descriptor(str(path), self.polynomialOrder, self._physics_code, self.params, self.tableau)
        self.handle = Handle.mesh_file(path, self.polynomialOrder, self._physics_code, self.params,
                                       self.tableau, self.precision)
        self._description = None
        self._mesh_file = str(path)
        self._mass = None
        self.n_basis = D["n_basis"]
        self.n_elements = D["n_elements"]
        return self

    def quadraturePoints(self):
        return self.handle.quadrature_points(self.n_elements, self.dim)

    def setInitialSolution(self, u0, vec=0):
        """L2 projection of u0(x[n, dim]) -> [n] or [n, V] (setInitialSolution)."""
        x = self.quadraturePoints()
        vals = np.asarray(u0(x.reshape(-1, self.dim)), dtype=float)
        self.handle.project(vals.reshape(-1, self.numberOfVariables), vec)

    # -- time stepping ------------------------------------------------------
    def computeOneTimeStep(self, time, dt):
        return self.handle.step(time, dt, 1)

    def computeTimeSteps(self, time, dt, nsteps):
        return self.handle.step(time, dt, nsteps)

    def computeOneTimeStepAdaptive(self, time, maximumRelativeError, dtMax):
        """computeOneTimeStep(time, maximumRelativeError, dtMax) (HpgemAPISimplified_Impl.h:822-861):
        one accepted step of the embedded tableau; the next step's estimate is kept in
        ``dtEstimate`` (the reference keeps it in a static variable initialised from dt)."""
        time, self.dtEstimate, self.lastDt, self.lastRejections = self.handle.step_adaptive(
            time, maximumRelativeError, dtMax, self.dtEstimate)
        return time

    def solveAdaptive(self, initialTime, finalTime, maximumRelativeError, dt=math.inf,
                      numberOfOutputFrames=1, u0=None):
        """The adaptive branch of HpgemAPISimplified::solve (HpgemAPISimplified_Impl.h:976-1045):
        steps until finalTime, each limited by dt and by the next output time and the final
        time; returns (time, number of accepted steps)."""
        T = finalTime - initialTime
        if math.isfinite(dt):
            steps = int(math.ceil(T / dt))
            if numberOfOutputFrames > 0:
                steps += (numberOfOutputFrames - steps % numberOfOutputFrames) % numberOfOutputFrames
                dt = T / steps
        outputDt = T / numberOfOutputFrames
        outputTime = outputDt + initialTime
        if u0 is not None:
            self.setInitialSolution(u0)
        self.dtEstimate = dt
        time, n = initialTime, 0
        while time < finalTime - 1e-14:
            n += 1
            time = self.computeOneTimeStepAdaptive(time, maximumRelativeError,
                                                   min(min(dt, outputTime - time), finalTime - time))
            if time > outputTime - 1e-12:
                outputTime += outputDt
        return time, n

    def computeTimeDerivative(self, in_vec, out_vec, time=None):
        """computeTimeDerivative(in, out, time); the time matters for source terms only."""
        self.handle.time_derivative(in_vec, out_vec, time)

    def solve(self, initialTime, finalTime, dt, numberOfOutputFrames=1, u0=None):
        """Time loop of HpgemAPISimplified::solve (HpgemAPISimplified_Impl.h:976-1045):
        the step count is ceil(T/dt) rounded up to a multiple of the number of
        output frames, and dt is recomputed from it."""
        T = finalTime - initialTime
        steps = int(math.ceil(T / dt))
        if numberOfOutputFrames > 0:
            steps += (numberOfOutputFrames - steps % numberOfOutputFrames) % numberOfOutputFrames
            dt = T / steps
        if u0 is not None:
            self.setInitialSolution(u0)
        return self.handle.step(initialTime, dt, steps), steps, dt

    # -- state and errors -----------------------------------------------------
    def getTimeIntegrationVector(self, vec=0):
        return self.handle.get_state(vec).reshape(self.n_elements, self.numberOfVariables * self.n_basis)

    def setTimeIntegrationVector(self, vec, values):
        self.handle.set_state(vec, values)

    def l2Distance(self, a, b):
        """L2 norm of the difference of two coefficient vectors (hpGEM order) of this
        mesh: sqrt(sum_e |J_e| d_e^T Mhat d_e), exact on affine elements (the element
        rule of order 2p+1 integrates the degree-2p mass integrand exactly)."""
        if getattr(self, "_mass", None) is None:
            from .descriptor import mesh_file_descriptor, structured_descriptor
            if self._description is not None:
                D = structured_descriptor(self._description, self.polynomialOrder, self._physics_code,
                                          self.params, self.tableau)
            else:
                D = mesh_file_descriptor(self._mesh_file, self.polynomialOrder, self._physics_code,
                                         self.params, self.tableau)
            phi = D["basis_values"]
            self._mass = np.einsum("q,qi,qj->ij", D["quad_weights"], phi, phi)
            self._absdet = np.abs(np.linalg.det(D["jacobians"]))
        nE, V, nB = self.n_elements, self.numberOfVariables, self.n_basis
        d = (np.asarray(a, dtype=float) - np.asarray(b, dtype=float)).reshape(nE, V, nB)
        return float(np.sqrt(np.einsum("evi,ij,evj,e->", d, self._mass, d, self._absdet)))

    def computeTotalError(self, exact, time, vec=0):
        """L2 error against exact(x[n, dim], t) -> [n] or [n, V], rule of order 2p+2."""
        x = self.handle.error_points(self.n_elements, self.dim)
        vals = np.asarray(exact(x.reshape(-1, self.dim), time), dtype=float)
        return self.handle.l2_error(vec, vals.reshape(-1, self.numberOfVariables))

    def computeMaxError(self, exact, time, vec=0):
        """computeMaxError (HpgemAPISimplified_Impl.h:499-530): per variable, the largest
        |u_h - exact| at the element quadrature points; exact(x[n, dim], t) -> [n] or [n, V]."""
        x = self.quadraturePoints()
        vals = np.asarray(exact(x.reshape(-1, self.dim), time), dtype=float)
        return self.handle.max_error(vec, vals.reshape(-1, self.numberOfVariables), self.numberOfVariables)


class HpgemAPILinear(HpgemAPISimplified):
    """HpgemAPILinear<DIM> (kernel/Base/HpgemAPILinear.h): the element and face
    matrices are built once before the time loop (createMassMatrices,
    createStiffnessMatrices) and every stage multiplies them
    (multiplyStiffnessMatrices) and solves with the stored mass matrix.
    ``physics`` "advection" has the integrands of
    tests/self/Basic/080AdvectionLinear_SelfTest.cpp, "wave" those of
    applications/ExampleMultipleVariableProblem/AcousticWaveLinear_Impl.h.
    Everything after readMesh is the inherited time loop."""

    def __init__(self, dim, order, physics="advection", advection=None, c_inv=1.0,
                 tableau="RK4_4", precision=_native.PRECISION_FP64):
        if physics not in ("advection", "wave", "wave_upwind"):
            raise ValueError("the linear applications are 'advection' and 'wave' (the reference's central "
                             "flux; 'wave_upwind' folds the upwind flux of the matrix-free wave the same way)")
        super().__init__(dim, order, physics, advection=advection, c_inv=c_inv, tableau=tableau,
                         precision=precision)

    def readMesh(self, description):
        """readMesh + tasksBeforeSolving (HpgemAPILinear_Impl.h:107-129, :500-506)."""
        self.handle = Handle.linear_structured(description, self.polynomialOrder, self._physics_code,
                                               self.params, self.tableau, self.precision)
        self._description = description
        self._mass = None
        self.n_basis = _basis_count(self.dim, description, self.polynomialOrder)
        self.n_elements = self.handle.vector_length // (self.numberOfVariables * self.n_basis)
        return self

    def setSourceTerm(self, g):
        """useSourceTerm (HpgemAPILinear_Impl.h:437-450): every stage adds the element
        integrals of phi_i g_v(x, t); g(x [n, dim], t) -> [n] or [n, V].  None: off."""
        self.handle.set_source(False, g, self.numberOfVariables)

    def setSourceTermAtBoundary(self, g):
        """useSourceTermAtBoundary (HpgemAPILinear_Impl.h:452-469): every stage adds, for
        every boundary face, the face integrals of phi_i g_v(x, n, t) to its element;
        g(x [n, dim], unit normals [n, dim], t) -> [n] or [n, V].  None: off."""
        self.handle.set_source(True, g, self.numberOfVariables)

    def readMeshFile(self, path):
        """readMesh(fileName) + tasksBeforeSolving on a Preprocessor "mesh 2" file."""
        from .descriptor import mesh_file_descriptor
        D = mesh_file_descriptor(str(path), self.polynomialOrder, self._physics_code, self.params, self.tableau)
        self.handle = Handle.linear_mesh_file(path, self.polynomialOrder, self._physics_code, self.params,
                                              self.tableau, self.precision)
        self._description = None
        self._mesh_file = str(path)
        self._mass = None
        self.n_basis = D["n_basis"]
        self.n_elements = D["n_elements"]
        return self


def _basis_count(dim, description, p):
    tri = "triangular" in description.split()
    if dim == 1:
        return p + 1
    if dim == 2:
        return (p + 1) * (p + 2) // 2 if tri else (p + 1) ** 2
    return (p + 1) * (p + 2) * (p + 3) // 6 if tri else (p + 1) ** 3


def Advection(dim, order, a, tableau="DormandPrince", **kw):
    """The matrix-free advection application of 090Advection_SelfTest.cpp."""
    return HpgemAPISimplified(dim, order, "advection", advection=a, tableau=tableau, **kw)


def AcousticWave(dim, order, c_inv=1.0, tableau="RK4_4", flux="central", **kw):
    """The acoustic-wave application of ExampleMultipleVariableProblem (RK4 default, main.cpp:74-75);
    flux "central" is the reference's, "upwind" the restated Riemann flux."""
    if flux not in ("central", "upwind"):
        raise ValueError("flux must be 'central' or 'upwind'")
    return HpgemAPISimplified(dim, order, "wave" if flux == "central" else "wave_upwind", c_inv=c_inv,
                              tableau=tableau, **kw)


def structured_description(n, lower, upper, triangular=False, periodic=True):
    """Text of a Preprocessor 'structured' mesh description (Preprocessor README)."""
    d = len(n)
    per = periodic if isinstance(periodic, (list, tuple)) else [periodic] * d
    return "structured 1 %d\n%s\n%s\n%s\n%s\n%s\n" % (
        d, " ".join(str(int(v)) for v in n), " ".join(repr(float(v)) for v in lower),
        " ".join(repr(float(v)) for v in upper), "triangular" if triangular else "rectangular",
        " ".join("true" if p else "false" for p in per))
