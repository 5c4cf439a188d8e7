"""Many independent problems advanced together (hgg_batch_* of the C ABI).

Each problem is an ordinary solver (its own mesh, order, physics, dt and step
count); the batch runs every RK stage of all problems of one kernel class as
one persistent launch, the classes of a step as parallel branches of one CUDA
graph, and stops each problem at exactly its own step count.
"""
import ctypes

from . import _native


class Batch:
    def __init__(self, capacity):
        self._lib = _native.load()
        raw = ctypes.c_void_p()
        _native.check_batch(self._lib.hgg_batch_create(int(capacity), ctypes.byref(raw)))
        self._raw = raw
        self._members = {}  # slot -> solver

    def close(self):
        if self._raw:
            self._lib.hgg_batch_destroy(self._raw)
            self._raw = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, code):
        return _native.check_batch(code, self._raw)

    def add(self, solver, dt, nsteps):
        """Adds a solver (HpgemAPISimplified with a mesh read) to advance nsteps of dt."""
        slot = ctypes.c_int32()
        self._check(self._lib.hgg_batch_add(self._raw, solver.handle._raw, float(dt), int(nsteps),
                                            ctypes.byref(slot)))
        self._members[slot.value] = solver
        return slot.value

    def remove(self, slot):
        self._check(self._lib.hgg_batch_remove(self._raw, int(slot)))
        return self._members.pop(slot)

    def step(self, nsteps):
        self._check(self._lib.hgg_batch_step(self._raw, int(nsteps)))

    def synchronize(self):
        self._check(self._lib.hgg_batch_synchronize(self._raw))

    def remaining(self, slot):
        return int(self._lib.hgg_batch_remaining(self._raw, int(slot)))

    def set_autotune(self, enable):
        self._check(self._lib.hgg_batch_set_autotune(self._raw, 1 if enable else 0))

    @property
    def cuda_stream(self):
        """The batch's CUDA stream handle (an integer, for torch.cuda.ExternalStream)."""
        return int(self._lib.hgg_batch_stream(self._raw) or 0)

    @property
    def launch_count(self):
        return int(self._lib.hgg_batch_launch_count(self._raw))

    @property
    def num_classes(self):
        return int(self._lib.hgg_batch_num_classes(self._raw))

    KINDS = {0: "dense", 1: "sum-factorised", 2: "sum-factorised slices", 3: "stored-matrix tiles",
             4: "tensor-core tiles"}

    def class_info(self):
        """One dict per kernel class with members: kernel kind, shape, dim, order, physics,
        precision, stages, members, elements, coefficients."""
        import numpy as np
        out = []
        for i in range(self.num_classes):
            v = np.zeros(10, dtype=np.int64)
            _native.check_batch(self._lib.hgg_batch_class_info(self._raw, i, ctypes.c_void_p(v.ctypes.data)),
                                self._raw)
            out.append(dict(kind=self.KINDS.get(int(v[0]), int(v[0])), shape=int(v[1]), dim=int(v[2]),
                            order=int(v[3]), physics=int(v[4]), precision=int(v[5]), stages=int(v[6]),
                            members=int(v[7]), elements=int(v[8]), coefficients=int(v[9])))
        return out

    def profile_step(self):
        """One step, class after class, each timed with CUDA events: ms per class (the order
        of class_info)."""
        import numpy as np
        n = self.num_classes
        ms = np.zeros(max(n, 1))
        _native.check_batch(self._lib.hgg_batch_profile_step(self._raw, ctypes.c_void_p(ms.ctypes.data), n),
                            self._raw)
        return ms[:n]
