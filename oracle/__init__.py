"""CPU oracle for the hpGEM explicit-DG time-stepping path.

TEST INFRASTRUCTURE ONLY.  Nothing in the ``hpgem_b200`` package imports,
links or runs anything in this folder; only the tests, the smoke check and the
CPU-baseline leg of ``bench.py`` use it, and only as a checker or as the timed
CPU reference.

What it is: a restatement, in numpy (set-up) and plain C (the stepping loop),
of hpGEM's own algorithm for ``HpgemAPISimplified::computeOneTimeStep`` on the
matrix-free advection (``tests/self/Basic/090Advection_SelfTest.cpp``) and
acoustic-wave (``applications/ExampleMultipleVariableProblem/AcousticWave_Impl.h``)
applications: the structured mesh of hpGEM's Preprocessor, the default H1
hierarchical DG basis, the Gauss rules of order 2p+1, the element loop and the
both-sides face loop evaluated at quadrature points, the element mass matrix
rebuilt by quadrature and LU-solved with partial pivoting in every stage, and
the Butcher-tableau Runge-Kutta update.  Every function cites the reference
file and line it follows.

How it is pinned (tests/test_oracle_*.py):
* the structured meshes against the Preprocessor's output in ``tests/files``;
* the basis functions and the quadrature rules against the known-answer
  integrals of hpGEM's quadrature unit tests;
* the whole pipeline against the L2-error goldens of the reference's
  advection self-test (1D / 2D triangles / 3D cubes, Dormand-Prince), at the
  reference test's own 1 % tolerance.
The reference itself cannot be built here under this project's rules (it needs
CMake, a generated source file and an external BLAS/LAPACK), so no
coefficient-level output of the reference is available; coefficient-level
parity of the GPU path is checked against this oracle.
"""
