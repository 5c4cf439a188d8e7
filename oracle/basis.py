"""hpGEM's default DG basis sets (test infrastructure only; see oracle/__init__.py).

Restates, function by function and in the same order, the sets built by
  createDGBasisFunctionSet1DH1Line        kernel/FE/BasisFunctions1DH1ConformingLine.cpp:85-108
  createDGBasisFunctionSet2DH1Square      kernel/FE/BasisFunctions2DH1ConformingSquare.cpp:164-184
  createDGBasisFunctions2DH1Triangle      kernel/FE/BasisFunctions2DH1ConformingTriangle.cpp:176-200
  createDGBasisFunctionSet3DH1Cube        kernel/FE/BasisFunctions3DH1ConformingCube.cpp:434-528
  createDGBasisFunctionSet3DH1Tetrahedron kernel/FE/BasisFunctions3DH1ConformingTetrahedron.cpp:366-409
with the Lobatto kernels of kernel/FE/helperFunctions.cpp:49-108 and the
barycentric coordinates of helperFunctions.cpp:140-168.

Values are the reference's ``eval`` formulas.  Gradients are the exact
derivatives of those formulas, taken by complex-step differentiation
(f'(x) = Im f(x + i h) / h, exact to rounding for polynomials); the
reference's hand-written ``evalDeriv*`` formulas are the product-rule
derivatives of its ``eval`` formulas, so both agree to rounding.
"""
import math

import numpy as np

from .refgeom import SHAPES


def lobatto(k, x):
    """Lobatto kernel of degree k without the (1 - x^2) factor.

    helperFunctions.cpp:49-92, including its degree-5 expression
    ``((33 x^2 - 30 x^2) + 5) x`` exactly as written there.
    """
    if k == 0:
        return math.sqrt(3.0 / 2.0) * -2.0 + 0.0 * x
    if k == 1:
        return math.sqrt(5.0 / 2.0) * x * -2.0
    if k == 2:
        return math.sqrt(7.0 / 2.0) * (5 * x * x - 1) / -2.0
    if k == 3:
        return math.sqrt(9.0 / 2.0) * (7 * x * x - 3) * x / -2.0
    if k == 4:
        return math.sqrt(11.0 / 2.0) * ((21 * x * x - 14) * x * x + 1) / -4.0
    if k == 5:
        return math.sqrt(13.0 / 2.0) * ((33 * x * x - 30 * x * x) + 5) * x / -4.0
    if k == 6:
        return math.sqrt(15.0 / 2.0) * (((429 * x * x - 495) * x * x + 135) * x * x - 5) / -32.0
    if k == 7:
        return math.sqrt(17.0 / 2.0) * (((715 * x * x - 1001) * x * x + 385) * x * x - 35) * x / -32.0
    if k == 8:
        return math.sqrt(19.0 / 2.0) * ((((2431 * x * x - 4004) * x * x + 2002) * x * x - 308)
                                        * x * x + 7) / -64.0
    if k == 9:
        return math.sqrt(21.0 / 2.0) * ((((4199 * x * x - 7956) * x * x + 4914) * x * x - 1092)
                                        * x * x + 63) * x / -64.0
    return legendre_deriv(k + 1, x)


def legendre(k, x):
    """helperFunctions.cpp:110-122 (three-term recurrence)."""
    if k == 0:
        return 1.0 + 0.0 * x
    if k == 1:
        return x
    return (2.0 * k - 1.0) / k * x * legendre(k - 1, x) - (k - 1.0) / k * legendre(k - 2, x)


def legendre_deriv(k, x):
    """helperFunctions.cpp:124-137."""
    if k == 0:
        return 0.0 * x
    if k == 1:
        return 1.0 + 0.0 * x
    return ((2.0 * k - 1.0) / k * (x * legendre_deriv(k - 1, x) + legendre(k - 1, x))
            - (k - 1.0) / k * legendre_deriv(k - 2, x))


def _line_set(p):
    fs = []
    if p == 0:
        return [lambda X: 1.0 + 0.0 * X[:, 0]]
    for node in (0, 1):
        npos = 2 * node - 1
        fs.append(lambda X, npos=npos: (1.0 + npos * X[:, 0]) / 2.0)
    for i in range(0, p - 1):
        fs.append(lambda X, i=i: (1 + X[:, 0]) * (1 - X[:, 0]) * lobatto(i, X[:, 0]) / 4.0)
    return fs


def _square_set(p):
    assert p > 0
    fs = []
    for node in range(4):
        n0 = (node % 2) * 2 - 1
        n1 = (node // 2) * 2 - 1
        fs.append(lambda X, n0=n0, n1=n1: (1 + n0 * X[:, 0]) * (1 + n1 * X[:, 1]) / 4.0)

    def face0(node0, node1, k):  # BasisFunction2DFaceSquare_0, Square.cpp:68-100
        mir = -1 if node0 > node1 else 1
        ep = -1 if node0 + node1 < 3 else 1
        return lambda X: ((1 + ep * X[:, 1]) * (1 - X[:, 0]) * (1 + X[:, 0])
                          * lobatto(k, mir * X[:, 0]) / 8.0)

    def face1(node0, node1, k):  # BasisFunction2DFaceSquare_1, Square.cpp:102-134
        mir = -1 if node0 > node1 else 1
        ep = -1 if node0 + node1 < 3 else 1
        return lambda X: ((1 + ep * X[:, 0]) * (1 - X[:, 1]) * (1 + X[:, 1])
                          * lobatto(k, mir * X[:, 1]) / 8.0)

    def interior(k0, k1):  # BasisFunction2DInteriorSquare, Square.cpp:136-162
        return lambda X: ((1 - X[:, 0]) * (1 + X[:, 0]) * (1 - X[:, 1]) * (1 + X[:, 1])
                          * lobatto(k0, X[:, 0]) * lobatto(k1, X[:, 1]) / 16.0)

    for i in range(0, p - 1):
        fs += [face0(0, 1, i), face0(2, 3, i), face1(0, 2, i), face1(1, 3, i)]
        for j in range(0, p - 1):
            fs.append(interior(i, j))
    return fs


def _bary2(node, X):
    return 1 - X[:, 0] - X[:, 1] if node == 0 else X[:, node - 1]


def _bary3(node, X):
    return 1 - X[:, 0] - X[:, 1] - X[:, 2] if node == 0 else X[:, node - 1]


def _triangle_set(p):
    assert p > 0
    fs = []
    for i in range(3):
        fs.append(lambda X, i=i: _bary2(i, X))
    for k in range(0, p - 1):
        for i in range(3):
            for j in range(i):
                # BasisFunction2DFaceTriangle(node0=i, node1=j, k): l0 l1 L_k(l1 - l0)
                fs.append(lambda X, a=i, b=j, k=k: (_bary2(a, X) * _bary2(b, X)
                                                    * lobatto(k, _bary2(b, X) - _bary2(a, X))))
        if k + 3 <= p:
            for j in range(k + 1):
                fs.append(lambda X, k0=k - j, k1=j: (
                    _bary2(0, X) * _bary2(1, X) * _bary2(2, X)
                    * lobatto(k0, _bary2(0, X) - _bary2(1, X))
                    * lobatto(k1, _bary2(1, X) - _bary2(2, X))))
    return fs


def _cube_set(p):
    assert p > 0
    fs = []
    cube = SHAPES["cube"]
    for node in range(8):
        n0 = (node % 2) * 2 - 1
        n1 = ((node // 2) % 2) * 2 - 1
        n2 = (node // 4) * 2 - 1
        fs.append(lambda X, n0=n0, n1=n1, n2=n2: (
            (1 + n0 * X[:, 0]) * (1 + n1 * X[:, 1]) * (1 + n2 * X[:, 2]) / 8.0))

    def edge(axis, node0, node1, k):  # BasisFunction3DEdgeCube_{0,1,2}, Cube.cpp:76-232
        m = 1 if node0 < node1 else -1
        pos = [(node0 % 2) * 2 - 1, ((node0 // 2) % 2) * 2 - 1, (node0 // 4) * 2 - 1]
        others = [a for a in range(3) if a != axis]
        return lambda X: ((1 - X[:, axis]) * (1 + X[:, axis])
                          * (1 + pos[others[0]] * X[:, others[0]])
                          * (1 + pos[others[1]] * X[:, others[1]])
                          * lobatto(k, m * X[:, axis]) / 16.0)

    def face(axis, node0, node1, node2, k_a, k_b):  # BasisFunction3DFaceCube_{0,1,2}, Cube.cpp:234-402
        pos = [(node0 % 2) * 2 - 1, ((node0 // 2) % 2) * 2 - 1, (node0 // 4) * 2 - 1][axis]
        ma = 1 if node0 < node1 else -1
        mb = 1 if node0 < node2 else -1
        a, b = [c for c in range(3) if c != axis]
        return lambda X: ((1 + pos * X[:, axis]) * (1 - X[:, a]) * (1 + X[:, a])
                          * (1 - X[:, b]) * (1 + X[:, b])
                          * lobatto(k_a, ma * X[:, a]) * lobatto(k_b, mb * X[:, b]) / 32.0)

    def interior(k0, k1, k2):  # BasisFunction3DInteriorCube, Cube.cpp:404-432
        return lambda X: ((1 - X[:, 0]) * (1 + X[:, 0]) * (1 - X[:, 1]) * (1 + X[:, 1])
                          * (1 - X[:, 2]) * (1 + X[:, 2]) * lobatto(k0, X[:, 0])
                          * lobatto(k1, X[:, 1]) * lobatto(k2, X[:, 2]) / 64.0)

    def faces(i, j):
        return [face(2, 0, 1, 2, i, j), face(1, 0, 1, 4, i, j), face(0, 0, 2, 4, i, j),
                face(0, 1, 3, 5, i, j), face(1, 2, 3, 6, i, j), face(2, 4, 5, 6, i, j)]

    for j in range(0, p - 1):
        for e in range(12):
            n0, n1 = cube["edges"][e]
            fs.append(edge(e // 4, n0, n1, j))
        fs += faces(j, j)
        fs.append(interior(j, j, j))
        for i in range(j):
            fs += faces(i, j)
            fs += faces(j, i)
            fs += [interior(i, i, j), interior(i, j, i), interior(j, i, i),
                   interior(j, j, i), interior(j, i, j), interior(i, j, j)]
            for k in range(i):
                fs += [interior(i, j, k), interior(i, k, j), interior(j, i, k),
                       interior(j, k, i), interior(k, i, j), interior(k, j, i)]
    return fs


def _tetrahedron_set(p):
    assert p > 0
    fs = []
    tet = SHAPES["tetrahedron"]
    for i in range(4):
        fs.append(lambda X, i=i: _bary3(i, X))
    for j in range(0, p - 1):
        for e in range(6):
            n0, n1 = tet["edges"][e]
            # BasisFunction3DEdgeTetrahedron: l0 l1 L_j(l0 - l1), Tetrahedron.cpp:73-78
            fs.append(lambda X, a=n0, b=n1, k=j: (_bary3(a, X) * _bary3(b, X)
                                                  * lobatto(k, _bary3(a, X) - _bary3(b, X))))
        if j > 0:
            for f in range(4):
                a, b, c = tet["faces"][f]
                for k in range(j):
                    # BasisFunction3DFaceTetrahedron, Tetrahedron.cpp:146-154
                    fs.append(lambda X, a=a, b=b, c=c, k0=j - k - 1, k1=k: (
                        _bary3(a, X) * _bary3(b, X) * _bary3(c, X)
                        * lobatto(k0, _bary3(a, X) - _bary3(b, X))
                        * lobatto(k1, _bary3(b, X) - _bary3(c, X))))
        if j > 1:
            for i in range(j - 1):
                for k in range(j - 1 - i):
                    # BasisFunction3DInteriorTetrahedron(i, j-i-k-2, k), Tetrahedron.cpp:258-267
                    fs.append(lambda X, k0=i, k1=j - i - k - 2, k2=k: (
                        _bary3(0, X) * _bary3(1, X) * _bary3(2, X) * _bary3(3, X)
                        * lobatto(k0, _bary3(0, X) - _bary3(1, X))
                        * lobatto(k1, _bary3(1, X) - _bary3(2, X))
                        * lobatto(k2, _bary3(2, X) - _bary3(3, X))))
    return fs


_SETS = {"line": _line_set, "square": _square_set, "triangle": _triangle_set,
         "cube": _cube_set, "tetrahedron": _tetrahedron_set}


def basis_set(shape, p):
    """List of the basis functions (callables on an (n, dim) point array)."""
    return _SETS[shape](p)


def tabulate(shape, p, points):
    """Values (n, nB) and reference gradients (n, nB, dim) at ``points``."""
    X = np.atleast_2d(np.asarray(points, dtype=float))
    fs = basis_set(shape, p)
    n, d = X.shape
    val = np.empty((n, len(fs)))
    grad = np.empty((n, len(fs), d))
    h = 1e-30
    for j, f in enumerate(fs):
        val[:, j] = np.real(f(X))
        for a in range(d):
            Xc = X.astype(complex)
            Xc[:, a] += 1j * h
            grad[:, j, a] = np.imag(f(Xc)) / h
    return val, grad
