"""Reference shapes of hpGEM (test infrastructure only; see oracle/__init__.py).

Vertex coordinates and the local vertex lists of faces (codim-1 entities)
and edges, as defined by hpGEM:
  line        kernel/Geometry/ReferenceLine.cpp:54-61
  square      kernel/Geometry/ReferenceSquare.cpp:60-107
  triangle    kernel/Geometry/ReferenceTriangle.cpp:59-60 (vertices (0,0),(1,0),(0,1))
  cube        kernel/Geometry/ReferenceCube.cpp:52-74
  tetrahedron kernel/Geometry/ReferenceTetrahedron.cpp:56-60
The face reference shape of each element is the shape of one dimension less
(cube -> square, square -> line, tetrahedron -> triangle, triangle -> line,
line -> point).
"""
import numpy as np

SHAPES = {
    "point": dict(dim=0, vertices=np.zeros((1, 0)), faces=[], edges=[], face_shape=None,
                  measure=1.0),
    "line": dict(dim=1, vertices=np.array([[-1.0], [1.0]]), faces=[[0], [1]], edges=[],
                 face_shape="point", measure=2.0),
    "square": dict(dim=2, vertices=np.array([[-1.0, -1.0], [1.0, -1.0], [-1.0, 1.0], [1.0, 1.0]]),
                   faces=[[0, 1], [0, 2], [1, 3], [2, 3]], edges=[], face_shape="line",
                   measure=4.0),
    "triangle": dict(dim=2, vertices=np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]),
                     faces=[[0, 1], [0, 2], [1, 2]], edges=[], face_shape="line",
                     measure=0.5),
    "cube": dict(dim=3, vertices=np.array([[-1.0, -1.0, -1.0], [1.0, -1.0, -1.0],
                                           [-1.0, 1.0, -1.0], [1.0, 1.0, -1.0],
                                           [-1.0, -1.0, 1.0], [1.0, -1.0, 1.0],
                                           [-1.0, 1.0, 1.0], [1.0, 1.0, 1.0]]),
                 faces=[[0, 1, 2, 3], [0, 1, 4, 5], [0, 2, 4, 6],
                        [1, 3, 5, 7], [2, 3, 6, 7], [4, 5, 6, 7]],
                 edges=[[0, 1], [2, 3], [4, 5], [6, 7], [0, 2], [1, 3],
                        [4, 6], [5, 7], [0, 4], [1, 5], [2, 6], [3, 7]],
                 face_shape="square", measure=8.0),
    "tetrahedron": dict(dim=3, vertices=np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0],
                                                  [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]),
                        faces=[[0, 3, 2], [0, 1, 3], [0, 2, 1], [1, 2, 3]],
                        edges=[[0, 1], [0, 2], [0, 3], [2, 3], [1, 3], [1, 2]],
                        face_shape="triangle", measure=1.0 / 6.0),
}

HYPERCUBES = ("line", "square", "cube")


def vertex_shape_functions(shape, xi):
    """Shape functions N_k(xi) of the vertices of ``shape`` at points xi (n, dim).

    Linear (barycentric) on simplices, multilinear on hypercubes; they define the
    vertex-based maps used for reference-to-physical maps
    (kernel/Geometry/Mappings/MappingToPhysSimplexLinear_Impl.h:51-64,
    MappingToPhysHypercubeLinear.cpp) and for face-to-element maps.
    """
    xi = np.atleast_2d(np.asarray(xi))
    n = xi.shape[0]
    if shape == "point":
        return np.ones((n, 1))
    if shape in HYPERCUBES:
        d = SHAPES[shape]["dim"]
        out = np.ones((n, 2 ** d), dtype=xi.dtype)
        for k in range(2 ** d):
            for i in range(d):
                s = 1.0 if (k >> i) & 1 else -1.0
                out[:, k] = out[:, k] * (1.0 + s * xi[:, i]) / 2.0
        return out
    d = SHAPES[shape]["dim"]
    out = np.empty((n, d + 1), dtype=xi.dtype)
    out[:, 0] = 1.0 - xi.sum(axis=1)
    out[:, 1:] = xi
    return out
