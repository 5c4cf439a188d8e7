"""Structured meshes of hpGEM's Preprocessor (test infrastructure only).

``structured_mesh`` restates ``StructuredReader`` of
applications/Preprocessor/lib/hpgem.cpp:55-265: the node numbering with x
fastest (getNodeCoordinates, :100-137), the extra coordinates that periodic
nodes carry (:116-125), the element vertex lists with periodic wrap-around
(:159-181) and the 2-triangle / 5-tetrahedron split with its alternating
rotation (:139-158, :182-221).  hpGEM's mesh reader keeps the element and
vertex order of the file (kernel/Base/MeshManipulator_Impl.h:1641-1680).

``build_faces`` pairs element faces by their sets of global node numbers, the
way hpGEM's mesh reader couples elements through shared nodes; periodic
copies of a node share its number, so periodic faces pair up like interior
ones.  Faces are numbered in order of first appearance; the first element
that owns a face is its left element.
"""
import numpy as np

from .refgeom import SHAPES


def parse_description(text):
    """Parse a ``structured 1 <dim>`` description (applications/Preprocessor/README.md)."""
    toks = text.split()
    assert toks[0] == "structured" and toks[1] == "1", "not a structured description"
    dim = int(toks[2])
    k = 3
    n = [int(t) for t in toks[k:k + dim]]; k += dim
    lower = [float(t) for t in toks[k:k + dim]]; k += dim
    upper = [float(t) for t in toks[k:k + dim]]; k += dim
    kind = toks[k]; k += 1
    assert kind in ("triangular", "rectangular"), kind
    periodic = [t == "true" for t in toks[k:k + dim]]
    return dict(n=n, lower=lower, upper=upper, triangular=kind == "triangular",
                periodic=periodic)


class Mesh:
    """Elements as vertex lists (node ids + physical coordinates) plus a face table."""

    def __init__(self, shape, element_nodes, element_coords):
        self.shape = shape
        self.dim = SHAPES[shape]["dim"]
        self.element_nodes = np.asarray(element_nodes, dtype=np.int64)
        self.element_coords = np.asarray(element_coords, dtype=float)
        self.faces = build_faces(shape, self.element_nodes)

    @property
    def n_elements(self):
        return len(self.element_nodes)


def structured_mesh(n, lower, upper, triangular, periodic):
    """Restatement of StructuredReader (applications/Preprocessor/lib/hpgem.cpp:55-265)."""
    dim = len(n)
    n_elem = list(n)
    n_nodes = [n_elem[i] + (0 if periodic[i] else 1) for i in range(dim)]
    size = [upper[i] - lower[i] for i in range(dim)]  # hpgem.cpp:87-89

    # getNodeCoordinates, hpgem.cpp:100-137: each node lists its coordinates;
    # a node with index 0 in a periodic direction also carries the copy shifted
    # by the period (doubling the list once per such direction).
    total_nodes = int(np.prod(n_nodes))
    node_coords = []
    idx = [0] * dim
    for _ in range(total_nodes):
        coords = [[lower[i] + idx[i] * size[i] / n_elem[i] for i in range(dim)]]
        for i in range(dim):
            if periodic[i] and idx[i] == 0:
                for c in list(coords):
                    c2 = list(c)
                    c2[i] += size[i]
                    coords.append(c2)
        node_coords.append(coords)
        for i in range(dim):
            idx[i] += 1
            if idx[i] < n_nodes[i]:
                break
            idx[i] = 0

    # getElements, hpgem.cpp:139-265
    rotate = [2, 0, 3, 1, 6, 4, 7, 5]
    if dim == 2:
        corners = [[0, 1, 2], [1, 3, 2]]
    elif dim == 3:
        corners = [[1, 2, 4, 7], [0, 1, 2, 4], [1, 3, 2, 7], [1, 4, 5, 7], [2, 6, 4, 7]]
    else:
        assert not triangular, "no simplices in this dimension"
        corners = []
    if not triangular:
        corners_used = None
    mult = [1]
    for i in range(1, dim):
        mult.append(mult[-1] * n_nodes[i - 1])

    elem_nodes, elem_coords = [], []
    loop = [0] * dim
    tri_index = 0
    total_cells = int(np.prod(n_elem))
    n_out = total_cells * (len(corners) if triangular else 1)
    for _ in range(n_out):
        ids = [0]
        for i in range(dim):
            cur = len(ids)
            for j in range(cur):
                ids[j] += loop[i] * mult[i]
                ids.append(ids[j] + mult[i])
        verts = []
        for j in range(len(ids)):
            sub = 0
            prev_periodic = 0
            node = ids[j]
            for i in range(dim):
                bit = (j >> i) & 1
                if bit and loop[i] == n_nodes[i] - 1:
                    node -= n_nodes[i] * mult[i]
                    sub += 1 << prev_periodic
                    prev_periodic += 1
                if periodic[i] and loop[i] + (j & (1 << i)) == 0:
                    prev_periodic += 1
            verts.append((node, node_coords[node][sub]))
        if triangular:
            pattern = corners[tri_index]
            verts = [verts[c] for c in pattern]
            tri_index += 1
            if tri_index == len(corners):
                tri_index = 0
        elem_nodes.append([v[0] for v in verts])
        elem_coords.append([v[1] for v in verts])
        if tri_index == 0:
            for i in range(dim):
                corners = [[rotate[k] for k in c] for c in corners]
                loop[i] += 1
                if loop[i] < n_elem[i]:
                    break
                if loop[i] % 2 == 1:
                    corners = [[rotate[k] for k in c] for c in corners]
                loop[i] = 0
    shape = {1: "line", 2: "triangle" if triangular else "square",
             3: "tetrahedron" if triangular else "cube"}[dim]
    return Mesh(shape, elem_nodes, elem_coords)


def mesh_from_description(text):
    d = parse_description(text)
    return structured_mesh(d["n"], d["lower"], d["upper"], d["triangular"], d["periodic"])


def build_faces(shape, element_nodes):
    """Face table: rows (left element, right element or -1, left local face,
    right local face or -1, k) plus, per face, the right-side vertex
    correspondence ``perm`` (for left-face vertex i, the index in the right
    element's local face vertex list holding the same global node)."""
    fl = SHAPES[shape]["faces"]
    seen = {}
    rows, perms = [], []
    for e, nodes in enumerate(element_nodes):
        for f, loc in enumerate(fl):
            gids = tuple(int(nodes[v]) for v in loc)
            key = tuple(sorted(gids))
            if key in seen:
                fid = seen.pop(key)
                lrow = rows[fid]
                assert lrow[1] == -1, "face shared by more than two elements"
                left_gids = [int(element_nodes[lrow[0]][v]) for v in fl[lrow[2]]]
                perm = [gids.index(g) for g in left_gids]
                rows[fid] = [lrow[0], e, lrow[2], f]
                perms[fid] = perm
            else:
                seen[key] = len(rows)
                rows.append([e, -1, f, -1])
                perms.append(None)
    return {"table": np.asarray(rows, dtype=np.int64), "perm": perms}
