"""Regenerate the golden fixtures in this folder from the hpGEM reference tree.

This script is the only committed code that reads the reference checkout.  It
is run by hand (``python tests/golden/make_golden.py /path/to/hpgem``) on a
machine that has the reference; its JSON output is committed so that the tests
need nothing but this repository.  What it extracts, and from where:

* ``meshes.json``: element connectivity and vertex coordinates of the small
  structured meshes under ``tests/files/*.hpgem`` (written by hpGEM's
  Preprocessor from ``tests/files/sources/*.hpgem``), parsed from the
  "mesh 2" text format read by ``MeshManipulator::readMesh``
  (``kernel/Base/MeshManipulator_Impl.h:1505-``).
* ``simplex_rules.json``: points and weights of the triangle and tetrahedron
  Gauss rules (``kernel/Integration/QuadratureRules/
  GaussQuadratureRulesFor{Triangle,Tetrahedron}.cpp``).  These are published
  tables (Dunavant; Keast) that hpGEM transcribes; parity of the initial L2
  projection needs the very same points.
* ``quadrature_integrals.json``: the known-answer checks of the quadrature
  unit tests (``tests/unit/Integration/QuadratureRules/0[2-6]0*.cpp``): the
  integral of every default H1 basis function of a given order over the
  reference shape, as an if/else chain on the basis-function index.
* ``advection_goldens.json``: the L2-error tables of
  ``tests/self/Basic/090Advection_SelfTest.cpp:303-337``.
* ``advection_linear_goldens.json``: the L2-error tables of the stored-matrix
  self-test ``tests/self/Basic/080AdvectionLinear_SelfTest.cpp:255-297``
  (non-periodic meshes, inflow boundary through the boundary source term), with
  the mesh file names of ``tests/self/TestMeshes.h`` behind each table.
* ``mesh_files/*.hpgem``: three of those Preprocessor outputs as they are
  (the fully periodic 1D line, 2D triangle and 3D cube meshes), for the tests
  of the library's "mesh 2" reader; their structured descriptions are in
  ``meshes.json``.
"""
import json
import math
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _tokens(path):
    with open(path) as f:
        return f.read().split()


def parse_mesh2(path):
    """Parse a "mesh 2" file into node coordinate lists and element lists.

    Returns ``{"dim", "nodes": [[coords...], ...], "elements": [[(node, coord_index)...]]}``.
    Layout (written by the Preprocessor, read by MeshManipulator::readMesh):
    header ``mesh 2``; ``nNodes nElements dim [nFaces [nEdges]]``; a partition
    line; ``zones`` + count + names; ``nodes`` then per node a partition line
    and ``k x_1 ... x_{k*dim}``; ``elements`` then per element
    ``n node_1 off_1 ... node_n off_n zone ...`` followed by a shadow line.
    """
    with open(path) as f:
        lines = [ln.strip() for ln in f.read().splitlines()]
    assert lines[0] == "mesh 2", path
    head = [int(t) for t in lines[1].split()]
    n_nodes, n_elem, dim = head[0], head[1], head[2]
    i = 2
    while lines[i] != "zones":
        i += 1
    n_zones = int(lines[i + 1])
    i = i + 2 + n_zones
    assert lines[i] == "nodes", (path, lines[i])
    i += 1
    nodes = []
    for _ in range(n_nodes):
        i += 1  # partition line
        toks = lines[i].split()
        k = int(toks[0])
        vals = [float.fromhex(t) for t in toks[1:]]
        assert len(vals) == k * dim
        nodes.append([vals[j * dim:(j + 1) * dim] for j in range(k)])
        i += 1
    assert lines[i] == "elements", (path, lines[i])
    i += 1
    elements = []
    for _ in range(n_elem):
        toks = [int(t) for t in lines[i].split()]
        n = toks[0]
        pairs = [(toks[1 + 2 * j], toks[2 + 2 * j]) for j in range(n)]
        elements.append(pairs)
        i += 2  # element line + shadow line
    return {"dim": dim, "nodes": nodes, "elements": elements}


def parse_source(path):
    toks = open(path).read().split()
    assert toks[0] == "structured" and toks[1] == "1"
    dim = int(toks[2])
    k = 3
    n = [int(t) for t in toks[k:k + dim]]; k += dim
    lo = [float(t) for t in toks[k:k + dim]]; k += dim
    hi = [float(t) for t in toks[k:k + dim]]; k += dim
    kind = toks[k]; k += 1
    per = [t == "true" for t in toks[k:k + dim]]
    return {"dim": dim, "n": n, "lower": lo, "upper": hi,
            "triangular": kind == "triangular", "periodic": per}


MESHES = [
    ("unitLineN4Per", "unitLineN4Per.hpgem", "unitLineN4Per.hpgem"),
    ("unitSquareN1", "unitSquareN1.hpgem", None),
    ("2Drectangular1", "2Drectangular1mesh.hpgem", "2Drectangular1source.hpgem"),
    ("2Dtriangular1", "2Dtriangular1mesh.hpgem", "2Dtriangular1source.hpgem"),
    ("unitSquareTrianglesN4Per", "unitSquareTrianglesN4Per.hpgem",
     "unitSquareTrianglesN4Per.hpgem"),
    ("unitSquareTrianglesN4", "unitSquareTrianglesN4.hpgem", None),
    ("3Drectangular1", "3Drectangular1mesh.hpgem", "3Drectangular1source.hpgem"),
    ("unitCubeN4Per", "unitCubeN4Per.hpgem", "unitCubeN4Per.hpgem"),
    ("unitCubeN2Tet", "unitCubeN2Tet.hpgem", "unitCubeN2Tet.hpgem"),
    ("3Dtriangular1", "3Dtriangular1mesh.hpgem", "3Dtriangular1source.hpgem"),
    ("3Dtriangular2", "3Dtriangular2mesh.hpgem", "3Dtriangular2source.hpgem"),
    # non-periodic meshes of the stored-matrix self-test (080AdvectionLinear_SelfTest)
    ("unitLineN4", "unitLineN4.hpgem", "unitLineN4.hpgem"),
    ("unitSquareTrianglesN2", "unitSquareTrianglesN2.hpgem", "unitSquareTrianglesN2.hpgem"),
    ("unitCubeN4", "unitCubeN4.hpgem", "unitCubeN4.hpgem"),
]


# Preprocessor outputs kept as files for the mesh reader's tests (fully periodic)
MESH_FILES = ["unitLineN4Per.hpgem", "unitSquareTrianglesN4Per.hpgem", "unitCubeN4Per.hpgem"]


def extract_meshes(ref):
    out = {}
    for name, mesh_file, src_file in MESHES:
        files = os.path.join(ref, "tests", "files")
        src_path = os.path.join(files, "sources", src_file or mesh_file)
        if not os.path.exists(src_path):
            continue
        src = parse_source(src_path)
        m = parse_mesh2(os.path.join(files, mesh_file))
        elems = []
        coords = []
        for el in m["elements"]:
            elems.append([nd for nd, _ in el])
            coords.append([m["nodes"][nd][off] for nd, off in el])
        out[name] = {"source": src, "element_nodes": elems,
                     "element_coords": coords}
    return out


def extract_rules(ref):
    out = {}
    qdir = os.path.join(ref, "kernel", "Integration", "QuadratureRules")
    for fname, shape in (("GaussQuadratureRulesForTriangle.cpp", "triangle"),
                         ("GaussQuadratureRulesForTetrahedron.cpp", "tetrahedron")):
        text = open(os.path.join(qdir, fname)).read()
        # constructors: "Name::Name()" ... until the closing "}\n\n"
        tv = re.search(r"const double TET_VOLUME\s*=\s*([0-9.eE+-]+);", text)
        tet_volume = float(tv.group(1)) if tv else None
        # rules written as StandardGaussQuadratureRule(name, order, geo, {{w * TET_VOLUME, {x, y, z}}, ...})
        for m in re.finditer(r"\n(\w+)::\1\(\)\s*:\s*StandardGaussQuadratureRule(?:<3>)?\(\s*"
                             r"\"[^\"]*\",\s*(\d+),(.*?)\}\)\s*\{\}", text, re.S):
            cls, order, body = m.group(1), int(m.group(2)), m.group(3)
            pts, w = [], []
            for pm in re.finditer(r"\{\s*([0-9.eE+-]+)\s*\*\s*TET_VOLUME\s*,\s*\{([^}]*)\}\s*\}", body):
                w.append(float(pm.group(1)) * tet_volume)
                pts.append([float(t) for t in pm.group(2).split(",")])
            out.setdefault(shape, {})[cls] = {"order": order, "points": pts, "weights": w}
        for m in re.finditer(r"\n(\w+)::\1\(\)(.*?)\n}\n", text, re.S):
            cls, body = m.group(1), m.group(2)
            om = re.search(r"std::size_t %s::order\(\) const \{\s*return (\d+);" % cls, text)
            if om is None:
                continue
            order = int(om.group(1))
            weights = {}
            for wm in re.finditer(r"weight_\[(\d+)\]\s*=\s*([^;]+);", body):
                weights[int(wm.group(1))] = float(eval(" ".join(wm.group(2).split())))
            pts = []
            for pm in re.finditer(r"gp_\.push_back\(\s*\{([^}]*)\}\s*\)", body):
                pts.append([float(eval(" ".join(t.split()))) for t in pm.group(1).split(",")])
            if not pts:
                continue
            w = [weights[i] for i in range(len(pts))]
            out.setdefault(shape, {})[cls] = {"order": order, "points": pts,
                                             "weights": w}
    return out


def _cxx_expr_to_py(s):
    s = s.replace("std::sqrt", "math.sqrt").replace("&&", " and ").replace("||", " or ")
    return s


def _balanced(text, i):
    """Return (inner, end) of the parenthesised group starting at text[i] == '('."""
    assert text[i] == "("
    depth = 0
    for j in range(i, len(text)):
        if text[j] == "(":
            depth += 1
        elif text[j] == ")":
            depth -= 1
            if depth == 0:
                return text[i + 1:j], j + 1
    raise ValueError("unbalanced")


def extract_integrals(ref):
    qdir = os.path.join(ref, "tests", "unit", "Integration", "QuadratureRules")
    files = {"line": "020GaussQuadratureRulesForLine_UnitTest.cpp",
             "square": "030GaussQuadratureRulesForSquare_UnitTest.cpp",
             "triangle": "040GaussQuadratureRulesForTriangle_UnitTest.cpp",
             "cube": "050GaussQuadratureRuleForCube_UnitTest.cpp",
             "tetrahedron": "060GaussQuadratureRuleForTetrahedron_UnitTest.cpp"}
    out = {}
    for shape, fname in files.items():
        text = open(os.path.join(qdir, fname)).read()
        body = text[text.index("functions->eval(i, point);"):]
        body = body[:body.index("delete functions")]
        chain = []
        pos = 0
        while True:
            m = re.compile(r"(else\s+if|if|else)\s*(\(|\{)").search(body, pos)
            if m is None:
                break
            if m.group(2) == "(":
                cond, after = _balanced(body, m.end() - 1)
                cond = " ".join(cond.split())
            else:
                cond, after = "True", m.end() - 1
            c = body.index("CHECK", after)
            check, pos = _balanced(body, body.index("(", c))
            check = " ".join(check.split()).strip()
            while check.startswith("(") and _balanced(check, 0)[1] == len(check):
                check = check[1:-1].strip()
            a = check.index("std::abs")
            absarg, _ = _balanced(check, check.index("(", a))
            rest = absarg.replace("integrated", "", 1).strip()
            if rest == "":
                expected = 0.0
            else:
                v = float(eval(_cxx_expr_to_py(rest[1:]), {"math": math}))
                expected = v if rest[0] == "-" else -v
            chain.append([_cxx_expr_to_py(cond), expected])
        calls = [[c, int(o)] for c, o in
                 re.findall(r"^\s*testRule\(QuadratureRules::(\w+)::Instance\(\),\s*(\d+)\);",
                            text, re.M)]
        out[shape] = {"rules": calls, "chain": chain}
    return out


def extract_advection_goldens(ref):
    text = open(os.path.join(ref, "tests", "self", "Basic",
                             "090Advection_SelfTest.cpp")).read()
    out = {}
    for dim, key in ((1, "dim1Meshes"), (2, "dim2P1Meshes"), (3, "dim3Meshes")):
        m = re.search(key + r"\s*=\s*\{(\w+)\(([^)]*)\),\s*\{(.*?)\}\}", text, re.S)
        vals = [float(v) for v in re.findall(r"([0-9.]+e[-+]\d+)", m.group(3))]
        out[str(dim)] = {"mesh_list": m.group(1), "min_level": m.group(2) or None,
                         "errors": vals}
    for dim, key in ((1, "dim1Params"), (2, "dim2P1Params"), (3, "dim3Params")):
        m = re.search(r"AdvectionParameters\s+" + key + r"\s*=\s*\{([^}]*)\}", text)
        p, t_end, steps = [t.strip() for t in m.group(1).split(",")]
        out[str(dim)].update({"p": int(p), "end_time": float(t_end),
                              "time_steps": int(steps)})
    return out


def extract_linear_advection_goldens(ref):
    """The L2-error tables of 080AdvectionLinear_SelfTest.cpp:255-297 with their
    mesh lists (TestMeshes.h) and parameters (p, end time, time steps)."""
    text = open(os.path.join(ref, "tests", "self", "Basic",
                             "080AdvectionLinear_SelfTest.cpp")).read()
    out = {}
    for key in ("dim1", "dim2P1", "dim2P2", "dim3"):
        m = re.search(key + r"Meshes\s*=\s*\{(\w+)\(([^)]*)\),\s*\{(.*?)\}\}", text, re.S)
        vals = [float(v) for v in re.findall(r"([0-9.]+e[-+]\d+)", m.group(3))]
        levels = [int(t) for t in m.group(2).split(",")] if m.group(2).strip() else []
        out[key] = {"mesh_list": m.group(1), "levels": levels, "errors": vals}
        m = re.search(r"AdvectionParameters\s+" + key + r"Params\s*=\s*\{([^}]*)\}", text)
        p, t_end, steps = [t.strip() for t in m.group(1).split(",")]
        out[key].update({"p": int(p), "end_time": float(t_end), "time_steps": int(steps)})
    # the file names behind each mesh list, in level order
    meshes = open(os.path.join(ref, "tests", "self", "TestMeshes.h")).read()
    for blob in out.values():
        m = re.search(r"std::vector<std::string> " + blob["mesh_list"] + r"\(.*?limit\((.*?)minLevel", meshes, re.S)
        blob["files"] = re.findall(r'"(\w+)\.hpgem"', m.group(1))
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <hpgem source tree>")
    ref = sys.argv[1]
    blobs = {
        "meshes.json": extract_meshes(ref),
        "simplex_rules.json": extract_rules(ref),
        "quadrature_integrals.json": extract_integrals(ref),
        "advection_goldens.json": extract_advection_goldens(ref),
        "advection_linear_goldens.json": extract_linear_advection_goldens(ref),
    }
    for name, blob in blobs.items():
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(blob, f, separators=(",", ":"))
        print(name, os.path.getsize(os.path.join(HERE, name)), "bytes")
    os.makedirs(os.path.join(HERE, "mesh_files"), exist_ok=True)
    for fname in MESH_FILES:
        dst = os.path.join(HERE, "mesh_files", fname)
        with open(os.path.join(ref, "tests", "files", fname)) as fi, open(dst, "w") as fo:
            fo.write(fi.read())
        print(os.path.join("mesh_files", fname), os.path.getsize(dst), "bytes")


if __name__ == "__main__":
    main()
