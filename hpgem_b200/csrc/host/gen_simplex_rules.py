"""Writes simplex_rules.inc: the triangle and tetrahedron Gauss rules as C arrays.

These rules are published tables (Dunavant for triangles, Keast and others
for tetrahedra) that hpGEM carries in
kernel/Integration/QuadratureRules/GaussQuadratureRulesFor{Triangle,Tetrahedron}.cpp.
The initial L2 projection and the error norms only agree with hpGEM's if the
very same points are used, so the values are taken over unchanged from the
extracted fixture tests/golden/simplex_rules.json (see tests/golden/make_golden.py).
Run: python hpgem_b200/csrc/host/gen_simplex_rules.py
"""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))

# registry order of kernel/Integration/QuadratureRules/AllGaussQuadratureRules.cpp:72-101
REGISTRY = {"triangle": ["Tn2_1_1", "Tn2_2_3", "Tn2_4_6", "T2_5_7", "T2_6_12", "T2_8_16",
                         "T2_9_19", "T2_10_25", "T2_11_28"],
            "tetrahedron": ["Tn3_1_1", "Tn3_2_4", "Tn3_3_10", "Tn3_4_14", "T3_5_14", "T3_6_24",
                            "T3_7_31", "T3_8_43", "T3_9_53", "T3_10_126"]}


def main():
    with open(os.path.join(ROOT, "tests", "golden", "simplex_rules.json")) as f:
        tables = json.load(f)
    lines = ["// Generated by gen_simplex_rules.py; do not edit.",
             "// {name, shape (3 = triangle, 5 = tetrahedron), order, n_points, offset into kSimplexData}",
             "// kSimplexData holds, per point, the weight followed by the coordinates."]
    data = []
    entries = []
    for shape, code in (("triangle", 3), ("tetrahedron", 5)):
        for name in REGISTRY[shape]:
            t = tables[shape][name]
            entries.append('{"%s", %d, %d, %d, %d}' % (name, code, t["order"], len(t["weights"]),
                                                       len(data)))
            for w, pt in zip(t["weights"], t["points"]):
                data.append(w)
                data.extend(pt)
    lines.append("static const SimplexRuleEntry kSimplexRules[] = {")
    lines += ["    %s," % e for e in entries]
    lines.append("};")
    lines.append("static const double kSimplexData[] = {")
    for i in range(0, len(data), 4):
        lines.append("    " + ", ".join("%.17g" % v for v in data[i:i + 4]) + ",")
    lines.append("};")
    with open(os.path.join(HERE, "simplex_rules.inc"), "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
