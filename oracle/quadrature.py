"""Gauss quadrature rules as hpGEM selects them (test infrastructure only).

Rule choice restates AllGaussQuadratureRules::getRule
(kernel/Integration/QuadratureRules/AllGaussQuadratureRules.cpp:138-158): the
first registered rule, in order of increasing order, whose order is at least
the requested one.  The registry is AllGaussQuadratureRules.cpp:58-117.

* line / square / cube: tensor-product Gauss-Legendre rules with n = 1..6
  points per direction (orders 1, 3, ..., 11).  Point order follows the
  reference: x fastest on the square (GaussQuadratureRulesForSquare.cpp:152-182),
  z fastest on the cube (GaussQuadratureRulesForCube.cpp:282-304).  Nodes and
  weights come from numpy's Gauss-Legendre routine; they agree with the
  reference's closed forms and decimal tables to rounding.
* triangle / tetrahedron: the published tables hpGEM carries
  (GaussQuadratureRulesFor{Triangle,Tetrahedron}.cpp), read from the golden
  fixture ``tests/golden/simplex_rules.json`` that tests/golden/make_golden.py
  extracts from the reference.
"""
import json
import os

import numpy as np

_GOLDEN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "tests", "golden", "simplex_rules.json")

TRIANGLE_REGISTRY = ["Tn2_1_1", "Tn2_2_3", "Tn2_4_6", "T2_5_7", "T2_6_12", "T2_8_16",
                     "T2_9_19", "T2_10_25", "T2_11_28"]
TETRAHEDRON_REGISTRY = ["Tn3_1_1", "Tn3_2_4", "Tn3_3_10", "Tn3_4_14", "T3_5_14", "T3_6_24",
                        "T3_7_31", "T3_8_43", "T3_9_53", "T3_10_126"]

_simplex_cache = None


def _simplex_tables():
    global _simplex_cache
    if _simplex_cache is None:
        with open(_GOLDEN) as f:
            _simplex_cache = json.load(f)
    return _simplex_cache


class Rule:
    def __init__(self, name, order, points, weights):
        self.name = name
        self.order = order
        self.points = np.asarray(points, dtype=float)
        self.weights = np.asarray(weights, dtype=float)

    def __len__(self):
        return len(self.weights)


def gauss_line(n):
    x, w = np.polynomial.legendre.leggauss(n)
    return x, w


def _tensor_rule(shape, n):
    x, w = gauss_line(n)
    if shape == "point":
        return Rule("Cn0_inf_1", 10 ** 9, np.zeros((1, 0)), [1.0])
    if shape == "line":
        return Rule("C1_%d" % n, 2 * n - 1, x[:, None], w)
    if shape == "square":
        pts = [[x[i], x[j]] for j in range(n) for i in range(n)]
        wts = [w[i] * w[j] for j in range(n) for i in range(n)]
        return Rule("C2_%d" % n, 2 * n - 1, pts, wts)
    if shape == "cube":
        pts = [[x[i], x[j], x[k]] for i in range(n) for j in range(n) for k in range(n)]
        wts = [w[i] * w[j] * w[k] for i in range(n) for j in range(n) for k in range(n)]
        return Rule("C3_%d" % n, 2 * n - 1, pts, wts)
    raise KeyError(shape)


def registry(shape):
    """All rules of hpGEM's registry for ``shape``, sorted as getRule scans them."""
    if shape == "point":
        return [_tensor_rule("point", 1)]
    if shape in ("line", "square", "cube"):
        return [_tensor_rule(shape, n) for n in range(1, 7)]
    tables = _simplex_tables()[shape]
    names = TRIANGLE_REGISTRY if shape == "triangle" else TETRAHEDRON_REGISTRY
    rules = []
    for name in names:  # AllGaussQuadratureRules::addRule keeps them sorted by order
        t = tables[name]
        r = Rule(name, t["order"], t["points"], t["weights"])
        pos = 0
        while pos < len(rules) and rules[pos].order < r.order:
            pos += 1
        rules.insert(pos, r)
    return rules


def rule_by_name(shape, name):
    for r in registry(shape):
        if r.name == name:
            return r
    raise KeyError(name)


def get_rule(shape, order):
    """AllGaussQuadratureRules::getRule (AllGaussQuadratureRules.cpp:138-158)."""
    for r in registry(shape):
        if r.order >= order:
            return r
    raise ValueError("No quadrature rule found for %s and order %d" % (shape, order))
