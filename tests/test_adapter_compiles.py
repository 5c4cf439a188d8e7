"""CPU: the hpGEM-side adapter (include/hpgem_b200_simplified.hpp, the subclass a
maintainer adds to an hpGEM application) compiles against the reference's own
kernel headers: g++ -fsyntax-only with both dimensions instantiated, so every
hpGEM call it makes (mesh lists, quadrature rules, basis tabulation, face maps,
normals, Butcher tableau, time-integration vectors) names a real member with the
types used.  Skipped where the reference sources or g++ are absent."""
import os
import shutil
import subprocess

import pytest

from oracle.reference_tree import kernel_include_dir

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def _compile(source, tmp_path):
    kernel = kernel_include_dir()
    if kernel is None or shutil.which("g++") is None:
        pytest.skip("reference headers or g++ not available")
    src = tmp_path / "use_adapter.cpp"
    src.write_text(source)
    return subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", kernel, "-I", INCLUDE, str(src)],
                          capture_output=True, text=True, timeout=300)


def test_gpu_simplified_compiles_against_hpgem_headers(tmp_path):
    r = _compile('#include "hpgem_b200_simplified.hpp"\n'
                 "template class hpgem_b200::GpuSimplified<2>;\n"
                 "template class hpgem_b200::GpuSimplified<3>;\n", tmp_path)
    assert r.returncode == 0, r.stderr[-4000:]


def test_the_check_catches_a_wrong_member(tmp_path):
    # the same compile with a member hpGEM does not have fails: the check is real
    r = _compile('#include "hpgem_b200_simplified.hpp"\n'
                 "template class hpgem_b200::GpuSimplified<2>;\n"
                 "int f(hpgem_b200::GpuSimplified<2> *p) { return p->no_such_member_; }\n", tmp_path)
    assert r.returncode != 0 and "no_such_member_" in r.stderr
