"""The C++ drop-in (taichi_collisional_b200/host/tc_force_shim.hpp) compiles against the
reference's own Body/Bodies types and globals (exafmm.h) and links against the C ABI."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
import oracle  # noqa: E402

REF = oracle.reference_dir() or ""

PROGRAM = r"""
#include <cmath>
#include <cstring>
#include <list>
#include "exafmm.h"
#include "taichi_collisional_b200/host/tc_force_shim.hpp"
int main(int argc, char**) {
  exafmm::P = EXPANSION;
  exafmm::bodies.resize(3);
  if (argc > 5) exafmm::get_force_and_potential(exafmm::bodies, false);
  if (argc > 6) exafmm::get_force_and_potential(exafmm::bodies, true);
  return 0;
}
"""


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "exafmm.h")), reason="reference tree not present")
@pytest.mark.parametrize("tree,defs", [("", []), ("", ["-DTC_SHIM_ERROR_MAC"]),
                                       ("taichi_with_jerks", ["-DTC_SHIM_JERKS"]),
                                       ("taichi_with_jerks", ["-DTC_SHIM_JERKS", "-DTC_SHIM_THETA"])])
def test_shim_compiles_and_links_against_reference_types(tmp_path, tree, defs):
    src = tmp_path / "shim_main.cpp"
    src.write_text(PROGRAM)
    inc = os.path.join(REF, tree) if tree else REF
    cmd = ["g++", "-std=gnu++14", "-DEXPANSION=8", "-DHUGE=HUGE_VAL", *defs, "-I", inc, "-I", ROOT, str(src), "-o",
           str(tmp_path / "shim"), "-L", os.path.join(ROOT, "taichi_collisional_b200"), "-ltaichi_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "taichi_collisional_b200")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
