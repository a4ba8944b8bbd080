"""The builder's CTA composition (csrc/tile_order.h: group_of_slot) on the CPU.

Each builder warp takes a group of consecutive cells; its group index is also
its emission tile, which the scan and the assembly use to put the model's rows
in canonical CSR order.  The mapping from a CTA's warp slots to groups must
therefore be a bijection on every layer's slots (padding slots included), or
rows would be lost or written twice.  The header is compiled here with the host
compiler and checked for every grid side up to 300 and every cells-per-warp,
and for the edge-first order it promises.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "e2e_gpu_dp_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <vector>
#include "tile_order.h"

using e2e::group_of_slot;
using e2e::kEdgeBand;

static bool edge_group(int64_t grp, int g, int cpw) {
  for (int t = 0; t < cpw; ++t) {
    const int64_t c = grp * cpw + t;
    const int i = (int)(c / g), j = (int)(c % g);
    if (i < kEdgeBand || i >= g - kEdgeBand || j < kEdgeBand || j >= g - kEdgeBand) return true;
  }
  return false;
}

int main() {
  long checked = 0, reordered = 0;
  for (int cpw = 1; cpw <= 32; cpw *= 2) {
    for (int g = 1; g <= 300; ++g) {
      const int64_t nc = (int64_t)g * g;
      const int64_t tiles = (nc + 31) / 32, nslots = tiles * (32 / cpw);
      std::vector<char> seen((size_t)nslots, 0);
      std::vector<int64_t> order((size_t)nslots);
      bool identity = true;
      for (int64_t s = 0; s < nslots; ++s) {
        const int64_t grp = group_of_slot(s, g, cpw);
        if (grp < 0 || grp >= nslots || seen[(size_t)grp]) {
          std::printf("FAIL not a bijection: g=%d cpw=%d slot=%lld group=%lld\n", g, cpw, (long long)s,
                      (long long)grp);
          return 1;
        }
        seen[(size_t)grp] = 1;
        order[(size_t)s] = grp;
        identity = identity && grp == s;
      }
      if (!identity) {  // every edge group before every interior group
        bool interior_seen = false;
        for (int64_t s = 0; s < nslots; ++s) {
          const int64_t grp = order[(size_t)s];
          if (grp * cpw >= nc) continue;  // padding
          const bool e = edge_group(grp, g, cpw);
          if (e && interior_seen) {
            std::printf("FAIL order: g=%d cpw=%d slot=%lld\n", g, cpw, (long long)s);
            return 1;
          }
          interior_seen = interior_seen || !e;
        }
      }
      if (g % cpw != 0 && !identity) {
        std::printf("FAIL expected the identity: g=%d cpw=%d\n", g, cpw);
        return 1;
      }
      ++checked;
      reordered += identity ? 0 : 1;
    }
  }
  std::printf("ok %ld %ld\n", checked, reordered);
  return 0;
}
"""


def test_group_of_slot_is_a_bijection_with_edge_groups_first(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    src = tmp_path / "tile_order_check.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "tile_order_check"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", CSRC, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    ok, checked, reordered = out.stdout.split()
    assert ok == "ok" and int(checked) == 6 * 300
    assert int(reordered) > 300  # most grids take the edge-first order
