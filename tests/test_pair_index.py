"""The pair list's index (PairIndex in bearing_b200/host/world.cpp, the flat hash table standing in
for the reference's Map from pair key to pair, src/pairs.js) against std::unordered_map under
random inserts, updates, lookups and removals: a small C++ driver compiled with the host source
runs the same operations on both and reports the first difference.  The tables stay small, about
half full, so probes wrap around the end of the arrays and removals shift entries across it."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "tests", "_build")

DRIVER = r"""
#include "../../bearing_b200/host/world.cpp"
#include <cstdio>
#include <random>
#include <unordered_map>

int main(int argc, char** argv) {
  const int ops = std::atoi(argv[1]), span = std::atoi(argv[2]);
  std::mt19937_64 rng(static_cast<uint64_t>(std::atoll(argv[3])));
  PairIndex index;
  std::unordered_map<uint64_t, int32_t> want;
  for (int op = 0; op < ops; op++) {
    const int x = static_cast<int>(rng() % span), y = static_cast<int>(rng() % span);
    const uint64_t k = (static_cast<uint64_t>(x) << 32) | static_cast<uint32_t>(y);
    const int what = static_cast<int>(rng() % 3);
    if (what == 0) {
      const int32_t v = static_cast<int32_t>(rng() % 1000000);
      index.set(k, v);
      want[k] = v;
    } else if (what == 1) {
      index.erase(k);
      want.erase(k);
    }
    if (index.contains(k) != (want.count(k) > 0) || index.used != want.size()) {
      std::printf("op %d: key %d,%d present %d want %d, %zu entries want %zu\n", op, x, y, index.contains(k),
                  static_cast<int>(want.count(k)), index.used, want.size());
      return 1;
    }
    if (op % 997 == 0) {   // every entry where it should be, with its value
      for (const auto& kv : want) {
        const size_t at = index.find(kv.first);
        if (index.keys[at] != kv.first || index.vals[at] != kv.second) {
          std::printf("op %d: entry lost or wrong\n", op);
          return 1;
        }
      }
    }
  }
  std::printf("ok %zu entries, %zu slots\n", index.used, index.keys.size());
  return 0;
}
"""


@pytest.fixture(scope="module")
def driver():
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no g++")
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(BUILD, "pair_index.cpp")
    exe = os.path.join(BUILD, "pair_index")
    with open(src, "w") as f:
        f.write(DRIVER)
    subprocess.run([cxx, "-std=c++17", "-O2", "-o", exe, src, os.path.join(ROOT, "bearing_b200", "host", "collide.cpp"),
                    "-lpthread"], check=True, capture_output=True)
    return exe


@pytest.mark.parametrize("ops,span,seed", [(200_000, 6, 1), (200_000, 40, 2), (400_000, 400, 3)],
                         ids=["36-keys", "1600-keys", "160000-keys"])
def test_the_index_agrees_with_a_map(driver, ops, span, seed):
    r = subprocess.run([driver, str(ops), str(span), str(seed)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok")
