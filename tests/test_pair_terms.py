"""The host's vectorised irregular pair terms (abyss_b200/csrc/host/pair_terms.cpp),
which gather each neighbour's record themselves, equal, bit for bit, the same
formula evaluated one neighbour at a time.

The file is compiled as the library's Makefile compiles it (g++ -O3
-ffp-contract=off -fno-fast-math -fno-math-errno), once per instruction set its
target_clones attribute selects from (AVX-512, AVX2, baseline x86-64), and each
build is compared with an unvectorised scalar evaluation (-O0) of the
per-neighbour prediction and force terms of ComputeAcceleration.cpp:14-190, on
random neighbour sets with the edge cases the integrator meets: neighbours
already at the new time (dt = 0), signed zeros, massless neighbours, eps2 = 0.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "abyss_b200", "csrc", "host", "pair_terms.cpp")
FLAGS = ["-O3", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fno-math-errno"]

SCALAR = r"""
#include <cmath>
#include "pair_terms.h"
namespace scalar_terms {
using abyss_host::NbRec;
void irregular_terms(int nn, const int *nb, const int *slot, const NbRec *rec, const double *pos, const double *vel,
                     double new_time, double scale, double eps2, double *ta, double *tj) {
  for (int k = 0; k < nn; ++k) {
    const NbRec &q = rec[slot[nb[k]]];
    const double dt = (new_time - q.t) * scale;
    double x[3], v[3], r2 = 0.0, vx = 0.0;
    for (int d = 0; d < 3; ++d) {
      double pj, vj;
      if (dt == 0) {
        pj = q.x[d];
        vj = q.v[d];
      } else {
        pj = ((q.a1[d] * dt / 3 + q.a0[d]) * dt / 2 + q.v[d]) * dt + q.x[d];
        vj = (q.a1[d] * dt / 2 + q.a0[d]) * dt + q.v[d];
      }
      x[d] = pj - pos[d];
      v[d] = vj - vel[d];
      r2 += x[d] * x[d];
      vx += v[d] * x[d];
    }
    const double r2s = r2 + eps2;
    const double m_r3 = q.m / (r2s * std::sqrt(r2s));
    for (int d = 0; d < 3; ++d) {
      ta[3 * k + d] = m_r3 * x[d];
      tj[3 * k + d] = m_r3 * (v[d] - 3 * x[d] * vx / r2s);
    }
  }
}
}
"""

DRIVER = r"""
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>
#include "pair_terms.h"
using abyss_host::NbRec;
#define SIG int, const int *, const int *, const NbRec *, const double *, const double *, double, double, double, \
            double *, double *
namespace abyss_host { void irregular_terms(SIG); }
namespace scalar_terms { void irregular_terms(SIG); }
int main() {
  std::mt19937_64 rng(11);
  std::normal_distribution<double> N(0, 1);
  std::uniform_real_distribution<double> U(0, 1);
  long bad = 0, total = 0;
  const int n = 600;
  for (int trial = 0; trial < 4000; ++trial) {
    std::vector<NbRec> rec(n);
    std::vector<int> slot(n);
    std::iota(slot.begin(), slot.end(), 0);
    std::shuffle(slot.begin(), slot.end(), rng);
    const double new_time = U(rng) * 2, scale = trial % 3 == 0 ? 1.0 : 0.0625 * (1 + U(rng));
    for (NbRec &q : rec) {
      for (int d = 0; d < 3; ++d) {
        q.x[d] = N(rng) * 0.1;
        q.v[d] = N(rng);
        q.a0[d] = N(rng) * 10;
        q.a1[d] = N(rng) * 100;
        if (rng() % 17 == 0) q.x[d] = q.v[d] = -0.0;
        if (rng() % 19 == 0) { q.a1[d] = -0.0; q.a0[d] = 0.0; }
      }
      q.t = rng() % 4 == 0 ? new_time : new_time - U(rng) * 0.01;
      q.m = rng() % 23 == 0 ? 0.0 : U(rng) * 1e-3 + 1e-6;
    }
    const int nn = 1 + (int)(rng() % 130);
    std::vector<int> nb(nn);
    for (int &j : nb) j = (int)(rng() % n);
    std::sort(nb.begin(), nb.end());
    std::vector<double> ta1(3 * nn), tj1(3 * nn), ta2(3 * nn), tj2(3 * nn);
    double pos[3], vel[3];
    for (int d = 0; d < 3; ++d) { pos[d] = N(rng) * 0.1; vel[d] = N(rng); }
    const double eps2 = trial % 5 == 0 ? 0.0 : 1e-8;
    abyss_host::irregular_terms(nn, nb.data(), slot.data(), rec.data(), pos, vel, new_time, scale, eps2, ta1.data(),
                                tj1.data());
    scalar_terms::irregular_terms(nn, nb.data(), slot.data(), rec.data(), pos, vel, new_time, scale, eps2,
                                  ta2.data(), tj2.data());
    for (int i = 0; i < 3 * nn; ++i) {
      ++total;
      if (std::memcmp(&ta1[i], &ta2[i], 8) || std::memcmp(&tj1[i], &tj2[i], 8)) ++bad;
    }
  }
  std::printf("%ld %ld\n", total, bad);
  return 0;
}
"""


def _cpu_flags():
    try:
        with open("/proc/cpuinfo") as f:
            return set(re.search(r"^flags\s*:(.*)$", f.read(), re.M).group(1).split())
    except Exception:
        return set()


@pytest.mark.parametrize("isa", ["avx512f", "avx2", "x86-64"])
def test_vectorised_terms_equal_scalar(tmp_path, isa):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    if isa != "x86-64" and isa not in _cpu_flags():
        pytest.skip(f"host CPU has no {isa}")
    # the product source with its target_clones attribute taken out, built for one ISA
    src = open(SRC).read()
    src = re.sub(r"__attribute__\(\(target_clones\([^)]*\)\)\)", "", src)
    assert "irregular_terms" in src
    (tmp_path / "terms.cpp").write_text(src)
    (tmp_path / "scalar.cpp").write_text(SCALAR)
    (tmp_path / "main.cpp").write_text(DRIVER)
    march = {"avx512f": ["-mavx512f", "-mavx2", "-mfma"], "avx2": ["-mavx2", "-mno-avx512f"],
             "x86-64": ["-mno-avx2", "-mno-avx512f"]}[isa]
    exe = tmp_path / "cmp"
    inc = "-I" + os.path.dirname(SRC)
    subprocess.run(["g++", *FLAGS, *march, inc, "-c", "terms.cpp", "-o", "terms.o"], cwd=tmp_path, check=True)
    subprocess.run(["g++", "-O0", "-std=c++17", "-ffp-contract=off", inc, "-c", "scalar.cpp", "-o", "scalar.o"],
                   cwd=tmp_path, check=True)
    subprocess.run(["g++", "-O1", "-std=c++17", inc, "main.cpp", "terms.o", "scalar.o", "-o", str(exe)],
                   cwd=tmp_path, check=True)
    total, bad = map(int, subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split())
    assert total > 100000 and bad == 0, f"{bad} of {total} terms differ"
