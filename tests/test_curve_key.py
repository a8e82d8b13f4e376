"""The Hilbert key that orders active targets for anchor offsets
(abyss_b200/csrc/curve.cuh), compiled for the host and checked on the CPU:

  * the 32^3 corner cube of the 1024^3 grid maps onto keys 0 .. 32767, one
    each (the curve starts at the origin and fills that cube first);
  * consecutive keys are face-adjacent cells (the property that keeps a run of
    consecutive targets compact; Z-order breaks it at every octant boundary);
  * random points agree with an independent numpy restatement of Skilling's
    transpose method.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = r"""
#include "curve.cuh"
#include <cstdio>
int main() {
  unsigned a, b, c;
  while (std::scanf("%u %u %u", &a, &b, &c) == 3) std::printf("%u\n", abyss::hilbert_key10(a, b, c));
  return 0;
}
"""


@pytest.fixture(scope="module")
def keyfn(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    d = tmp_path_factory.mktemp("curve")
    src = d / "k.cpp"
    src.write_text(SRC)
    exe = d / "k"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "abyss_b200", "csrc"), str(src), "-o",
                    str(exe)], check=True)

    def keys(pts):
        inp = "\n".join(f"{a} {b} {c}" for a, b, c in pts)
        out = subprocess.run([str(exe)], input=inp, capture_output=True, text=True, check=True).stdout.split()
        return np.array(out, dtype=np.int64)

    return keys


def numpy_hilbert(q, bits=10):
    X = q.astype(np.int64).T.copy()
    top = 1 << (bits - 1)
    Q = top
    while Q > 1:
        P = Q - 1
        for i in range(3):
            m = (X[i] & Q) != 0
            X[0] = np.where(m, X[0] ^ P, X[0])
            t = np.where(m, 0, (X[0] ^ X[i]) & P)
            X[0] ^= t
            X[i] ^= t
        Q >>= 1
    X[1] ^= X[0]
    X[2] ^= X[1]
    t = np.zeros_like(X[0])
    Q = top
    while Q > 1:
        t = np.where((X[2] & Q) != 0, t ^ (Q - 1), t)
        Q >>= 1
    X ^= t
    key = np.zeros(q.shape[0], np.int64)
    for b in range(bits - 1, -1, -1):
        for d in range(3):
            key = (key << 1) | ((X[d] >> b) & 1)
    return key


def test_corner_cube_is_filled_first_and_steps_are_adjacent(keyfn):
    g = np.stack(np.meshgrid(np.arange(32), np.arange(32), np.arange(32), indexing="ij"), -1).reshape(-1, 3)
    k = keyfn(g)
    assert np.array_equal(np.sort(k), np.arange(32 ** 3))
    walk = g[np.argsort(k)]
    step = np.abs(np.diff(walk, axis=0)).sum(axis=1)
    assert np.all(step == 1)


def test_random_points_match_restatement(keyfn):
    q = np.random.default_rng(5).integers(0, 1024, (5000, 3))
    assert np.array_equal(keyfn(q), numpy_hilbert(q))
