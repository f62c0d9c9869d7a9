"""CPU test of the small dense non-symmetric eigensolver of the EOM Davidson
(aces-ii_b200/csrc/eig_small.h): a g++ harness against numpy.linalg.eig on
random matrices, matrices with complex pairs, diagonally dominant
Davidson-like subspace matrices and a defective-looking near-degenerate case."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HARNESS = r"""
#include <cstdio>
#include <vector>
#include "eig_small.h"
int main() {
  int n;
  while (std::scanf("%d", &n) == 1) {
    std::vector<double> A((size_t)n * n);
    for (auto &x : A) std::scanf("%lf", &x);
    auto ev = acesb200::small::eig_values(A, n);
    for (auto &z : ev) std::printf("%.17g %.17g ", z.real(), z.imag());
    double lo = 1e300;
    for (auto &z : ev) if (std::abs(z.imag()) < 1e-9 && z.real() < lo) lo = z.real();
    auto y = acesb200::small::eig_vector(A, n, lo);
    std::printf("| %.17g |", lo);
    for (double v : y) std::printf(" %.17g", v);
    std::printf("\n");
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("eig")
    src = d / "h.cpp"
    src.write_text(HARNESS)
    exe = d / "h"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "aces-ii_b200", "csrc"),
                    str(src), "-o", str(exe)], check=True, capture_output=True, text=True)
    return str(exe)


def run(harness, mats):
    inp = "".join(f"{m.shape[0]} " + " ".join(repr(float(x)) for x in m.ravel()) + "\n"
                  for m in mats)
    out = subprocess.run([harness], input=inp, capture_output=True, text=True, check=True).stdout
    res = []
    for line, m in zip(out.strip().split("\n"), mats):
        head, lo, vec = line.split("|")
        z = np.array([float(x) for x in head.split()]).reshape(-1, 2)
        res.append((z[:, 0] + 1j * z[:, 1], float(lo), np.array([float(x) for x in vec.split()])))
    return res


def test_eigenvalues_match_numpy(harness):
    rng = np.random.default_rng(1)
    mats = []
    for n in (1, 2, 3, 5, 8, 13, 21, 40, 60):
        mats.append(rng.normal(size=(n, n)))                                   # complex pairs
        A = np.diag(np.sort(rng.uniform(0.2, 3.0, n))) + 0.05 * rng.normal(size=(n, n))
        mats.append(A)                                                         # Davidson-like
    mats.append(np.diag([1.0, 1.0 + 1e-9, 2.0]) + 1e-6 * np.triu(np.ones((3, 3)), 1))
    for m, (ev, lo, y) in zip(mats, run(harness, mats)):
        ref = np.linalg.eigvals(m)
        key = lambda z: (round(z.real, 6), round(z.imag, 6))
        got, exp = sorted(ev, key=key), sorted(ref, key=key)
        scale = max(1.0, np.abs(ref).max())
        assert np.abs(np.array(got) - np.array(exp)).max() < 1e-9 * scale, m.shape
        real = ref[np.abs(ref.imag) < 1e-9].real
        if real.size:
            assert abs(lo - real.min()) < 1e-9 * scale
            # the eigenvector of the lowest real eigenvalue
            r = m @ y - lo * y
            assert np.linalg.norm(r) < 1e-7 * scale * np.linalg.norm(y)
