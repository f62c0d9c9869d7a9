"""The adjoint of a resort term as an inverse resort (aces-ii_b200/csrc/
perm_plan.cuh) against the scattered update it replaces, on the CPU: random
extents, every axis order of a dense block, size-1 axes, blocks inside larger
arrays and terms that are not dense bijections (which must keep the scatter).
Compiled with g++ from the header itself."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "aces-ii_b200", "csrc")

PROGRAM = r"""
#include "perm_plan.cuh"
#include <algorithm>
#include <cstdio>
#include <cstdint>
#include <vector>
using acesb200::inverse_perm_plan;
static uint64_t st = 0x9E3779B97F4A7C15ull;
static unsigned rnd(unsigned k) { st ^= st << 13; st ^= st >> 7; st ^= st << 17; return (unsigned)(st % k); }
int main() {
  long long bad = 0, planned = 0, refused = 0;
  for (int trial = 0; trial < 20000; ++trial) {
    int n[4];
    for (int k = 0; k < 4; ++k) n[k] = 1 + rnd(rnd(3) == 0 ? 1 : 6);
    // a dense block in a random axis order, or perturbed strides
    int perm[4] = {0, 1, 2, 3};
    for (int i = 3; i > 0; --i) std::swap(perm[i], perm[rnd(i + 1)]);
    long long s[4], acc = 1;
    for (int j = 3; j >= 0; --j) { s[perm[j]] = acc; acc *= n[perm[j]]; }
    const int mode = rnd(4);
    long long pad = 0;
    if (mode == 1) { const int k = rnd(4); s[k] += 1; }                 // not dense
    if (mode == 2) { pad = 1 + rnd(5); }                                // block at an offset
    if (mode == 3) { const int k = rnd(4); if (n[k] == 1) s[k] = 7; }   // stride of a size-1 axis
    long long total = (long long)n[0] * n[1] * n[2] * n[3];
    long long span = pad + 1;
    for (int k = 0; k < 4; ++k) span += (long long)(n[k] - 1) * s[k];
    std::vector<double> ob(total), scat(span + 8, 0.0), gath(span + 8, 0.0);
    for (long long i = 0; i < total; ++i) ob[i] = 1.0 + (double)rnd(1000);
    const double alpha = 0.75;
    // scatter reference: src_bar[pad + i.s] += alpha out_bar[i]
    for (int i0 = 0; i0 < n[0]; ++i0) for (int i1 = 0; i1 < n[1]; ++i1)
      for (int i2 = 0; i2 < n[2]; ++i2) for (int i3 = 0; i3 < n[3]; ++i3) {
        const long long o = ((long long)(i0 * n[1] + i1) * n[2] + i2) * n[3] + i3;
        scat[pad + i0 * s[0] + i1 * s[1] + i2 * s[2] + i3 * s[3]] += alpha * ob[o];
      }
    int m[4]; long long t[4];
    if (!inverse_perm_plan(n, s, m, t)) {
      ++refused;
      // a refused term must be one that is not a dense bijection
      if (mode == 0 || mode == 2 || (mode == 3)) {
        bool dense = true;   // recheck: strides of axes > 1 form a dense block
        std::vector<std::pair<long long, int>> v;
        for (int k = 0; k < 4; ++k) if (n[k] > 1) v.push_back({s[k], n[k]});
        std::sort(v.rbegin(), v.rend());
        long long e = 1;
        for (int j = (int)v.size() - 1; j >= 0; --j) { if (v[j].first != e) dense = false; e *= v[j].second; }
        if (dense) { if (bad < 5) printf("refused a dense term\n"); ++bad; }
      }
      continue;
    }
    ++planned;
    // gather: blk_bar[j] += alpha out_bar[j.t] over the block of extents m
    for (int j0 = 0; j0 < m[0]; ++j0) for (int j1 = 0; j1 < m[1]; ++j1)
      for (int j2 = 0; j2 < m[2]; ++j2) for (int j3 = 0; j3 < m[3]; ++j3) {
        const long long b = ((long long)(j0 * m[1] + j1) * m[2] + j2) * m[3] + j3;
        gath[pad + b] += alpha * ob[j0 * t[0] + j1 * t[1] + j2 * t[2] + j3 * t[3]];
      }
    for (size_t q = 0; q < scat.size(); ++q)
      if (scat[q] != gath[q]) { if (bad < 5) printf("mismatch trial %d\n", trial); ++bad; break; }
  }
  printf("planned %lld refused %lld bad %lld\n", planned, refused, bad);
  return bad != 0 || planned < 1000 || refused < 100;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_inverse_resort_plan_equals_scatter(tmp_path):
    src = tmp_path / "perm_plan_check.cpp"
    exe = tmp_path / "perm_plan_check"
    src.write_text(PROGRAM)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout
    assert r.stdout.strip().endswith("bad 0")
