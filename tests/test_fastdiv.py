"""The engine's FastDiv (multiply-high division by a run-time invariant
divisor, aces-ii_b200/csrc/common.cuh) against plain integer division on the
CPU: the host branch of FastDiv::div is the same formula as the device
branch (umulhi(n, m) + n) >> s.  Compiled with g++ from the header itself."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "aces-ii_b200", "csrc")

PROGRAM = r"""
#include "common.cuh"
#include <cstdio>
#include <cstdint>
using acesb200::FastDiv;
static uint64_t state = 88172645463325252ull;
static unsigned rnd() { state ^= state << 13; state ^= state >> 7; state ^= state << 17;
                        return (unsigned)state; }
static long long bad = 0;
static void check(const FastDiv &f, unsigned n) {
  if (f.div(n) != n / f.d) { if (bad < 5) printf("d=%u n=%u\n", f.d, n); ++bad; }
}
static void edges(const FastDiv &f) {
  const unsigned lim = 1u << 31;
  for (unsigned n = 0; n < 4096; ++n) check(f, n);
  // around multiples of d spread over [0, 2^31)
  const unsigned long long step = f.d > 4096 ? f.d : (unsigned long long)f.d * (lim / f.d / 4096 + 1);
  for (unsigned long long k = step; k < lim; k += step)
    for (int e = -1; e <= 1; ++e) if (k + e < lim) check(f, (unsigned)(k + e));
  for (unsigned n = lim - 4096; n < lim; ++n) check(f, n);
  for (int r = 0; r < 20000; ++r) check(f, rnd() & (lim - 1));
}
int main() {
  for (unsigned d = 1; d <= 4096; ++d) edges(FastDiv(d));
  for (int r = 0; r < 2000; ++r) { unsigned d = (rnd() & 0x7fffffffu) | 1u; edges(FastDiv(d)); }
  // divisors of the workloads' index splits, every n below 2^31
  const unsigned full[] = {180u, 32400u};
  for (unsigned d : full) { FastDiv f(d); for (unsigned n = 0; n < (1u << 31); ++n) check(f, n); }
  printf("bad %lld\n", bad);
  return bad != 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_fastdiv_matches_integer_division(tmp_path):
    src = tmp_path / "fastdiv_check.cpp"
    exe = tmp_path / "fastdiv_check"
    src.write_text(PROGRAM)
    cuda_inc = "/usr/local/cuda/include"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, "-I", cuda_inc, str(src), "-o",
                    str(exe)], check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout
    assert r.stdout.strip().endswith("bad 0")
