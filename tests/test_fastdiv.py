"""Index decoding: the invariant-divisor division of csrc/fastdiv.cuh
(compiled here as host code with nvcc, no GPU) against exact division."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "grace_b200", "csrc")

PROGRAM = r"""
#include <cstdio>
#include <cstdint>
#include "fastdiv.cuh"
using grb::fast_div;
using grb::make_fastdiv;
static uint64_t state = 0x9E3779B97F4A7C15ull;
static uint32_t rnd() {
  state ^= state << 13; state ^= state >> 7; state ^= state << 17;
  return (uint32_t)(state >> 11);
}
static int check(uint32_t d, uint32_t n) {
  const grb::FastDiv f = make_fastdiv(d);
  if (fast_div(n, f) != n / d) { std::printf("FAIL d=%u n=%u got %u\n", d, n, fast_div(n, f)); return 1; }
  return 0;
}
int main() {
  int bad = 0;
  const uint32_t edge[] = {0u, 1u, 2u, 3u, 0x7fffffffu, 0x80000000u, 0xfffffffeu, 0xffffffffu};
  for (uint32_t d = 1; d <= 4096 && !bad; ++d) {
    for (uint32_t e : edge) bad |= check(d, e);
    for (uint32_t k = 0; k < 64; ++k) {
      const uint32_t m = d * k;
      bad |= check(d, m) | check(d, m + 1) | check(d, m ? m - 1 : 0);
    }
    for (int r = 0; r < 256; ++r) bad |= check(d, rnd());
  }
  for (int r = 0; r < 2000000 && !bad; ++r) {
    const uint32_t d = (rnd() >> (rnd() % 31)) | 1u;
    bad |= check(d, rnd()) | check(d + 1, rnd());
  }
  for (int l = 0; l < 32 && !bad; ++l) {
    const uint32_t p = 1u << l;
    for (uint32_t e : edge) bad |= check(p, e) | check(p + 1, e) | (p > 2 ? check(p - 1, e) : 0);
  }
  std::printf(bad ? "fail\n" : "ok\n");
  return bad;
}
"""


@pytest.mark.skipif(shutil.which(os.environ.get("NVCC", "nvcc")) is None, reason="nvcc not found")
def test_fast_div_matches_exact_division(tmp_path):
    src = tmp_path / "fastdiv_check.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "fastdiv_check"
    subprocess.run([os.environ.get("NVCC", "nvcc"), "-O2", "-std=c++17", "-I", CSRC, str(src), "-o", str(exe)],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout
