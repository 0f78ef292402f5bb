"""The kernels' frame time without a division (`frame_seconds` in
harvest_cuda_b200/csrc/hv_device.cuh): q = RN(f * RN(1/1000)) corrected
once by its remainder, q + RN(f - 1000 q) * RN(1/1000) with fused
multiply-adds, must equal the IEEE quotient f / 1000.0 that WORLD's
`i * 1 / 1000.0` computes. C's fma() is the same correctly rounded operation
as the device's __fma_rn, so the scheme is checked here with gcc on the host:
every f below 2^26 and a strided sweep of the rest of the int range (the
full range up to 2^31 was checked the same way when the helper was written)."""
import shutil
import subprocess

import pytest

SOURCE = r"""
#include <math.h>
#include <stdint.h>
#include <stdio.h>
static int check(int64_t f) {
  const double inv = 1.0 / 1000.0, x = (double)f;
  const double q = x * inv;
  return fma(fma(-q, 1000.0, x), inv, q) == x / 1000.0;
}
int main(void) {
  long long bad = 0;
  for (int64_t f = 0; f < (1LL << 26); ++f) bad += !check(f);
  for (int64_t f = 1LL << 26; f < (1LL << 31); f += 997) bad += !check(f);
  bad += !check(2147483647LL);
  printf("%lld\n", bad);
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_frame_seconds_equals_division(tmp_path):
    src = tmp_path / "frame_time.c"
    exe = tmp_path / "frame_time"
    src.write_text(SOURCE)
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe), str(src), "-lm"], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    assert int(out) == 0
