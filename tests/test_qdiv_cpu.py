"""The reciprocal division of the kernels (qdiv in csrc/step_common.cuh:
q = a*y, then q + (a - q*b)*y with y = 1/b and exact fused multiply-adds),
checked on the CPU with C's fma(), which rounds once like the GPU's DFMA:

* normal numerators and quotients: equal to a / b bit for bit, including
  divisors whose mantissa is just below 2;
* subnormal numerators: the remainder is no longer exact and the quotient may
  differ from a / b, by at most two units in the last place (one in almost
  every case that differs; 4 M random cases).
"""
import subprocess

import pytest

SRC = r"""
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
static uint64_t s = 88172645463325252ull;
static uint64_t rnd(void) { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; }
static double qdiv(double a, double b, double y) {
    const double q = a * y;
    const double e = fma(-q, b, a);
    return e == 0.0 ? q : fma(e, y, q);
}
static int64_t ulps(double x, double z) {
    int64_t i, j; memcpy(&i, &x, 8); memcpy(&j, &z, 8);
    return i > j ? i - j : j - i;
}
int main(void) {
    long bad_normal = 0, bad_sub = 0, n_sub = 0; int64_t worst_sub = 0;
    for (int k = 0; k < 4000000; ++k) {
        int kk = 1 + (int)(rnd() % 64);
        double b = (k & 1) ? 2.0 - kk * 0x1p-52 : 1.0 + (double)(rnd() >> 11) * 0x1p-53;
        b = ldexp(b, (int)(rnd() % 64) - 32);
        const double y = 1.0 / b;
        double m = 1.0 + (double)(rnd() >> 11) * 0x1p-53;
        double a = ldexp(m, (int)(rnd() % 2000) - 1000);
        if (fabs(a / b) >= 0x1p-1022 && isfinite(a / b) && qdiv(a, b, y) != a / b) ++bad_normal;
        double as = (double)(rnd() >> 12) * 0x1p-1074;       /* subnormal numerator */
        if (as != 0.0 && as < 0x1p-1022) {
            ++n_sub;
            const double d = qdiv(as, b, y), z = as / b;
            if (d != z) { ++bad_sub; if (ulps(d, z) > worst_sub) worst_sub = ulps(d, z); }
        }
    }
    printf("%ld %ld %ld %lld\n", bad_normal, bad_sub, n_sub, (long long)worst_sub);
    return 0;
}
"""


def test_qdiv_normal_exact_subnormal_within_two_ulps(tmp_path):
    src = tmp_path / "q.c"
    src.write_text(SRC)
    exe = tmp_path / "q"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-std=c99", str(src), "-o", str(exe), "-lm"], check=True)
    bad_normal, bad_sub, n_sub, worst = map(int, subprocess.run([str(exe)], capture_output=True, text=True,
                                                               check=True).stdout.split())
    assert bad_normal == 0
    assert n_sub > 1000000
    assert worst <= 2, worst
    print("subnormal numerators whose quotient differs: %d of %d" % (bad_sub, n_sub))
