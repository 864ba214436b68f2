"""The shared-divisor quotient of the strict step kernels
(mage_b200/csrc/gam_quot.cuh), compiled for the host with g++ (no GPU): it
must equal the IEEE division a/d bit for bit

* on random operand bit patterns over the whole exponent range (normal,
  subnormal, zero, infinity and NaN operands included; NaN results compare
  as NaN), half of them with exponents drawn next to the ends of the fast
  path's range;
* on quotients next to rounding midpoints: a = RN(m d) for a midpoint m
  between two doubles (and its two neighbours), and quotients A/D constructed
  to lie within 2^-107 of a midpoint, the hardest cases for a division built
  from a reciprocal;
* on signed zeros.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r"""
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include "gam_quot.cuh"
static uint64_t sm(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double bits(uint64_t u) { double d; memcpy(&d, &u, 8); return d; }
static bool same(double x, double y) { return memcmp(&x, &y, 8) == 0 || (x != x && y != y); }
int main(int argc, char** argv) {
    const long n = atol(argv[1]);
    uint64_t s = 20261203;
    long bad = 0, hard = 0;
    for (long i = 0; i < n; i++) {
        uint64_t ua = sm(s), ud = sm(s);
        if (i & 1) {  // exponents next to the ends of the fast range [2^-450, 2^450)
            const int ea = 1023 + (int)(sm(s) % 1000) - 500, ed = 1023 + (int)(sm(s) % 1000) - 500;
            ua = (ua & 0x800FFFFFFFFFFFFFull) | ((uint64_t)ea << 52);
            ud = (ud & 0x800FFFFFFFFFFFFFull) | ((uint64_t)ed << 52);
        }
        const double a = bits(ua), d = bits(ud);
        const gam::QuotExact q(d);
        if (!same(q(a), a / d)) bad++;
        // a next to m*d for a midpoint m in [0.5, 2) and d in [1, 2)
        const double dd = bits((sm(s) & 0xFFFFFFFFFFFFFull) | (1023ull << 52));
        const double qq = bits((sm(s) & 0xFFFFFFFFFFFFFull) | ((1022ull + (sm(s) & 1)) << 52));
        const double ulp = std::nextafter(qq, 4.0) - qq;
        const double am = std::fma(qq, dd, 0.5 * ulp * dd);
        const gam::QuotExact q2(dd);
        for (double x : {am, std::nextafter(am, 8.0), std::nextafter(am, 0.0)})
            if (!same(q2(x), x / dd)) bad++;
        // quotients within 2^-107 of a midpoint: for an odd 54-bit M, the
        // divisor D = t M^-1 (mod 2^54) makes M D = A 2^54 + t, so A / D is
        // M 2^-54 (a midpoint between two doubles) minus t / (2^54 D)
        const uint64_t M = (sm(s) & ((1ull << 53) - 1)) | (1ull << 53) | 1ull;
        uint64_t inv = M;  // Newton iteration for M^-1 mod 2^64
        for (int it = 0; it < 6; it++) inv *= 2 - M * inv;
        for (long t : {1L, -1L, 3L, -3L}) {
            const uint64_t D = ((uint64_t)t * inv) & ((1ull << 54) - 1);
            if (D < (1ull << 52) || D >= (1ull << 53)) continue;
            const unsigned __int128 P = (unsigned __int128)M * D;
            const unsigned __int128 Aw = t > 0 ? P >> 54 : (P + (unsigned __int128)(-t)) >> 54;
            if (Aw >= ((unsigned __int128)1 << 53)) continue;
            const double A = (double)(uint64_t)Aw, Dd = (double)D;
            const gam::QuotExact q3(Dd);
            if (!same(q3(A), A / Dd)) bad++;
            if (!same(q3(-A), -A / Dd)) bad++;
            hard++;
        }
    }
    if (hard < n / 4) bad++;  // the construction must have produced cases
    for (double a : {0.0, -0.0})
        for (double d : {3.0, -3.0, 1e-300, -1e300}) {
            const gam::QuotExact q(d);
            if (!same(q(a), a / d)) bad++;
        }
    printf("%ld\n", bad);
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_shared_divisor_quotient_equals_ieee_division(tmp_path):
    src = tmp_path / "quot.cpp"
    exe = tmp_path / "quot"
    src.write_text(HARNESS)
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "mage_b200", "csrc"),
                    str(src), "-o", str(exe), "-lm"], check=True)
    out = subprocess.run([str(exe), "4000000"], check=True, capture_output=True, text=True).stdout
    assert int(out.strip()) == 0
