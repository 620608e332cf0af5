"""The 576-bit arithmetic that jumps a RANLUX generator ahead
(qcdgpu_b200/csrc/qg_rlx576.h), compiled for the host and checked against
Python's exact integers: the subtract-with-borrow step x_n = x_{n-10} -
x_{n-24} - c (mod 2^24) is multiplication by 2^-24 modulo m = 2^576 - 2^240
+ 1 on the state's encoding, the encoding of states the generator reaches
decodes back to the same words and borrow, products are reduced exactly,
and a jump of k steps lands on the state k steps of the recurrence give."""
import os
import random
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
B = 1 << 24
M = B ** 24 - B ** 10 + 1

HARNESS = r"""
#include <cstdio>
#include <cstdint>
#include "qg_rlx576.h"
using namespace qg::rlx;
static void swb(uint32_t (&L)[24], uint32_t &c)
{
    int32_t v = (int32_t)L[14] - (int32_t)L[0] - (int32_t)c;
    c = v < 0;
    if (v < 0) v += 1 << 24;
    for (int k = 0; k < 23; k++) L[k] = L[k + 1];
    L[23] = (uint32_t)v;
}
static void hex(const uint32_t *x) { for (int k = kLimbs - 1; k >= 0; k--) printf("%08x", x[k]); }
int main()
{
    unsigned long long s = 88172645463325252ull;
    auto rnd = [&]() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; };
    uint32_t L[24], c = 0;
    for (int k = 0; k < 24; k++) L[k] = (uint32_t)(rnd() & 0xFFFFFF);
    for (int n = 0; n < 64; n++) swb(L, c);
    for (int t = 0; t < 120; t++) {
        for (int n = 0; n < 7; n++) swb(L, c);
        uint32_t E[kLimbs], L2[24], c2, Mx[kLimbs], J[kLimbs], Lj[24], cj;
        encode(L, c, E);
        decode(E, L2, c2);
        int same = c2 == c;
        for (int k = 0; k < 24; k++) same &= L2[k] == L[k];
        const unsigned long long jump = 1 + rnd() % 5000;
        binv_pow(jump, Mx);
        mulmod(E, Mx, J);
        decode(J, Lj, cj);
        uint32_t Ls[24], cs = c;
        for (int k = 0; k < 24; k++) Ls[k] = L[k];
        for (unsigned long long n = 0; n < jump; n++) swb(Ls, cs);
        int jumped = cj == cs;
        for (int k = 0; k < 24; k++) jumped &= Lj[k] == Ls[k];
        printf("S");
        for (int k = 0; k < 24; k++) printf(" %u", L[k]);
        printf(" %u %d %d %llu E ", c, same, jumped, jump);
        hex(E);
        printf(" P ");
        hex(Mx);
        printf("\n");
    }
    for (int t = 0; t < 60; t++) {
        uint32_t a[kLimbs], b[kLimbs], r[kLimbs];
        for (int k = 0; k < kLimbs; k++) { a[k] = (uint32_t)rnd(); b[k] = (uint32_t)rnd(); }
        a[17] &= 0x7FFFFFFFu; b[17] &= 0x7FFFFFFFu;   // below m
        mulmod(a, b, r);
        printf("M ");
        hex(a); printf(" "); hex(b); printf(" "); hex(r); printf("\n");
    }
}
"""


def test_ranlux_jump_arithmetic(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "h.cpp"
    src.write_text(HARNESS)
    exe = tmp_path / "h"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "qcdgpu_b200", "csrc"), str(src), "-o",
                    str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    binv = pow(B, -1, M)
    states = products = 0
    carries = 0
    for line in out:
        f = line.split()
        if not f:
            continue
        if f[0] == "S":
            L = list(map(int, f[1:25]))
            c, same, jumped, jump = int(f[25]), int(f[26]), int(f[27]), int(f[28])
            E = int(f[30], 16)
            assert E == (sum(x * B ** k for k, x in enumerate(L)) - sum(x * B ** k for k, x in enumerate(L[14:]))
                         + c) % M
            # one step of the recurrence is multiplication by 2^-24 (mod m)
            v = L[14] - L[0] - c
            L1, c1 = L[1:] + [v % B], int(v < 0)
            E1 = (sum(x * B ** k for k, x in enumerate(L1)) - sum(x * B ** k for k, x in enumerate(L1[14:]))
                  + c1) % M
            assert E1 == binv * E % M
            assert int(f[32], 16) == pow(binv, jump, M)
            assert same == 1 and jumped == 1
            states += 1
            carries += c
        elif f[0] == "M":
            a, b, r = (int(x, 16) for x in f[1:4])
            assert r == a * b % M
            products += 1
    assert states == 120 and products == 60 and 0 < carries < states
