// qg_rlx576.h -- RANLUX as a linear congruential generator, for jumping a
// generator ahead without running it.
//
// The subtract-with-borrow recurrence x_n = x_{n-10} - x_{n-24} - c_{n-1}
// (mod b = 2^24; c_n its borrow) is, on a suitable encoding of its state,
// multiplication by a = b^-1 modulo m = b^24 - b^10 + 1 = 2^576 - 2^240 + 1
// (Marsaglia & Zaman 1991; Luescher 1994).  With the last 24 words oldest
// first, L[0] = x_{n-24} .. L[23] = x_{n-1}, and the carry c = c_{n-1}, the
// encoding is
//     E = sum_k L[k] b^k - sum_{k<10} L[14+k] b^k + c   (mod m),
// so that E(after one step) = a E (mod m), and k steps ahead is one
// multiplication by a^k.  The map back reads the words off as digits:
// b E_n = E_{n-1} + x_{n-1} m, i.e. x_{n-1} = floor(b E_n / m) and E_{n-1}
// the remainder; 24 such steps give L, and the carry is E minus the
// encoding of L with c = 0.
//
// Residues are 18 little-endian 32-bit limbs.  Host and device code.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define QG_RLX_HD __host__ __device__ __forceinline__
#else
#define QG_RLX_HD inline
#endif

namespace qg {
namespace rlx {

constexpr int kLimbs = 18;

// m = 2^576 - 2^240 + 1
QG_RLX_HD uint32_t m_limb(int k) { return k == 0 ? 1u : k == 7 ? 0xFFFF0000u : k >= 8 ? 0xFFFFFFFFu : 0u; }

// r (N limbs, N >= 18) >= m ?
template <int N>
QG_RLX_HD bool ge_m(const uint32_t *r)
{
    bool above = false, decided = false;
#pragma unroll
    for (int k = N - 1; k >= 0; k--) {
        const uint32_t mk = k < kLimbs ? m_limb(k) : 0u;
        if (!decided && r[k] != mk) { above = r[k] > mk; decided = true; }
    }
    return decided ? above : true;
}
// r (N limbs) -= m
template <int N>
QG_RLX_HD void sub_m(uint32_t *r)
{
    uint64_t borrow = 0;
#pragma unroll
    for (int k = 0; k < N; k++) {
        const uint64_t s = (uint64_t)r[k] - (k < kLimbs ? m_limb(k) : 0u) - borrow;
        r[k] = (uint32_t)s;
        borrow = (s >> 63) & 1u;
    }
}

// t (N limbs) + h (NH limbs) * (2^240 - 1) into t; the caller sizes t for
// the sum
template <int N, int NH>
QG_RLX_HD void add_fold(uint32_t *t, const uint32_t *h)
{
    // h << 240: 7 limbs and 16 bits
    uint32_t sh[N];
#pragma unroll
    for (int k = 0; k < N; k++) sh[k] = 0;
#pragma unroll
    for (int k = 0; k < NH; k++) {
        const uint64_t v = (uint64_t)h[k] << 16;
        if (k + 7 < N) sh[k + 7] |= (uint32_t)v;
        if (k + 8 < N) sh[k + 8] |= (uint32_t)(v >> 32);
    }
    // sh -= h (sh >= h), then t += sh
    uint64_t borrow = 0, carry = 0;
#pragma unroll
    for (int k = 0; k < N; k++) {
        const uint64_t d = (uint64_t)sh[k] - (k < NH ? h[k] : 0u) - borrow;
        borrow = (d >> 63) & 1u;
        const uint64_t s2 = (uint64_t)t[k] + (uint32_t)d + carry;
        t[k] = (uint32_t)s2;
        carry = s2 >> 32;
    }
}

// r = (a b) mod m
QG_RLX_HD void mulmod(const uint32_t (&a)[kLimbs], const uint32_t (&b)[kLimbs], uint32_t (&r)[kLimbs])
{
    uint32_t p[2 * kLimbs];
#pragma unroll
    for (int k = 0; k < 2 * kLimbs; k++) p[k] = 0;
#pragma unroll
    for (int i = 0; i < kLimbs; i++) {
        uint64_t carry = 0;
#pragma unroll
        for (int j = 0; j < kLimbs; j++) {
            const uint64_t s = (uint64_t)a[i] * b[j] + p[i + j] + carry;
            p[i + j] = (uint32_t)s;
            carry = s >> 32;
        }
        p[i + kLimbs] = (uint32_t)carry;
    }
    // p = H 2^576 + L == L + H (2^240 - 1): 27 limbs, then once more: 19
    uint32_t t[27];
#pragma unroll
    for (int k = 0; k < 27; k++) t[k] = k < kLimbs ? p[k] : 0u;
    add_fold<27, kLimbs>(t, p + kLimbs);
    uint32_t u[19];
#pragma unroll
    for (int k = 0; k < 19; k++) u[k] = k < kLimbs ? t[k] : 0u;
    add_fold<19, 27 - kLimbs>(u, t + kLimbs);
    while (ge_m<19>(u)) sub_m<19>(u);
#pragma unroll
    for (int k = 0; k < kLimbs; k++) r[k] = u[k];
}

// the encoding of a state: L[0] (oldest) .. L[23] (newest) words < 2^24
QG_RLX_HD void encode(const uint32_t (&L)[24], uint32_t c, uint32_t (&E)[kLimbs])
{
    // A = sum L[k] 2^(24k), B = sum_{k<10} L[14+k] 2^(24k); E = A + (m - B) + c
    uint32_t A[19], B[kLimbs];
#pragma unroll
    for (int k = 0; k < 19; k++) A[k] = 0;
#pragma unroll
    for (int k = 0; k < kLimbs; k++) B[k] = 0;
#pragma unroll
    for (int k = 0; k < 24; k++) {
        const int bit = 24 * k, w = bit >> 5, o = bit & 31;
        const uint64_t v = (uint64_t)L[k] << o;
        A[w] |= (uint32_t)v;
        A[w + 1] |= (uint32_t)(v >> 32);
        if (k < 10) {
            const uint64_t v2 = (uint64_t)L[14 + k] << o;
            B[w] |= (uint32_t)v2;
            B[w + 1] |= (uint32_t)(v2 >> 32);
        }
    }
    // A += m - B + c
    uint64_t borrow = 0, carry = c;
#pragma unroll
    for (int k = 0; k < 19; k++) {
        const uint64_t d = (uint64_t)(k < kLimbs ? m_limb(k) : 0u) - (k < kLimbs ? B[k] : 0u) - borrow;
        borrow = (d >> 63) & 1u;
        const uint64_t s = (uint64_t)A[k] + (uint32_t)d + carry;
        A[k] = (uint32_t)s;
        carry = s >> 32;
    }
    while (ge_m<19>(A)) sub_m<19>(A);
#pragma unroll
    for (int k = 0; k < kLimbs; k++) E[k] = A[k];
}

// the state of an encoding: words L (oldest first) and the carry
QG_RLX_HD void decode(const uint32_t (&E)[kLimbs], uint32_t (&L)[24], uint32_t &c)
{
    uint32_t e[kLimbs];
#pragma unroll
    for (int k = 0; k < kLimbs; k++) e[k] = E[k];
#pragma unroll 1
    for (int step = 1; step <= 24; step++) {
        // b e = q m + r: with b e = q0 2^576 + lo (q0 = the top 24 bits of e),
        // r = lo + q0 (2^240 - 1) - (q - q0) m; lo + q0 2^240 - q0 touches
        // limbs 0 and 7, 8 and their carries only
        uint32_t t[19];
        uint32_t q = e[kLimbs - 1] >> 8;
#pragma unroll
        for (int k = kLimbs - 1; k > 0; k--) t[k] = (e[k] << 24) | (e[k - 1] >> 8);
        t[0] = e[0] << 24;
        t[kLimbs] = 0;
        uint64_t acc = (uint64_t)t[7] + ((uint64_t)q << 16);
        t[7] = (uint32_t)acc;
#pragma unroll
        for (int k = 8; k <= kLimbs; k++) {
            acc = (acc >> 32) + t[k];
            t[k] = (uint32_t)acc;
        }
        uint64_t borrow = q;
#pragma unroll
        for (int k = 0; k <= kLimbs; k++) {
            const uint64_t d = (uint64_t)t[k] - borrow;
            t[k] = (uint32_t)d;
            borrow = (d >> 63) & 1u;
        }
        while (ge_m<19>(t)) { sub_m<19>(t); q++; }
#pragma unroll
        for (int k = 0; k < kLimbs; k++) e[k] = t[k];
        L[24 - step] = q;                       // x_{n-step}
    }
    uint32_t E0[kLimbs];
    encode(L, 0u, E0);
    // c = E - E0 (mod m), 0 or 1
    uint64_t borrow = 0;
    uint32_t d0 = 0;
    uint32_t nz = 0;
#pragma unroll
    for (int k = 0; k < kLimbs; k++) {
        const uint64_t s = (uint64_t)E[k] - E0[k] - borrow;
        borrow = (s >> 63) & 1u;
        if (k == 0) d0 = (uint32_t)s; else nz |= (uint32_t)s;
    }
    c = (!borrow && !nz && d0 == 1u) ? 1u : 0u;
}

// a^e mod m for a = b^-1 = 2^576 - 2^552 - 2^240 + 2^216 + 1 (host)
inline void binv_pow(uint64_t e, uint32_t (&r)[kLimbs])
{
    uint32_t a[kLimbs], x[kLimbs];
    for (int k = 0; k < kLimbs; k++) { a[k] = m_limb(k); r[k] = k == 0 ? 1u : 0u; }
    // m - 2^552 + 2^216: 2^552 = limb 17 bit 8, 2^216 = limb 6 bit 24
    a[17] -= 1u << 8;
    a[6] += 1u << 24;
    while (e) {
        if (e & 1u) { mulmod(r, a, x); for (int k = 0; k < kLimbs; k++) r[k] = x[k]; }
        mulmod(a, a, x);
        for (int k = 0; k < kLimbs; k++) a[k] = x[k];
        e >>= 1;
    }
}

}  // namespace rlx
}  // namespace qg
