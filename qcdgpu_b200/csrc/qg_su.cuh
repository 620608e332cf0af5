// qg_su.cuh -- SU(2)/SU(3) link algebra, staples, Kennedy-Pendleton /
// Cabibbo-Marinari heatbath and overrelaxation for the sm_100a sweep kernels.
//
// Real is the link precision (the reference's hgpu_float, SU(N)/kernel/
// complex.h:69-91).  In float mode the heatbath promotes to double exactly
// where the reference's float kernels do through double literals
// (SU(N)/suncl/su3_update_cl.cl:620,625,650-653).
//
// Every multiply-add is an explicit fma in a fixed order and the file is
// compiled with -fmad=false, and the transcendentals on the update path
// (sin, cos, log) are this file's own routines -- sin and cos in the link
// precision, log in double as the reference promotes it -- so a sweep is a
// fixed sequence of IEEE operations: the CPU oracle that performs the same
// sequence reproduces it bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace qg {

template <typename Real> struct R4 { Real x, y, z, w; };
template <typename Real> struct CX { Real re, im; };
// 12-real compressed SU(3): rows 1,2; uv1 = Re(u11,u12,u13,u23),
// uv2 = Im(u11,u12,u13,u23), uv3 = (Re u21, Re u22, Im u21, Im u22)
// (the gpu_su_3 form of SU(N)/suncl/model.cl:146-165)
template <typename Real> struct G3 { R4<Real> uv1, uv2, uv3; };
// full 3x3 complex matrix, row major
template <typename Real> struct M3 { CX<Real> m[3][3]; };
// 2x2 complex block (su_2 of model.cl:168-173): (u1 u2; v1 v2)
template <typename Real> struct S2 { CX<Real> u1, u2, v1, v2; };

__device__ __forceinline__ float FMA(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double FMA(double a, double b, double c) { return fma(a, b, c); }

// ------------------------------------------------- elementary functions
// sin/cos for |x| < 16: Cody-Waite reduction by pi/2 with a three-part
// constant, Taylor polynomials of degree 17 (sin) / 18 (cos) on
// [-pi/4, pi/4] in Horner form (truncation < 1e-19).
__device__ __forceinline__ void qg_sincos(double x, double *s, double *c)
{
    const double INV_PIO2 = 0.63661977236758134308;
    const double P1 = 1.5707963267948966, P2 = 6.123233995736766e-17, P3 = -1.4973849048591698e-33;
    double n = rint(x * INV_PIO2);
    double f = FMA(-n, P1, x);
    f = FMA(-n, P2, f);
    f = FMA(-n, P3, f);
    double f2 = f * f;
    double ps = 2.8114572543455206e-15;                 // 1/17!
    ps = FMA(ps, f2, -7.6471637318198164e-13);           // -1/15!
    ps = FMA(ps, f2, 1.6059043836821613e-10);            // 1/13!
    ps = FMA(ps, f2, -2.5052108385441720e-08);           // -1/11!
    ps = FMA(ps, f2, 2.7557319223985893e-06);            // 1/9!
    ps = FMA(ps, f2, -1.9841269841269841e-04);           // -1/7!
    ps = FMA(ps, f2, 8.3333333333333333e-03);            // 1/5!
    ps = FMA(ps, f2, -1.6666666666666667e-01);           // -1/3!
    double sn = FMA(ps * f2, f, f);
    double pc = -1.5619206968586225e-16;                 // -1/18!
    pc = FMA(pc, f2, 4.7794773323873853e-14);            // 1/16!
    pc = FMA(pc, f2, -1.1470745597729725e-11);           // -1/14!
    pc = FMA(pc, f2, 2.0876756987868099e-09);            // 1/12!
    pc = FMA(pc, f2, -2.7557319223985888e-07);           // -1/10!
    pc = FMA(pc, f2, 2.4801587301587302e-05);            // 1/8!
    pc = FMA(pc, f2, -1.3888888888888889e-03);           // -1/6!
    pc = FMA(pc, f2, 4.1666666666666667e-02);            // 1/4!
    pc = FMA(pc, f2, -0.5);
    double cs = FMA(pc, f2, 1.0);
    int q = ((int)n) & 3;
    double ss = (q == 0) ? sn : (q == 1) ? cs : (q == 2) ? -sn : -cs;
    double cc = (q == 0) ? cs : (q == 1) ? -sn : (q == 2) ? -cs : sn;
    *s = ss;
    *c = cc;
}

// sin/cos in float for |x| < 1024 (the FP32 heatbath's float cos and
// sincos, as the reference's float kernels evaluate them): Cody-Waite
// reduction by pi/2 with a three-part float constant, Taylor polynomials of
// degree 9 (sin) / 10 (cos) on [-pi/4, pi/4] in Horner form (truncation
// below 2e-9, under the float rounding of the result)
__device__ __forceinline__ void qg_sincosf(float x, float *s, float *c)
{
    const float INV_PIO2 = 0.6366197466850281f;
    const float P1 = 1.5707963705062866f, P2 = -4.371138828673793e-08f, P3 = -1.7151245100058819e-15f;
    const float n = rintf(x * INV_PIO2);
    float f = fmaf(-n, P1, x);
    f = fmaf(-n, P2, f);
    f = fmaf(-n, P3, f);
    const float f2 = f * f;
    float ps = 2.7557318844628753e-06f;                 // 1/9!
    ps = fmaf(ps, f2, -1.9841270113829523e-04f);         // -1/7!
    ps = fmaf(ps, f2, 8.333333767950535e-03f);           // 1/5!
    ps = fmaf(ps, f2, -1.666666716337204e-01f);          // -1/3!
    const float sn = fmaf(ps * f2, f, f);
    float pc = -2.755731998149713e-07f;                  // -1/10!
    pc = fmaf(pc, f2, 2.4801587642286904e-05f);          // 1/8!
    pc = fmaf(pc, f2, -1.3888889225199819e-03f);         // -1/6!
    pc = fmaf(pc, f2, 4.16666679084301e-02f);            // 1/4!
    pc = fmaf(pc, f2, -0.5f);
    const float cs = fmaf(pc, f2, 1.0f);
    const int q = ((int)n) & 3;
    *s = (q == 0) ? sn : (q == 1) ? cs : (q == 2) ? -sn : -cs;
    *c = (q == 0) ? cs : (q == 1) ? -sn : (q == 2) ? -cs : sn;
}

// natural log of a positive normal y, table-driven (P. T. P. Tang, ACM
// TOMS 16 (1990) 378-400): y = 2^e m, m in [1, 2); k = the nearest multiple
// of 1/128 to m - 1 (from the top 8 mantissa bits, k in 0..128); with
// c_k = RN(1/(1 + k/128)) the reduced argument r = fma(m, c_k, -1) has
// |r| <= 2^-8, so log1p(r) needs the Taylor terms to r^7 only; then
// log y = (e ln2_hi + L_hi) + ((e ln2_lo + L_lo) + log1p(r)), L = -log c_k.
// The heads are multiples of 2^-32, so their sum is exact, and for y just
// below 1 (k = 128, c = 1/2, L = ln 2) heads and tails cancel exactly.  No
// division.  The table is qg_logtab.h (gen_logtab.py); read through the
// read-only data cache.
#include "qg_logtab.h"
static __device__ const double kLogC[QG_LOG_TABLE_SIZE] = QG_LOG_C_INIT;
static __device__ const double kLogHi[QG_LOG_TABLE_SIZE] = QG_LOG_LHI_INIT;
static __device__ const double kLogLo[QG_LOG_TABLE_SIZE] = QG_LOG_LLO_INIT;

__device__ __forceinline__ double qg_log(double y)
{
    const long long b = __double_as_longlong(y);
    const int e = (int)(b >> 52) - 1023;
    const int k = (int)(((b >> 44) & 0xFF) + 1) >> 1;
    const double m = __longlong_as_double((b & 0x000FFFFFFFFFFFFFLL) | 0x3FF0000000000000LL);
    const double c = __ldg(kLogC + k), lh = __ldg(kLogHi + k), ll = __ldg(kLogLo + k);
    const double r = FMA(m, c, -1.0);
    double q = 1.0 / 7.0;
    q = FMA(q, r, -1.0 / 6.0);
    q = FMA(q, r, 1.0 / 5.0);
    q = FMA(q, r, -0.25);
    q = FMA(q, r, 1.0 / 3.0);
    q = FMA(q, r, -0.5);
    const double r2 = r * r;
    const double l1p = FMA(r2, q, r);
    const double de = (double)e;
    const double hi = FMA(de, QG_LN2_HI, lh);
    const double lo = FMA(de, QG_LN2_LO, ll);
    return hi + (lo + l1p);
}

// exp(x) for |x| <= 700: x = k ln2 + r (Cody-Waite, ln 2 in two parts),
// |r| <= ln2/2, Taylor polynomial of degree 13 in Horner form (truncation
// < 1e-17 relative), scaled by 2^k (exact)
__device__ __forceinline__ double qg_exp(double x)
{
    x = fmin(fmax(x, -700.0), 700.0);
    const double LN2_HI = 6.93147180369123816490e-01, LN2_LO = 1.90821492927058770002e-10;
    const double k = rint(x * 1.44269504088896340736);
    double r = FMA(-k, LN2_HI, x);
    r = FMA(-k, LN2_LO, r);
    double p = 1.0 / 6227020800.0;                      // 1/13!
    p = FMA(p, r, 1.0 / 479001600.0);                    // 1/12!
    p = FMA(p, r, 1.0 / 39916800.0);
    p = FMA(p, r, 1.0 / 3628800.0);
    p = FMA(p, r, 1.0 / 362880.0);
    p = FMA(p, r, 1.0 / 40320.0);
    p = FMA(p, r, 1.0 / 5040.0);
    p = FMA(p, r, 1.0 / 720.0);
    p = FMA(p, r, 1.0 / 120.0);
    p = FMA(p, r, 1.0 / 24.0);
    p = FMA(p, r, 1.0 / 6.0);
    p = FMA(p, r, 0.5);
    p = FMA(p, r, 1.0);
    p = FMA(p, r, 1.0);
    return ldexp(p, (int)k);
}

template <typename Real> struct RC;
template <> struct RC<float> {
    static constexpr float PI = 3.141592653589793f;
    static constexpr float PI2 = 6.283185307179586f;
    __device__ static float sn(float a) { float s, c; qg_sincosf(a, &s, &c); return s; }
    __device__ static float cs(float a) { float s, c; qg_sincosf(a, &s, &c); return c; }
    __device__ static float sq(float a) { return sqrtf(a); }
};
template <> struct RC<double> {
    static constexpr double PI = 3.1415926535897932384626433832795;
    static constexpr double PI2 = 6.2831853071795864769252867665590;
    __device__ static double sn(double a) { double s, c; qg_sincos(a, &s, &c); return s; }
    __device__ static double cs(double a) { double s, c; qg_sincos(a, &s, &c); return c; }
    __device__ static double sq(double a) { return sqrt(a); }
};

// ------------------------------------------------------- complex kernels
// sum_k a_k b_k, k = 0,1,2, accumulated in that order
template <typename Real>
__device__ __forceinline__ CX<Real> dot3(const CX<Real> *a, int as, const CX<Real> *b, int bs)
{
    CX<Real> r;
    r.re = a[0].re * b[0].re;
    r.re = FMA(-a[0].im, b[0].im, r.re);
    r.im = a[0].re * b[0].im;
    r.im = FMA(a[0].im, b[0].re, r.im);
#pragma unroll
    for (int k = 1; k < 3; k++) {
        const CX<Real> &x = a[k * as], &y = b[k * bs];
        r.re = FMA(x.re, y.re, r.re);
        r.re = FMA(-x.im, y.im, r.re);
        r.im = FMA(x.re, y.im, r.im);
        r.im = FMA(x.im, y.re, r.im);
    }
    return r;
}
// sum_k a_k conj(b_k)
template <typename Real>
__device__ __forceinline__ CX<Real> dotc3(const CX<Real> *a, int as, const CX<Real> *b, int bs)
{
    CX<Real> r;
    r.re = a[0].re * b[0].re;
    r.re = FMA(a[0].im, b[0].im, r.re);
    r.im = a[0].im * b[0].re;
    r.im = FMA(-a[0].re, b[0].im, r.im);
#pragma unroll
    for (int k = 1; k < 3; k++) {
        const CX<Real> &x = a[k * as], &y = b[k * bs];
        r.re = FMA(x.re, y.re, r.re);
        r.re = FMA(x.im, y.im, r.re);
        r.im = FMA(x.im, y.re, r.im);
        r.im = FMA(-x.re, y.im, r.im);
    }
    return r;
}
// sum_k conj(a_k) b_k
template <typename Real>
__device__ __forceinline__ CX<Real> cdot3(const CX<Real> *a, int as, const CX<Real> *b, int bs)
{
    CX<Real> r;
    r.re = a[0].re * b[0].re;
    r.re = FMA(a[0].im, b[0].im, r.re);
    r.im = a[0].re * b[0].im;
    r.im = FMA(-a[0].im, b[0].re, r.im);
#pragma unroll
    for (int k = 1; k < 3; k++) {
        const CX<Real> &x = a[k * as], &y = b[k * bs];
        r.re = FMA(x.re, y.re, r.re);
        r.re = FMA(x.im, y.im, r.re);
        r.im = FMA(x.re, y.im, r.im);
        r.im = FMA(-x.im, y.re, r.im);
    }
    return r;
}

// row 3 = conj(row1 x row2) (lattice_reconstruct3, su3cl.cl:137-165)
template <typename Real>
__device__ __forceinline__ void fill_row3(M3<Real> &a)
{
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const int p = (j + 1) % 3, q = (j + 2) % 3;
        const CX<Real> &u1 = a.m[0][p], &u2 = a.m[0][q], &v1 = a.m[1][p], &v2 = a.m[1][q];
        // conj(u1 v2 - u2 v1)
        Real re = u1.re * v2.re;
        re = FMA(-u1.im, v2.im, re);
        re = FMA(-u2.re, v1.re, re);
        re = FMA(u2.im, v1.im, re);
        Real im = u2.re * v1.im;
        im = FMA(u2.im, v1.re, im);
        im = FMA(-u1.re, v2.im, im);
        im = FMA(-u1.im, v2.re, im);
        a.m[2][j].re = re;
        a.m[2][j].im = im;
    }
}

template <typename Real>
__device__ __forceinline__ M3<Real> expand(const G3<Real> &g)
{
    M3<Real> a;
    a.m[0][0] = { g.uv1.x, g.uv2.x }; a.m[0][1] = { g.uv1.y, g.uv2.y }; a.m[0][2] = { g.uv1.z, g.uv2.z };
    a.m[1][0] = { g.uv3.x, g.uv3.z }; a.m[1][1] = { g.uv3.y, g.uv3.w }; a.m[1][2] = { g.uv1.w, g.uv2.w };
    fill_row3(a);
    return a;
}
template <typename Real>
__device__ __forceinline__ G3<Real> compress(const M3<Real> &a)
{
    G3<Real> g;
    g.uv1 = { a.m[0][0].re, a.m[0][1].re, a.m[0][2].re, a.m[1][2].re };
    g.uv2 = { a.m[0][0].im, a.m[0][1].im, a.m[0][2].im, a.m[1][2].im };
    g.uv3 = { a.m[1][0].re, a.m[1][1].re, a.m[1][0].im, a.m[1][1].im };
    return g;
}

// staple term U_a U_b^+ U_c^+ (lattice_staple_hermitian3, su3_update_cl.cl:294-307):
// rows 1,2 of P = A B^+, rows 1,2 of T = P C^+, row 3 of T by reconstruction
// (T is in SU(3)); row 3 of A is never formed
template <typename Real>
__device__ __forceinline__ M3<Real> staple_fwd3(const G3<Real> &ga, const G3<Real> &gb, const G3<Real> &gc)
{
    M3<Real> A = expand(ga), B = expand(gb), C = expand(gc), P, T;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) P.m[i][j] = dotc3(&A.m[i][0], 1, &B.m[j][0], 1);
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) T.m[i][j] = dotc3(&P.m[i][0], 1, &C.m[j][0], 1);
    fill_row3(T);
    return T;
}
// staple term U_a^+ U_b^+ U_c (lattice_staple_hermitian_backward3,
// su3_update_cl.cl:324-338) as the adjoint of H = C^+ R, R = B A: rows 1,2
// of R, row 3 of R by reconstruction, rows 1,2 of H, row 3 of H by
// reconstruction, T = H^+
template <typename Real>
__device__ __forceinline__ M3<Real> staple_bwd3(const G3<Real> &ga, const G3<Real> &gb, const G3<Real> &gc)
{
    M3<Real> A = expand(ga), B = expand(gb), C = expand(gc), R, H, T;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) R.m[i][j] = dot3(&B.m[i][0], 1, &A.m[0][j], 3);
    fill_row3(R);
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) H.m[i][j] = cdot3(&C.m[0][i], 3, &R.m[0][j], 3);
    fill_row3(H);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) T.m[i][j] = { H.m[j][i].re, -H.m[j][i].im };
    return T;
}

template <typename Real>
__device__ __forceinline__ void add3(M3<Real> &r, const M3<Real> &a, const M3<Real> &b)
{
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            r.m[i][j].re = a.m[i][j].re + b.m[i][j].re;
            r.m[i][j].im = a.m[i][j].im + b.m[i][j].im;
        }
}

// Gram-Schmidt on rows 1,2 (lattice_GramSchmidt3, su3_update_cl.cl:228-291)
// in precision Acc; the compressed result
template <typename Acc, typename Real>
__device__ __forceinline__ G3<Real> gs3(const G3<Real> &g)
{
    Acc u[3][2] = { { (Acc)g.uv1.x, (Acc)g.uv2.x }, { (Acc)g.uv1.y, (Acc)g.uv2.y }, { (Acc)g.uv1.z, (Acc)g.uv2.z } };
    Acc v[3][2] = { { (Acc)g.uv3.x, (Acc)g.uv3.z }, { (Acc)g.uv3.y, (Acc)g.uv3.w }, { (Acc)g.uv1.w, (Acc)g.uv2.w } };
    Acc n2 = u[0][0] * u[0][0];
    n2 = FMA(u[0][1], u[0][1], n2);
#pragma unroll
    for (int k = 1; k < 3; k++) { n2 = FMA(u[k][0], u[k][0], n2); n2 = FMA(u[k][1], u[k][1], n2); }
    Acc inu = (Acc)1 / sqrt(n2);
#pragma unroll
    for (int k = 0; k < 3; k++) { u[k][0] = u[k][0] * inu; u[k][1] = u[k][1] * inu; }
    // sc = sum_k v_k conj(u_k)
    Acc sr = v[0][0] * u[0][0], si = v[0][1] * u[0][0];
    sr = FMA(v[0][1], u[0][1], sr);
    si = FMA(-v[0][0], u[0][1], si);
#pragma unroll
    for (int k = 1; k < 3; k++) {
        sr = FMA(v[k][0], u[k][0], sr); sr = FMA(v[k][1], u[k][1], sr);
        si = FMA(v[k][1], u[k][0], si); si = FMA(-v[k][0], u[k][1], si);
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {          // v <- v - sc u
        Acc r = FMA(-sr, u[k][0], v[k][0]);
        r = FMA(si, u[k][1], r);
        Acc i = FMA(-sr, u[k][1], v[k][1]);
        i = FMA(-si, u[k][0], i);
        v[k][0] = r; v[k][1] = i;
    }
    Acc m2 = v[0][0] * v[0][0];
    m2 = FMA(v[0][1], v[0][1], m2);
#pragma unroll
    for (int k = 1; k < 3; k++) { m2 = FMA(v[k][0], v[k][0], m2); m2 = FMA(v[k][1], v[k][1], m2); }
    Acc inv = (Acc)1 / sqrt(m2);
#pragma unroll
    for (int k = 0; k < 3; k++) { v[k][0] = v[k][0] * inv; v[k][1] = v[k][1] * inv; }
    G3<Real> r;
    r.uv1 = { (Real)u[0][0], (Real)u[1][0], (Real)u[2][0], (Real)v[2][0] };
    r.uv2 = { (Real)u[0][1], (Real)u[1][1], (Real)u[2][1], (Real)v[2][1] };
    r.uv3 = { (Real)v[0][0], (Real)v[1][0], (Real)v[0][1], (Real)v[1][1] };
    return r;
}

// twisted boundary factor on Y links at x = N1-1 (su3_matrix_memory.cl:57-97):
// row 1 times exp(i(phi+omega)/2), row 2 times exp(i(omega-phi)/2)
template <typename Real>
__device__ __forceinline__ G3<Real> twist3(const G3<Real> &m, Real phi, Real omega)
{
    Real p = (phi + omega) / 2, q = (omega - phi) / 2;
    Real cp = RC<Real>::cs(p), sp = RC<Real>::sn(p), cq = RC<Real>::cs(q), sq = RC<Real>::sn(q);
    const R4<Real> &a = m.uv1, &b = m.uv2, &d = m.uv3;
    G3<Real> r;
    r.uv1 = { FMA(-b.x, sp, a.x * cp), FMA(-b.y, sp, a.y * cp), FMA(-b.z, sp, a.z * cp), FMA(-b.w, sq, a.w * cq) };
    r.uv2 = { FMA(a.x, sp, b.x * cp), FMA(a.y, sp, b.y * cp), FMA(a.z, sp, b.z * cp), FMA(a.w, sq, b.w * cq) };
    r.uv3 = { FMA(-d.z, sq, d.x * cq), FMA(-d.w, sq, d.y * cq), FMA(d.x, sq, d.z * cq), FMA(d.y, sq, d.w * cq) };
    return r;
}

// ---------------------------------------------------------------- SU(2)
// gpu_su_2 layout x=Re u11, y=Re u12, z=Im u11, w=Im u12
// (matrix_times2, su2_matrix_memory.cl:41-53)
template <typename Real>
__device__ __forceinline__ R4<Real> times2(const R4<Real> &u, const R4<Real> &v)
{
    R4<Real> a;
    a.x = u.x * v.x; a.x = FMA(-u.y, v.y, a.x); a.x = FMA(-u.z, v.z, a.x); a.x = FMA(-u.w, v.w, a.x);
    a.z = u.x * v.z; a.z = FMA(u.z, v.x, a.z); a.z = FMA(u.y, v.w, a.z); a.z = FMA(-u.w, v.y, a.z);
    a.y = u.x * v.y; a.y = FMA(u.y, v.x, a.y); a.y = FMA(u.w, v.z, a.y); a.y = FMA(-u.z, v.w, a.y);
    a.w = u.x * v.w; a.w = FMA(u.w, v.x, a.w); a.w = FMA(u.z, v.y, a.w); a.w = FMA(-u.y, v.z, a.w);
    return a;
}
template <typename Real>
__device__ __forceinline__ R4<Real> herm2(const R4<Real> &u) { return { u.x, -u.y, -u.z, -u.w }; }
template <typename Real>
__device__ __forceinline__ S2<Real> rec2(const R4<Real> &a)
{
    S2<Real> b;
    b.u1 = { a.x, a.z }; b.u2 = { a.y, a.w };
    b.v1 = { -a.y, a.w }; b.v2 = { a.x, -a.z };
    return b;
}
template <typename Real>
__device__ __forceinline__ S2<Real> add2(const S2<Real> &a, const S2<Real> &b)
{
    S2<Real> r;
    r.u1 = { a.u1.re + b.u1.re, a.u1.im + b.u1.im };
    r.u2 = { a.u2.re + b.u2.re, a.u2.im + b.u2.im };
    r.v1 = { a.v1.re + b.v1.re, a.v1.im + b.v1.im };
    r.v2 = { a.v2.re + b.v2.re, a.v2.im + b.v2.im };
    return r;
}
template <typename Real>
__device__ __forceinline__ S2<Real> staple_fwd2(const R4<Real> &u1, const R4<Real> &u2, const R4<Real> &u3)
{
    return rec2(times2(times2(u1, herm2(u2)), herm2(u3)));
}
template <typename Real>
__device__ __forceinline__ S2<Real> staple_bwd2(const R4<Real> &u1, const R4<Real> &u2, const R4<Real> &u3)
{
    return rec2(times2(times2(herm2(u1), herm2(u2)), u3));
}
// full 2x2 product (matrix_times_su2, su2cl.cl:43-60)
template <typename Real>
__device__ __forceinline__ S2<Real> mul2(const S2<Real> &u, const S2<Real> &v)
{
    S2<Real> t;
    const CX<Real> U[2][2] = { { u.u1, u.u2 }, { u.v1, u.v2 } }, W[2][2] = { { v.u1, v.u2 }, { v.v1, v.v2 } };
    CX<Real> T[2][2];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) {
            Real re = U[i][0].re * W[0][j].re;
            re = FMA(-U[i][0].im, W[0][j].im, re);
            re = FMA(U[i][1].re, W[1][j].re, re);
            re = FMA(-U[i][1].im, W[1][j].im, re);
            Real im = U[i][0].re * W[0][j].im;
            im = FMA(U[i][0].im, W[0][j].re, im);
            im = FMA(U[i][1].re, W[1][j].im, im);
            im = FMA(U[i][1].im, W[1][j].re, im);
            T[i][j] = { re, im };
        }
    t.u1 = T[0][0]; t.u2 = T[0][1]; t.v1 = T[1][0]; t.v2 = T[1][1];
    return t;
}

// ------------------------------------------------------------ heatbath
// Kennedy-Pendleton step on a 2x2 block a.  Prn::try_quad / dir_quad give
// the next float4 of this thread's stream.  Returns true when a try was
// accepted (a <- c*aH); on rejection the SU(3) path sets a to the identity
// and skips one PRN quad (su3_update_cl.cl:568-669; SU(2) group:
// su2_update_cl.cl:434-531).
template <typename Real, bool SU3PATH, class Prn>
__device__ __forceinline__ bool kp_step(S2<Real> &a, Real beta, Prn &prn, int nhit)
{
    R4<Real> aH;
    Real det;
    if (SU3PATH) {
        aH.x =  (a.u1.re + a.v2.re);
        aH.z = -(a.u1.im - a.v2.im);
        aH.y = -(a.u2.re - a.v1.re);
        aH.w = -(a.u2.im + a.v1.im);
        Real n2 = aH.x * aH.x;
        n2 = FMA(aH.y, aH.y, n2); n2 = FMA(aH.z, aH.z, n2); n2 = FMA(aH.w, aH.w, n2);
        det = RC<Real>::sq(n2);
        Real id = (Real)1 / det;
        aH.x *= id; aH.z *= id; aH.y *= id; aH.w *= id;
    } else {
        Real Mx = a.u1.re + a.v2.re, My = a.u1.im - a.v2.im;
        Real Mz = a.u2.re - a.v1.re, Mw = a.u2.im + a.v1.im;
        Real n2 = Mx * Mx;
        n2 = FMA(My, My, n2); n2 = FMA(Mz, Mz, n2); n2 = FMA(Mw, Mw, n2);
        det = RC<Real>::sq(n2);
        Real id = (Real)1 / det;
        aH.x = Mx * id; aH.z = -My * id; aH.y = -Mz * id; aH.w = -Mw * id;
    }
    Real bdet = beta * det;
    Real delta = 0;
    bool flag = false;
    for (int i = 0; i < nhit && !flag; i++) {
        R4<Real> rnd = prn.try_quad();
        Real cosrnd = RC<Real>::cs(RC<Real>::PI2 * rnd.y);
        double lx = qg_log(1.0 - (double)rnd.x), lz = qg_log(1.0 - (double)rnd.z);
        delta = (Real)(-FMA((double)(cosrnd * cosrnd), lz, lx) / (double)bdet);
        if ((double)(rnd.w * rnd.w) <= FMA(-0.5, (double)delta, 1.0)) flag = true;
        if (Prn::GID) { delta = cosrnd * cosrnd / bdet; flag = true; }
    }
    if (flag) {
        R4<Real> rnd = prn.dir_quad();
        Real cosal = (Real)(1.0 - (double)delta);
        Real costh = (Real)FMA(2.0, (double)rnd.x, -1.0);
        Real sinth = (Real)sqrt(1.0 - (double)(costh * costh));
        Real sinal = (Real)sqrt(1.0 - (double)(cosal * cosal));
        Real phi = RC<Real>::PI2 * rnd.y;
        Real sinphi = RC<Real>::sn(phi), cosphi = RC<Real>::cs(phi);
        R4<Real> c;
        c.x = cosal;
        c.z = sinal * costh;
        c.y = sinal * sinth * sinphi;
        c.w = sinal * sinth * cosphi;
        a = rec2(times2(c, aH));
        return true;
    }
    if (SU3PATH) {
        a.u1 = { (Real)1, (Real)0 }; a.u2 = { (Real)0, (Real)0 };
        a.v1 = { (Real)0, (Real)0 }; a.v2 = { (Real)1, (Real)0 };
        prn.skip();
    }
    return false;
}

// microcanonical reflection of the block (Creutz 1987, Brown & Woch 1987;
// the reference has no overrelaxation): V = aH^2 with aH = h / |h| the
// normalised SU(2) projection h = (x; y, z, w) of the block, written in
// closed form as V = (x^2 - y^2 - z^2 - w^2, 2xy, 2xz, 2xw) / |h|^2 --
// one reciprocal, no square root
template <typename Real>
__device__ __forceinline__ void or_step(S2<Real> &a)
{
    const Real hx =  (a.u1.re + a.v2.re);
    const Real hz = -(a.u1.im - a.v2.im);
    const Real hy = -(a.u2.re - a.v1.re);
    const Real hw = -(a.u2.im + a.v1.im);
    Real n2 = hx * hx;
    n2 = FMA(hy, hy, n2); n2 = FMA(hz, hz, n2); n2 = FMA(hw, hw, n2);
    Real v0 = hx * hx;
    v0 = FMA(-hy, hy, v0); v0 = FMA(-hz, hz, v0); v0 = FMA(-hw, hw, v0);
    const Real inv = (Real)1 / n2;
    const Real t = (hx + hx) * inv;
    R4<Real> v = { v0 * inv, hy * t, hz * t, hw * t };
    a = rec2(v);
}

// rows i, j of U <- V (rows i, j) for the 2x2 block V = (u1 u2; v1 v2)
template <typename Real>
__device__ __forceinline__ void rotate_rows(M3<Real> &U, int i, int j, const S2<Real> &V)
{
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const CX<Real> x = U.m[i][k], y = U.m[j][k];
        Real re = V.u1.re * x.re; re = FMA(-V.u1.im, x.im, re); re = FMA(V.u2.re, y.re, re); re = FMA(-V.u2.im, y.im, re);
        Real im = V.u1.re * x.im; im = FMA(V.u1.im, x.re, im); im = FMA(V.u2.re, y.im, im); im = FMA(V.u2.im, y.re, im);
        Real re2 = V.v1.re * x.re; re2 = FMA(-V.v1.im, x.im, re2); re2 = FMA(V.v2.re, y.re, re2); re2 = FMA(-V.v2.im, y.im, re2);
        Real im2 = V.v1.re * x.im; im2 = FMA(V.v1.im, x.re, im2); im2 = FMA(V.v2.re, y.im, im2); im2 = FMA(V.v2.im, y.re, im2);
        U.m[i][k] = { re, im };
        U.m[j][k] = { re2, im2 };
    }
}

// Cabibbo-Marinari over the SU(2) subgroups (1,2), (1,3), (2,3)
// (lattice_heatbath3, su3_update_cl.cl:672-779): for each subgroup the 2x2
// block of W = U staple, a Kennedy-Pendleton draw (or the reflection when
// OR), and the rotation of the two rows of U; then Gram-Schmidt after a
// heatbath update.  The reflections keep U unitary to rounding, so an
// overrelaxation update stores U as it is: every link is reunitarised by
// its heatbath update once per sweep (and by the global pass).
// LOOP runs the three subgroups as a runtime loop (rows and columns picked
// by selects) so that the heatbath draw's code appears once; the
// arithmetic is the unrolled form's.
template <typename Real>
__device__ __forceinline__ CX<Real> pick3(const CX<Real> &a, const CX<Real> &b, const CX<Real> &c, int k)
{
    return k == 0 ? a : (k == 1 ? b : c);
}

template <typename Real, bool OR, class Prn, bool LOOP = false>
__device__ __forceinline__ G3<Real> cm3(const M3<Real> &S, const G3<Real> &m0, Real beta, Prn &prn, int nhit,
                                        int nhitpar)
{
    G3<Real> reslt = m0;
    M3<Real> U = expand(m0);
    for (int n = 0; n < nhitpar; n++) {
        if constexpr (LOOP) {
#pragma unroll 1
            for (int sg = 0; sg < 3; sg++) {
                const int i = (sg == 2) ? 1 : 0, j = (sg == 0) ? 1 : 2;
                CX<Real> ri[3], rj[3], ci[3], cj[3];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    ri[k] = pick3(U.m[0][k], U.m[1][k], U.m[2][k], i);
                    rj[k] = pick3(U.m[0][k], U.m[1][k], U.m[2][k], j);
                    ci[k] = pick3(S.m[k][0], S.m[k][1], S.m[k][2], i);
                    cj[k] = pick3(S.m[k][0], S.m[k][1], S.m[k][2], j);
                }
                S2<Real> r0;
                r0.u1 = dot3(ri, 1, ci, 1);
                r0.u2 = dot3(ri, 1, cj, 1);
                r0.v1 = dot3(rj, 1, ci, 1);
                r0.v2 = dot3(rj, 1, cj, 1);
                if (OR) or_step(r0); else kp_step<Real, true>(r0, beta, prn, nhit);
                M3<Real> R;
#pragma unroll
                for (int k = 0; k < 3; k++) { R.m[0][k] = ri[k]; R.m[1][k] = rj[k]; }
                rotate_rows(R, 0, 1, r0);
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    if (i == 0) U.m[0][k] = R.m[0][k]; else U.m[1][k] = R.m[0][k];
                    if (j == 1) U.m[1][k] = R.m[1][k]; else U.m[2][k] = R.m[1][k];
                }
            }
        } else {
#pragma unroll
            for (int sg = 0; sg < 3; sg++) {
                const int i = (sg == 2) ? 1 : 0, j = (sg == 0) ? 1 : 2;
                S2<Real> r0;
                r0.u1 = dot3(&U.m[i][0], 1, &S.m[0][i], 3);
                r0.u2 = dot3(&U.m[i][0], 1, &S.m[0][j], 3);
                r0.v1 = dot3(&U.m[j][0], 1, &S.m[0][i], 3);
                r0.v2 = dot3(&U.m[j][0], 1, &S.m[0][j], 3);
                if (OR) or_step(r0); else kp_step<Real, true>(r0, beta, prn, nhit);
                rotate_rows(U, i, j, r0);
            }
        }
        reslt = OR ? compress(U) : gs3<Real>(compress(U));
        U = expand(reslt);
    }
    return reslt;
}

}  // namespace qg
