// qg_pair.cuh -- the SU(3) algebra of qg_su.cuh on pairs of links.
//
// Each value is a float2 holding the same quantity of two different links
// (lane x = link 0, lane y = link 1), and every operation is the packed
// FP32 instruction (__ffma2_rn / __fmul2_rn / __fadd2_rn) that performs, in
// each lane, exactly the IEEE operation the scalar code performs in the
// same order -- so a lane's result is bit-identical to the scalar path,
// while one instruction issue does the work of two.  Negations are exact,
// so fma(-a, b, c) is written with whichever operand is cheaper to negate.
#pragma once
#include "qg_su.cuh"

namespace qg {

using F2 = float2;
__device__ __forceinline__ F2 pmul(F2 a, F2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ F2 pfma(F2 a, F2 b, F2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ F2 padd(F2 a, F2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ F2 pneg(F2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ F2 psub(F2 a, F2 b) { return __fadd2_rn(a, pneg(b)); }
__device__ __forceinline__ F2 pair(float a, float b) { return make_float2(a, b); }

struct CX2 { F2 re, im; };
struct M32 { CX2 m[3][3]; };
struct G32 { F2 uv1[4], uv2[4], uv3[4]; };     // the 12-real form, component-wise
struct S22 { CX2 u1, u2, v1, v2; };

__device__ __forceinline__ G32 gpair(const G3<float> &a, const G3<float> &b)
{
    G32 g;
    g.uv1[0] = pair(a.uv1.x, b.uv1.x); g.uv1[1] = pair(a.uv1.y, b.uv1.y);
    g.uv1[2] = pair(a.uv1.z, b.uv1.z); g.uv1[3] = pair(a.uv1.w, b.uv1.w);
    g.uv2[0] = pair(a.uv2.x, b.uv2.x); g.uv2[1] = pair(a.uv2.y, b.uv2.y);
    g.uv2[2] = pair(a.uv2.z, b.uv2.z); g.uv2[3] = pair(a.uv2.w, b.uv2.w);
    g.uv3[0] = pair(a.uv3.x, b.uv3.x); g.uv3[1] = pair(a.uv3.y, b.uv3.y);
    g.uv3[2] = pair(a.uv3.z, b.uv3.z); g.uv3[3] = pair(a.uv3.w, b.uv3.w);
    return g;
}
__device__ __forceinline__ void gsplit(const G32 &g, G3<float> &a, G3<float> &b)
{
    a.uv1 = { g.uv1[0].x, g.uv1[1].x, g.uv1[2].x, g.uv1[3].x };
    a.uv2 = { g.uv2[0].x, g.uv2[1].x, g.uv2[2].x, g.uv2[3].x };
    a.uv3 = { g.uv3[0].x, g.uv3[1].x, g.uv3[2].x, g.uv3[3].x };
    b.uv1 = { g.uv1[0].y, g.uv1[1].y, g.uv1[2].y, g.uv1[3].y };
    b.uv2 = { g.uv2[0].y, g.uv2[1].y, g.uv2[2].y, g.uv2[3].y };
    b.uv3 = { g.uv3[0].y, g.uv3[1].y, g.uv3[2].y, g.uv3[3].y };
}

// sum_k a_k b_k (dot3)
__device__ __forceinline__ CX2 pdot3(const CX2 *a, int as, const CX2 *b, int bs)
{
    CX2 r;
    r.re = pmul(a[0].re, b[0].re);
    r.re = pfma(pneg(a[0].im), b[0].im, r.re);
    r.im = pmul(a[0].re, b[0].im);
    r.im = pfma(a[0].im, b[0].re, r.im);
#pragma unroll
    for (int k = 1; k < 3; k++) {
        const CX2 &x = a[k * as], &y = b[k * bs];
        r.re = pfma(x.re, y.re, r.re);
        r.re = pfma(pneg(x.im), y.im, r.re);
        r.im = pfma(x.re, y.im, r.im);
        r.im = pfma(x.im, y.re, r.im);
    }
    return r;
}
// sum_k a_k conj(b_k) (dotc3)
__device__ __forceinline__ CX2 pdotc3(const CX2 *a, int as, const CX2 *b, int bs)
{
    CX2 r;
    r.re = pmul(a[0].re, b[0].re);
    r.re = pfma(a[0].im, b[0].im, r.re);
    r.im = pmul(a[0].im, b[0].re);
    r.im = pfma(pneg(a[0].re), b[0].im, r.im);
#pragma unroll
    for (int k = 1; k < 3; k++) {
        const CX2 &x = a[k * as], &y = b[k * bs];
        r.re = pfma(x.re, y.re, r.re);
        r.re = pfma(x.im, y.im, r.re);
        r.im = pfma(x.im, y.re, r.im);
        r.im = pfma(pneg(x.re), y.im, r.im);
    }
    return r;
}
// sum_k conj(a_k) b_k (cdot3)
__device__ __forceinline__ CX2 pcdot3(const CX2 *a, int as, const CX2 *b, int bs)
{
    CX2 r;
    r.re = pmul(a[0].re, b[0].re);
    r.re = pfma(a[0].im, b[0].im, r.re);
    r.im = pmul(a[0].re, b[0].im);
    r.im = pfma(pneg(a[0].im), b[0].re, r.im);
#pragma unroll
    for (int k = 1; k < 3; k++) {
        const CX2 &x = a[k * as], &y = b[k * bs];
        r.re = pfma(x.re, y.re, r.re);
        r.re = pfma(x.im, y.im, r.re);
        r.im = pfma(x.re, y.im, r.im);
        r.im = pfma(pneg(x.im), y.re, r.im);
    }
    return r;
}

// row 3 = conj(row1 x row2) (fill_row3)
__device__ __forceinline__ void pfill_row3(M32 &a)
{
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const int p = (j + 1) % 3, q = (j + 2) % 3;
        const CX2 &u1 = a.m[0][p], &u2 = a.m[0][q], &v1 = a.m[1][p], &v2 = a.m[1][q];
        F2 re = pmul(u1.re, v2.re);
        re = pfma(pneg(u1.im), v2.im, re);
        re = pfma(pneg(u2.re), v1.re, re);
        re = pfma(u2.im, v1.im, re);
        F2 im = pmul(u2.re, v1.im);
        im = pfma(u2.im, v1.re, im);
        im = pfma(pneg(u1.re), v2.im, im);
        im = pfma(pneg(u1.im), v2.re, im);
        a.m[2][j].re = re;
        a.m[2][j].im = im;
    }
}

__device__ __forceinline__ M32 pexpand(const G32 &g)
{
    M32 a;
    a.m[0][0] = { g.uv1[0], g.uv2[0] }; a.m[0][1] = { g.uv1[1], g.uv2[1] }; a.m[0][2] = { g.uv1[2], g.uv2[2] };
    a.m[1][0] = { g.uv3[0], g.uv3[2] }; a.m[1][1] = { g.uv3[1], g.uv3[3] }; a.m[1][2] = { g.uv1[3], g.uv2[3] };
    pfill_row3(a);
    return a;
}
__device__ __forceinline__ G32 pcompress(const M32 &a)
{
    G32 g;
    g.uv1[0] = a.m[0][0].re; g.uv1[1] = a.m[0][1].re; g.uv1[2] = a.m[0][2].re; g.uv1[3] = a.m[1][2].re;
    g.uv2[0] = a.m[0][0].im; g.uv2[1] = a.m[0][1].im; g.uv2[2] = a.m[0][2].im; g.uv2[3] = a.m[1][2].im;
    g.uv3[0] = a.m[1][0].re; g.uv3[1] = a.m[1][1].re; g.uv3[2] = a.m[1][0].im; g.uv3[3] = a.m[1][1].im;
    return g;
}


// staple terms (staple_fwd3 / staple_bwd3)
__device__ __forceinline__ M32 pstaple_fwd3(const G32 &ga, const G32 &gb, const G32 &gc)
{
    M32 A = pexpand(ga), B = pexpand(gb), C = pexpand(gc), P, T;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) P.m[i][j] = pdotc3(&A.m[i][0], 1, &B.m[j][0], 1);
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) T.m[i][j] = pdotc3(&P.m[i][0], 1, &C.m[j][0], 1);
    pfill_row3(T);
    return T;
}
__device__ __forceinline__ M32 pstaple_bwd3(const G32 &ga, const G32 &gb, const G32 &gc)
{
    M32 A = pexpand(ga), B = pexpand(gb), C = pexpand(gc), R, H, T;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) R.m[i][j] = pdot3(&B.m[i][0], 1, &A.m[0][j], 3);
    pfill_row3(R);
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) H.m[i][j] = pcdot3(&C.m[0][i], 3, &R.m[0][j], 3);
    pfill_row3(H);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) T.m[i][j] = { H.m[j][i].re, pneg(H.m[j][i].im) };
    return T;
}
__device__ __forceinline__ void padd3(M32 &r, const M32 &a, const M32 &b)
{
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            r.m[i][j].re = padd(a.m[i][j].re, b.m[i][j].re);
            r.m[i][j].im = padd(a.m[i][j].im, b.m[i][j].im);
        }
}

// per-lane 1 / x as the scalar code computes it ((Real)1 / x)
__device__ __forceinline__ F2 prcp_div(F2 x) { return pair(1.0f / x.x, 1.0f / x.y); }

// the SU(2) reflection of a 2x2 block (or_step, closed form)
__device__ __forceinline__ void por_step(S22 &a)
{
    const F2 hx = padd(a.u1.re, a.v2.re);
    const F2 hz = pneg(psub(a.u1.im, a.v2.im));
    const F2 hy = pneg(psub(a.u2.re, a.v1.re));
    const F2 hw = pneg(padd(a.u2.im, a.v1.im));
    F2 n2 = pmul(hx, hx);
    n2 = pfma(hy, hy, n2);
    n2 = pfma(hz, hz, n2);
    n2 = pfma(hw, hw, n2);
    F2 v0 = pmul(hx, hx);
    v0 = pfma(pneg(hy), hy, v0);
    v0 = pfma(pneg(hz), hz, v0);
    v0 = pfma(pneg(hw), hw, v0);
    const F2 inv = prcp_div(n2);
    const F2 t = pmul(padd(hx, hx), inv);
    const F2 ax = pmul(v0, inv), ay = pmul(hy, t), az = pmul(hz, t), aw = pmul(hw, t);
    // rec2
    a.u1 = { ax, az }; a.u2 = { ay, aw };
    a.v1 = { pneg(ay), aw }; a.v2 = { ax, pneg(az) };
}

// rows i, j of U <- V (rows i, j) (rotate_rows)
__device__ __forceinline__ void protate_rows(M32 &U, int i, int j, const S22 &V)
{
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const CX2 x = U.m[i][k], y = U.m[j][k];
        F2 re = pmul(V.u1.re, x.re); re = pfma(pneg(V.u1.im), x.im, re); re = pfma(V.u2.re, y.re, re);
        re = pfma(pneg(V.u2.im), y.im, re);
        F2 im = pmul(V.u1.re, x.im); im = pfma(V.u1.im, x.re, im); im = pfma(V.u2.re, y.im, im);
        im = pfma(V.u2.im, y.re, im);
        F2 re2 = pmul(V.v1.re, x.re); re2 = pfma(pneg(V.v1.im), x.im, re2); re2 = pfma(V.v2.re, y.re, re2);
        re2 = pfma(pneg(V.v2.im), y.im, re2);
        F2 im2 = pmul(V.v1.re, x.im); im2 = pfma(V.v1.im, x.re, im2); im2 = pfma(V.v2.re, y.im, im2);
        im2 = pfma(V.v2.im, y.re, im2);
        U.m[i][k] = { re, im };
        U.m[j][k] = { re2, im2 };
    }
}

// Cabibbo-Marinari overrelaxation of a pair (cm3<float, true>; no
// Gram-Schmidt after the reflections, as cm3)
__device__ __forceinline__ G32 pcm3_or(const M32 &S, const G32 &m0, int nhitpar)
{
    G32 reslt = m0;
    M32 U = pexpand(m0);
    for (int n = 0; n < nhitpar; n++) {
#pragma unroll
        for (int sg = 0; sg < 3; sg++) {
            const int i = (sg == 2) ? 1 : 0, j = (sg == 0) ? 1 : 2;
            S22 r0;
            r0.u1 = pdot3(&U.m[i][0], 1, &S.m[0][i], 3);
            r0.u2 = pdot3(&U.m[i][0], 1, &S.m[0][j], 3);
            r0.v1 = pdot3(&U.m[j][0], 1, &S.m[0][i], 3);
            r0.v2 = pdot3(&U.m[j][0], 1, &S.m[0][j], 3);
            por_step(r0);
            protate_rows(U, i, j, r0);
        }
        reslt = pcompress(U);
        U = pexpand(reslt);
    }
    return reslt;
}

// ----------------------------------------------------- rows of one link
// Pairing inside one link: a CX2 holds two entries of the SAME matrix
// (rows 0 and 1 of a column, or columns 0 and 1 of a row) and the other
// factor of each product is one scalar broadcast to both lanes, which costs
// the packed instruction nothing.  Every entry is still the scalar
// dot3 / dotc3 / cdot3 of qg_su.cuh in the same order, so the staple terms
// below equal staple_fwd3 / staple_bwd3 bit for bit.
__device__ __forceinline__ CX2 bcast(const CX<float> &a) { return { pair(a.re, a.re), pair(a.im, a.im) }; }
__device__ __forceinline__ CX2 cpair(const CX<float> &a, const CX<float> &b) { return { pair(a.re, b.re), pair(a.im, b.im) }; }
__device__ __forceinline__ CX<float> lane0(const CX2 &a) { return { a.re.x, a.im.x }; }
__device__ __forceinline__ CX<float> lane1(const CX2 &a) { return { a.re.y, a.im.y }; }

// SU(3) matrix with rows 0, 1 held column-wise in pairs: r01[j] = (m0j, m1j)
struct MR3 { CX2 r01[3]; CX<float> r2[3]; };

__device__ __forceinline__ M3<float> mr_unpack(const MR3 &a)
{
    M3<float> m;
#pragma unroll
    for (int j = 0; j < 3; j++) { m.m[0][j] = lane0(a.r01[j]); m.m[1][j] = lane1(a.r01[j]); m.m[2][j] = a.r2[j]; }
    return m;
}
// r = a + b entry-wise (add3)
__device__ __forceinline__ void mr_add(MR3 &r, const MR3 &a, const MR3 &b)
{
#pragma unroll
    for (int j = 0; j < 3; j++) {
        r.r01[j].re = padd(a.r01[j].re, b.r01[j].re);
        r.r01[j].im = padd(a.r01[j].im, b.r01[j].im);
        r.r2[j].re = a.r2[j].re + b.r2[j].re;
        r.r2[j].im = a.r2[j].im + b.r2[j].im;
    }
}

// staple_fwd3: rows 0, 1 of P = A B^+ and of T = P C^+ in row pairs
__device__ __forceinline__ MR3 staple_fwd3_rows(const G3<float> &ga, const G3<float> &gb, const G3<float> &gc)
{
    const M3<float> B = expand(gb), C = expand(gc);
    CX2 a[3];
    a[0] = { pair(ga.uv1.x, ga.uv3.x), pair(ga.uv2.x, ga.uv3.z) };
    a[1] = { pair(ga.uv1.y, ga.uv3.y), pair(ga.uv2.y, ga.uv3.w) };
    a[2] = { pair(ga.uv1.z, ga.uv1.w), pair(ga.uv2.z, ga.uv2.w) };
    CX2 pr[3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const CX2 b[3] = { bcast(B.m[j][0]), bcast(B.m[j][1]), bcast(B.m[j][2]) };
        pr[j] = pdotc3(a, 1, b, 1);
    }
    MR3 T;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const CX2 c[3] = { bcast(C.m[j][0]), bcast(C.m[j][1]), bcast(C.m[j][2]) };
        T.r01[j] = pdotc3(pr, 1, c, 1);
    }
    M3<float> t = mr_unpack(T);
    fill_row3(t);
#pragma unroll
    for (int j = 0; j < 3; j++) T.r2[j] = t.m[2][j];
    return T;
}

// staple_bwd3 (T = H^+, H = C^+ R, R = B A): R and H computed with pairs
// over columns 0, 1 (and H's column 2 with a pair over rows 0, 1), so that
// the rows 0, 1 of T = H^+ come out as row pairs
__device__ __forceinline__ MR3 staple_bwd3_rows(const G3<float> &ga, const G3<float> &gb, const G3<float> &gc)
{
    const M3<float> A = expand(ga), B = expand(gb), C = expand(gc);
    // columns 0, 1 of A by rows: ac[k] = (A_k0, A_k1)
    const CX2 ac[3] = { cpair(A.m[0][0], A.m[0][1]), cpair(A.m[1][0], A.m[1][1]), cpair(A.m[2][0], A.m[2][1]) };
    M3<float> R;
    CX2 rc[3];                                       // rc[k] = (R_k0, R_k1)
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const CX2 b[3] = { bcast(B.m[i][0]), bcast(B.m[i][1]), bcast(B.m[i][2]) };
        rc[i] = pdot3(b, 1, ac, 1);
        R.m[i][0] = lane0(rc[i]);
        R.m[i][1] = lane1(rc[i]);
        R.m[i][2] = dot3(&B.m[i][0], 1, &A.m[0][2], 3);
    }
    fill_row3(R);
    rc[2] = cpair(R.m[2][0], R.m[2][1]);
    MR3 T;
    CX2 h[2];                                        // h[i] = (H_i0, H_i1)
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const CX2 c[3] = { bcast(C.m[0][i]), bcast(C.m[1][i]), bcast(C.m[2][i]) };
        h[i] = pcdot3(c, 1, rc, 1);
    }
    // (H_02, H_12): pair over rows, C's columns 0, 1 by rows
    const CX2 cc[3] = { cpair(C.m[0][0], C.m[0][1]), cpair(C.m[1][0], C.m[1][1]), cpair(C.m[2][0], C.m[2][1]) };
    const CX2 r2[3] = { bcast(R.m[0][2]), bcast(R.m[1][2]), bcast(R.m[2][2]) };
    const CX2 h2 = pcdot3(cc, 1, r2, 1);
    M3<float> H;
    H.m[0][0] = lane0(h[0]); H.m[0][1] = lane1(h[0]); H.m[0][2] = lane0(h2);
    H.m[1][0] = lane0(h[1]); H.m[1][1] = lane1(h[1]); H.m[1][2] = lane1(h2);
    fill_row3(H);
    // T_ab = conj(H_ba): (T_0b, T_1b) = conj(H_b0, H_b1)
    T.r01[0] = { h[0].re, pneg(h[0].im) };
    T.r01[1] = { h[1].re, pneg(h[1].im) };
    T.r01[2] = { pair(H.m[2][0].re, H.m[2][1].re), pair(-H.m[2][0].im, -H.m[2][1].im) };
    T.r2[0] = { h2.re.x, -h2.im.x };
    T.r2[1] = { h2.re.y, -h2.im.y };
    T.r2[2] = { H.m[2][2].re, -H.m[2][2].im };
    return T;
}

// cm3 with OR (unrolled subgroups) with the two rows of each subgroup in
// pairs: the block's four dot products as two pair dots (rows i, j against
// one staple column), the rotation of rows i, j as pair FMAs with the
// block's coefficients paired (u1, v1), (u2, v2) and the old rows
// broadcast.  Equal to cm3<float, true, Prn, false> bit for bit.
__device__ __forceinline__ G3<float> cm3_or_rows(const M3<float> &S, const G3<float> &m0, int nhitpar)
{
    G3<float> reslt = m0;
    M3<float> U = expand(m0);
    for (int n = 0; n < nhitpar; n++) {
#pragma unroll
        for (int sg = 0; sg < 3; sg++) {
            const int i = (sg == 2) ? 1 : 0, j = (sg == 0) ? 1 : 2;
            CX2 a[3];
#pragma unroll
            for (int k = 0; k < 3; k++) a[k] = cpair(U.m[i][k], U.m[j][k]);
            const CX2 si[3] = { bcast(S.m[0][i]), bcast(S.m[1][i]), bcast(S.m[2][i]) };
            const CX2 sj[3] = { bcast(S.m[0][j]), bcast(S.m[1][j]), bcast(S.m[2][j]) };
            const CX2 d1 = pdot3(a, 1, si, 1);        // (u1, v1)
            const CX2 d2 = pdot3(a, 1, sj, 1);        // (u2, v2)
            S2<float> r0;
            r0.u1 = lane0(d1); r0.v1 = lane1(d1); r0.u2 = lane0(d2); r0.v2 = lane1(d2);
            or_step(r0);
            const F2 cr1 = pair(r0.u1.re, r0.v1.re), ci1 = pair(r0.u1.im, r0.v1.im);
            const F2 cr2 = pair(r0.u2.re, r0.v2.re), ci2 = pair(r0.u2.im, r0.v2.im);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const CX2 x = bcast(U.m[i][k]), y = bcast(U.m[j][k]);
                F2 re = pmul(cr1, x.re);
                re = pfma(pneg(ci1), x.im, re);
                re = pfma(cr2, y.re, re);
                re = pfma(pneg(ci2), y.im, re);
                F2 im = pmul(cr1, x.im);
                im = pfma(ci1, x.re, im);
                im = pfma(cr2, y.im, im);
                im = pfma(ci2, y.re, im);
                U.m[i][k] = { re.x, im.x };
                U.m[j][k] = { re.y, im.y };
            }
        }
        reslt = compress(U);
        U = expand(reslt);
    }
    return reslt;
}

}  // namespace qg
