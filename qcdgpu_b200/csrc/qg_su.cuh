// qg_su.cuh -- SU(2)/SU(3) link algebra, staples, Kennedy-Pendleton /
// Cabibbo-Marinari heatbath and overrelaxation for the sm_100a sweep kernels.
//
// Real is the link precision (the reference's hgpu_float, SU(N)/kernel/
// complex.h:69-91).  In float mode the heatbath promotes to double exactly
// where the reference's float kernels do through double literals
// (SU(N)/suncl/su3_update_cl.cl:620,625,650-653).  Everything is
// register-resident; no function here touches memory.
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
template <typename Real> struct S3 { CX<Real> u1, u2, u3, v1, v2, v3, w1, w2, w3; };
template <typename Real> struct S2 { CX<Real> u1, u2, v1, v2; };

template <typename Real> struct RC;
template <> struct RC<float> {
    static constexpr float PI = 3.141592653589793f;
    static constexpr float PI2 = 6.283185307179586f;
    __device__ static float sn(float a) { return sinf(a); }
    __device__ static float cs(float a) { return cosf(a); }
    __device__ static float sq(float a) { return sqrtf(a); }
};
template <> struct RC<double> {
    static constexpr double PI = 3.1415926535897932384626433832795;
    static constexpr double PI2 = 6.2831853071795864769252867665590;
    __device__ static double sn(double a) { return sin(a); }
    __device__ static double cs(double a) { return cos(a); }
    __device__ static double sq(double a) { return sqrt(a); }
};

// ---------------------------------------------------------------- SU(3)
// third row = conj(row1 x row2)  (lattice_reconstruct3, su3cl.cl:137-165)
template <typename Real>
__device__ __forceinline__ S3<Real> rec3(const G3<Real> &a)
{
    S3<Real> b;
    b.u1.re = a.uv1.x; b.u1.im = a.uv2.x;
    b.u2.re = a.uv1.y; b.u2.im = a.uv2.y;
    b.u3.re = a.uv1.z; b.u3.im = a.uv2.z;
    b.v1.re = a.uv3.x; b.v1.im = a.uv3.z;
    b.v2.re = a.uv3.y; b.v2.im = a.uv3.w;
    b.v3.re = a.uv1.w; b.v3.im = a.uv2.w;
    b.w1.re =  b.u2.re * b.v3.re - b.u2.im * b.v3.im - b.u3.re * b.v2.re + b.u3.im * b.v2.im;
    b.w1.im = -b.u2.re * b.v3.im - b.u2.im * b.v3.re + b.u3.re * b.v2.im + b.u3.im * b.v2.re;
    b.w2.re =  b.u3.re * b.v1.re - b.u3.im * b.v1.im - b.u1.re * b.v3.re + b.u1.im * b.v3.im;
    b.w2.im = -b.u3.re * b.v1.im - b.u3.im * b.v1.re + b.u1.re * b.v3.im + b.u1.im * b.v3.re;
    b.w3.re =  b.u1.re * b.v2.re - b.u1.im * b.v2.im - b.u2.re * b.v1.re + b.u2.im * b.v1.im;
    b.w3.im = -b.u1.re * b.v2.im - b.u1.im * b.v2.re + b.u2.re * b.v1.im + b.u2.im * b.v1.re;
    return b;
}

template <typename Real>
__device__ __forceinline__ G3<Real> compress3(const S3<Real> &s)
{
    G3<Real> g;
    g.uv1 = { s.u1.re, s.u2.re, s.u3.re, s.v3.re };
    g.uv2 = { s.u1.im, s.u2.im, s.u3.im, s.v3.im };
    g.uv3 = { s.v1.re, s.v2.re, s.v1.im, s.v2.im };
    return g;
}

// one product entry sum_k a_k b_k, k = 1,2,3 in order
template <typename Real>
__device__ __forceinline__ CX<Real> dot3(CX<Real> a1, CX<Real> a2, CX<Real> a3, CX<Real> b1, CX<Real> b2, CX<Real> b3)
{
    CX<Real> r;
    r.re = a1.re * b1.re - a1.im * b1.im + a2.re * b2.re - a2.im * b2.im + a3.re * b3.re - a3.im * b3.im;
    r.im = a1.re * b1.im + a1.im * b1.re + a2.re * b2.im + a2.im * b2.re + a3.re * b3.im + a3.im * b3.re;
    return r;
}

// rows 1,2 of compressed x compressed (matrix_times3, su3cl.cl:51-99)
template <typename Real>
__device__ __forceinline__ G3<Real> times3(const G3<Real> &a, const G3<Real> &b)
{
    S3<Real> u = rec3(a), v = rec3(b), t;
    t.u1 = dot3(u.u1, u.u2, u.u3, v.u1, v.v1, v.w1);
    t.u2 = dot3(u.u1, u.u2, u.u3, v.u2, v.v2, v.w2);
    t.u3 = dot3(u.u1, u.u2, u.u3, v.u3, v.v3, v.w3);
    t.v1 = dot3(u.v1, u.v2, u.v3, v.u1, v.v1, v.w1);
    t.v2 = dot3(u.v1, u.v2, u.v3, v.u2, v.v2, v.w2);
    t.v3 = dot3(u.v1, u.v2, u.v3, v.u3, v.v3, v.w3);
    return compress3(t);
}

// compressed hermitian conjugate (matrix_hermitian3, su3_update_cl.cl:86-110)
template <typename Real>
__device__ __forceinline__ G3<Real> herm3(const G3<Real> &a)
{
    S3<Real> u = rec3(a);
    G3<Real> g;
    g.uv1 = { u.u1.re, u.v1.re, u.w1.re, u.w2.re };
    g.uv2 = { -u.u1.im, -u.v1.im, -u.w1.im, -u.w2.im };
    g.uv3 = { u.u2.re, u.v2.re, -u.u2.im, -u.v2.im };
    return g;
}

template <typename Real>
__device__ __forceinline__ void add3(S3<Real> &r, const S3<Real> &a, const S3<Real> &b)
{
    const Real *pa = &a.u1.re, *pb = &b.u1.re;
    Real *pr = &r.u1.re;
#pragma unroll
    for (int i = 0; i < 18; i++) pr[i] = pa[i] + pb[i];
}

template <typename Real>
__device__ __forceinline__ S3<Real> staple_fwd3(const G3<Real> &u1, const G3<Real> &u2, const G3<Real> &u3)
{
    G3<Real> m2 = times3(u1, herm3(u2));
    return rec3(times3(m2, herm3(u3)));
}
template <typename Real>
__device__ __forceinline__ S3<Real> staple_bwd3(const G3<Real> &u1, const G3<Real> &u2, const G3<Real> &u3)
{
    G3<Real> m3 = times3(herm3(u1), herm3(u2));
    return rec3(times3(m3, u3));
}

// Gram-Schmidt on rows 1,2 (lattice_GramSchmidt3, su3_update_cl.cl:228-291),
// carried out in precision Acc.
template <typename Acc, typename Real>
__device__ __forceinline__ G3<Real> gs3(const G3<Real> &m)
{
    Acc t1x = m.uv1.x, t1y = m.uv1.y, t1z = m.uv1.z, t1w = m.uv1.w;
    Acc t2x = m.uv2.x, t2y = m.uv2.y, t2z = m.uv2.z, t2w = m.uv2.w;
    Acc nu = sqrt((t1x * t1x + t2x * t2x) + (t1y * t1y + t2y * t2y) + (t1z * t1z + t2z * t2z));
    Acc ur0 = t1x / nu, ur1 = t1y / nu, ur2 = t1z / nu;
    Acc ui0 = t2x / nu, ui1 = t2y / nu, ui2 = t2z / nu;
    Acc vr0 = m.uv3.x, vr1 = m.uv3.y, vr2 = t1w;
    Acc vi0 = m.uv3.z, vi1 = m.uv3.w, vi2 = t2w;
    Acc sr = (ur0 * vr0 + ui0 * vi0) + (ur1 * vr1 + ui1 * vi1) + (ur2 * vr2 + ui2 * vi2);
    Acc si = (ur0 * vi0 - ui0 * vr0) + (ur1 * vi1 - ui1 * vr1) + (ur2 * vi2 - ui2 * vr2);
    Acc nr0 = vr0 - ur0 * sr + ui0 * si, ni0 = vi0 - ur0 * si - ui0 * sr;
    Acc nr1 = vr1 - ur1 * sr + ui1 * si, ni1 = vi1 - ur1 * si - ui1 * sr;
    Acc nr2 = vr2 - ur2 * sr + ui2 * si, ni2 = vi2 - ur2 * si - ui2 * sr;
    Acc nv = sqrt((nr0 * nr0 + ni0 * ni0) + (nr1 * nr1 + ni1 * ni1) + (nr2 * nr2 + ni2 * ni2));
    G3<Real> r;
    r.uv1 = { (Real)ur0, (Real)ur1, (Real)ur2, (Real)(nr2 / nv) };
    r.uv2 = { (Real)ui0, (Real)ui1, (Real)ui2, (Real)(ni2 / nv) };
    r.uv3 = { (Real)(nr0 / nv), (Real)(nr1 / nv), (Real)(ni0 / nv), (Real)(ni1 / nv) };
    return r;
}

// twisted boundary factor on Y links at x = N1-1 (su3_matrix_memory.cl:57-97)
template <typename Real>
__device__ __forceinline__ G3<Real> twist3(const G3<Real> &m, Real phi, Real omega)
{
    Real p = (phi + omega) / 2, q = (omega - phi) / 2;
    Real cp = RC<Real>::cs(p), sp = RC<Real>::sn(p), cq = RC<Real>::cs(q), sq = RC<Real>::sn(q);
    const R4<Real> &a = m.uv1, &b = m.uv2, &d = m.uv3;
    G3<Real> r;
    r.uv1 = { a.x * cp - b.x * sp, a.y * cp - b.y * sp, a.z * cp - b.z * sp, a.w * cq - b.w * sq };
    r.uv2 = { b.x * cp + a.x * sp, b.y * cp + a.y * sp, b.z * cp + a.z * sp, b.w * cq + a.w * sq };
    r.uv3 = { d.x * cq - d.z * sq, d.y * cq - d.w * sq, d.z * cq + d.x * sq, d.w * cq + d.y * sq };
    return r;
}

// ---------------------------------------------------------------- SU(2)
// gpu_su_2 layout x=Re u11, y=Re u12, z=Im u11, w=Im u12
// (matrix_times2, su2_matrix_memory.cl:41-53)
template <typename Real>
__device__ __forceinline__ R4<Real> times2(const R4<Real> &u, const R4<Real> &v)
{
    R4<Real> a;
    a.x = u.x * v.x - u.y * v.y - u.z * v.z - u.w * v.w;
    a.z = u.x * v.z + u.z * v.x + u.y * v.w - u.w * v.y;
    a.y = u.x * v.y + u.y * v.x + u.w * v.z - u.z * v.w;
    a.w = u.x * v.w + u.w * v.x + u.z * v.y - u.y * v.z;
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
template <typename Real>
__device__ __forceinline__ S2<Real> mul2(const S2<Real> &u, const S2<Real> &v)
{
    S2<Real> t;
    t.u1.re = (u.u1.re * v.u1.re - u.u1.im * v.u1.im) + (u.u2.re * v.v1.re - u.u2.im * v.v1.im);
    t.u1.im = (u.u1.re * v.u1.im + u.u1.im * v.u1.re) + (u.u2.re * v.v1.im + u.u2.im * v.v1.re);
    t.u2.re = (u.u1.re * v.u2.re - u.u1.im * v.u2.im) + (u.u2.re * v.v2.re - u.u2.im * v.v2.im);
    t.u2.im = (u.u1.re * v.u2.im + u.u1.im * v.u2.re) + (u.u2.re * v.v2.im + u.u2.im * v.v2.re);
    t.v1.re = (u.v1.re * v.u1.re - u.v1.im * v.u1.im) + (u.v2.re * v.v1.re - u.v2.im * v.v1.im);
    t.v1.im = (u.v1.re * v.u1.im + u.v1.im * v.u1.re) + (u.v2.re * v.v1.im + u.v2.im * v.v1.re);
    t.v2.re = (u.v1.re * v.u2.re - u.v1.im * v.u2.im) + (u.v2.re * v.v2.re - u.v2.im * v.v2.im);
    t.v2.im = (u.v1.re * v.u2.im + u.v1.im * v.u2.re) + (u.v2.re * v.v2.im + u.v2.im * v.v2.re);
    return t;
}

// ------------------------------------------------------------ heatbath
// Kennedy-Pendleton step on a 2x2 block a.  Prn::next(k) returns the k-th
// float4 of this thread's stream.  Returns true when a try was accepted
// (a <- c*aH); on rejection the SU(3) path sets a to the identity and skips
// one PRN quad (su3_update_cl.cl:568-669; SU(2) group: su2_update_cl.cl:434-531).
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
        det = RC<Real>::sq(aH.x * aH.x + aH.y * aH.y + aH.z * aH.z + aH.w * aH.w);
        aH.x /= det; aH.z /= det; aH.y /= det; aH.w /= det;
    } else {
        Real Mx = a.u1.re + a.v2.re, My = a.u1.im - a.v2.im;
        Real Mz = a.u2.re - a.v1.re, Mw = a.u2.im + a.v1.im;
        det = RC<Real>::sq(Mx * Mx + My * My + Mz * Mz + Mw * Mw);
        aH.x = Mx / det; aH.z = -My / det; aH.y = -Mz / det; aH.w = -Mw / det;
    }
    Real bdet = beta * det;
    Real delta = 0;
    bool flag = false;
    for (int i = 0; i < nhit && !flag; i++) {
        R4<Real> rnd = prn.try_quad();
        Real cosrnd = RC<Real>::cs(RC<Real>::PI2 * rnd.y);
        delta = (Real)(-(log(1.0 - (double)rnd.x) + (double)(cosrnd * cosrnd) * log(1.0 - (double)rnd.z)) / (double)bdet);
        if ((double)(rnd.w * rnd.w) <= (1.0 - 0.5 * (double)delta)) flag = true;
        if (Prn::GID) { delta = cosrnd * cosrnd / bdet; flag = true; }
    }
    if (flag) {
        R4<Real> rnd = prn.dir_quad();
        Real cosal = (Real)(1.0 - (double)delta);
        Real costh = (Real)(2.0 * (double)rnd.x - 1.0);
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

// microcanonical reflection of the block: V = aH*aH (Creutz 1987,
// Brown & Woch 1987); the reference has no overrelaxation.
template <typename Real>
__device__ __forceinline__ void or_step(S2<Real> &a)
{
    R4<Real> aH;
    aH.x =  (a.u1.re + a.v2.re);
    aH.z = -(a.u1.im - a.v2.im);
    aH.y = -(a.u2.re - a.v1.re);
    aH.w = -(a.u2.im + a.v1.im);
    Real det = RC<Real>::sq(aH.x * aH.x + aH.y * aH.y + aH.z * aH.z + aH.w * aH.w);
    aH.x /= det; aH.z /= det; aH.y /= det; aH.w /= det;
    a = rec2(times2(aH, aH));
}

// entries of U0 * staple restricted to one subgroup block
template <typename Real>
__device__ __forceinline__ CX<Real> row_col(const S3<Real> &u, int r, const S3<Real> &s, int c)
{
    const CX<Real> *ur = (r == 0) ? &u.u1 : (r == 1) ? &u.v1 : &u.w1;
    const CX<Real> *s0 = &s.u1, *s1 = &s.v1, *s2 = &s.w1;
    return dot3(ur[0], ur[1], ur[2], s0[c], s1[c], s2[c]);
}

// Cabibbo-Marinari over the SU(2) subgroups (1,2), (1,3), (2,3);
// lattice_heatbath3, su3_update_cl.cl:672-779.  OR = true replaces each
// Kennedy-Pendleton step by the reflection.
template <typename Real, bool OR, class Prn>
__device__ __forceinline__ G3<Real> cm3(const S3<Real> &staple, const G3<Real> &m0, Real beta, Prn &prn,
                                        int nhit, int nhitpar)
{
    G3<Real> reslt = m0, Vg, m1, m2, m3 = m0;
    S3<Real> U0 = rec3(m0);
    S2<Real> r0;
    const R4<Real> z = { 0, 0, 0, 0 };
    for (int j = 0; j < nhitpar; j++) {
        r0.u1 = row_col(U0, 0, staple, 0); r0.u2 = row_col(U0, 0, staple, 1);
        r0.v1 = row_col(U0, 1, staple, 0); r0.v2 = row_col(U0, 1, staple, 1);
        if (OR) or_step(r0); else kp_step<Real, true>(r0, beta, prn, nhit);
        Vg.uv1 = { r0.u1.re, r0.u2.re, 0, 0 };
        Vg.uv2 = { r0.u1.im, r0.u2.im, 0, 0 };
        Vg.uv3 = { r0.v1.re, r0.v2.re, r0.v1.im, r0.v2.im };
        m1 = times3(Vg, m3);
        U0 = rec3(m1);

        r0.u1 = row_col(U0, 0, staple, 0); r0.u2 = row_col(U0, 0, staple, 2);
        r0.v1 = row_col(U0, 2, staple, 0); r0.v2 = row_col(U0, 2, staple, 2);
        if (OR) or_step(r0); else kp_step<Real, true>(r0, beta, prn, nhit);
        Vg.uv1 = { r0.u1.re, 0, r0.u2.re, 0 };
        Vg.uv2 = { r0.u1.im, 0, r0.u2.im, 0 };
        Vg.uv3 = { 0, 1, 0, 0 };
        m2 = times3(Vg, m1);
        U0 = rec3(m2);

        r0.u1 = row_col(U0, 1, staple, 1); r0.u2 = row_col(U0, 1, staple, 2);
        r0.v1 = row_col(U0, 2, staple, 1); r0.v2 = row_col(U0, 2, staple, 2);
        if (OR) or_step(r0); else kp_step<Real, true>(r0, beta, prn, nhit);
        Vg.uv1 = { 1, 0, 0, r0.u2.re };
        Vg.uv2 = { 0, 0, 0, r0.u2.im };
        Vg.uv3 = { 0, r0.u1.re, 0, r0.u1.im };
        m3 = times3(Vg, m2);
        reslt = gs3<Real>(m3);
        U0 = rec3(reslt);
    }
    (void)z;
    return reslt;
}

}  // namespace qg
