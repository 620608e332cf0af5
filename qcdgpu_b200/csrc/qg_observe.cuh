// qg_observe.cuh -- device pieces shared by the single-lattice kernels
// (qg_fields.cu) and the batched ones (qg_batch.cu): the FP64 view of a
// stored link, the plaquette and Polyakov-loop work of one site, the
// Gram-Schmidt pass of one element, the block sum and the final reduction.
#pragma once
#include "qg_internal.h"

namespace qg {

template <typename Real>
__device__ __forceinline__ Real param_real(double v) { return (Real)(float)v; }
template <>
__device__ __forceinline__ double param_real<double>(double v) { return v; }

// A stored link as a full 3x3 matrix in precision P -- FP64 for the
// observables (lattice_reconstruct3_double / 2_double,
// su3_measurements_cl.cl:292-319, su2_measurements_cl.cl:126-141); SU(2)
// is embedded in the upper 2x2 block with a zero third row and column.
template <int NC, typename Real, typename P>
__device__ __forceinline__ M3<P> load_as(const Field<Real> &U, const Geom &G, const Crd &c, int mu,
                                         const double *params, int twist)
{
    uint32_t e = cb_index(G, c, parity_of(c));
    M3<P> d;
    if (NC == 3) {
        G3<Real> m = U.ldg3(mu, e);
        if (twist && mu == 1 && c.x == G.n[0] - 1) m = twist3(m, param_real<Real>(params[1]), param_real<Real>(params[2]));
        G3<P> md;
        md.uv1 = { (P)m.uv1.x, (P)m.uv1.y, (P)m.uv1.z, (P)m.uv1.w };
        md.uv2 = { (P)m.uv2.x, (P)m.uv2.y, (P)m.uv2.z, (P)m.uv2.w };
        md.uv3 = { (P)m.uv3.x, (P)m.uv3.y, (P)m.uv3.z, (P)m.uv3.w };
        d = expand(md);
    } else {
        R4<Real> m = U.ldg2(mu, e);
        if (twist && mu == 1 && c.x == G.n[0] - 1) {
            Real ph = param_real<Real>(params[1]);
            R4<Real> om = { RC<Real>::cs(ph / 2), 0, RC<Real>::sn(ph / 2), 0 };
            m = times2(om, m);
        }
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) d.m[i][j] = { (P)0, (P)0 };
        d.m[0][0] = { (P)m.x, (P)m.z }; d.m[0][1] = { (P)m.y, (P)m.w };
        d.m[1][0] = { -(P)m.y, (P)m.w }; d.m[1][1] = { (P)m.x, -(P)m.z };
    }
    return d;
}
template <int NC, typename Real>
__device__ __forceinline__ M3<double> load_d(const Field<Real> &U, const Geom &G, const Crd &c, int mu,
                                             const double *params, int twist)
{
    return load_as<NC, Real, double>(U, G, c, mu, params, twist);
}

template <typename T>
__device__ __forceinline__ M3<T> mulf(const M3<T> &u, const M3<T> &v)
{
    M3<T> t;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) t.m[i][j] = dot3(&u.m[i][0], 1, &v.m[0][j], 3);
    return t;
}
// Re Tr(a b c^+ d^+) with the products and the trace in FP32: the
// operations of the FP64 form below, in the link precision
__device__ __forceinline__ float retr4f(const M3<float> &a, const M3<float> &b, const M3<float> &c,
                                        const M3<float> &d)
{
    M3<float> ab = mulf(a, b), abc;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) abc.m[i][j] = dotc3(&ab.m[i][0], 1, &c.m[j][0], 1);
    float tr = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) tr += dotc3(&abc.m[i][0], 1, &d.m[i][0], 1).re;
    return tr;
}
// Re Tr(a b c^+ d^+)  (lattice_retrace_plaquette3, su3_measurements_cl.cl:527-548)
__device__ __forceinline__ double retr4(const M3<double> &a, const M3<double> &b, const M3<double> &c,
                                        const M3<double> &d)
{
    M3<double> ab = mulf(a, b), abc, abcd;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) abc.m[i][j] = dotc3(&ab.m[i][0], 1, &c.m[j][0], 1);
    double tr = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) tr += dotc3(&abc.m[i][0], 1, &d.m[i][0], 1).re;
    (void)abcd;
    return tr;
}

// warp + block sum of K doubles; thread 0 writes the block's partials
template <int K>
__device__ __forceinline__ void block_sum_store(double (&v)[K], double *partials, uint32_t block = 0xffffffffu)
{
    if (block == 0xffffffffu) block = blockIdx.x;
    __shared__ double sh[K][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[k][wid] = x;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            double x = (lane < nw) ? sh[k][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) partials[(size_t)block * K + k] = x;
        }
    }
}

// lattice_measurement_plq + lattice_measurement (sun_measurements_cl.cl:
// 55-184,1178-1311) at site c: the xy,xz,yz (spatial) and xt,yt,zt
// (temporal) plaquettes in FP64, and the action (beta/N)(3N - ReTr)
template <int NC, typename Real>
__device__ __forceinline__ void plaq_site_c(const Field<Real> &U, const Geom &G, const double *params, int twist,
                                            const Crd &c, double (&v)[4])
{
    const Crd cx = step_plus(G, c, 0), cy = step_plus(G, c, 1), cz = step_plus(G, c, 2), ct = step_plus(G, c, 3);
    M3<double> m1 = load_d<NC, Real>(U, G, c, 0, params, twist);
    M3<double> m4 = load_d<NC, Real>(U, G, c, 1, params, twist);
    M3<double> m5 = load_d<NC, Real>(U, G, c, 2, params, twist);
    M3<double> m6 = load_d<NC, Real>(U, G, c, 3, params, twist);
    const double bet = (double)param_real<Real>(params[0]);
    double rs, rt;
    rs  = retr4(m1, load_d<NC, Real>(U, G, cx, 1, params, twist), load_d<NC, Real>(U, G, cy, 0, params, twist), m4);
    rs += retr4(m1, load_d<NC, Real>(U, G, cx, 2, params, twist), load_d<NC, Real>(U, G, cz, 0, params, twist), m5);
    rt  = retr4(m1, load_d<NC, Real>(U, G, cx, 3, params, twist), load_d<NC, Real>(U, G, ct, 0, params, twist), m6);
    rs += retr4(m4, load_d<NC, Real>(U, G, cy, 2, params, twist), load_d<NC, Real>(U, G, cz, 1, params, twist), m5);
    rt += retr4(m4, load_d<NC, Real>(U, G, cy, 3, params, twist), load_d<NC, Real>(U, G, ct, 1, params, twist), m6);
    rt += retr4(m5, load_d<NC, Real>(U, G, cz, 3, params, twist), load_d<NC, Real>(U, G, ct, 2, params, twist), m6);
    v[0] = rs; v[1] = rt;
    v[2] = bet * (3.0 * NC - rs);
    v[3] = bet * (3.0 * NC - rt);
}
// the same six plaquettes of an FP32-link lattice with FP32 products: each
// plaquette's trace in FP32, the site and lattice sums in FP64 (the
// plaquette of QG_MEAS_PLAQUETTE_F32)
template <int NC>
__device__ __forceinline__ void plaq_site_f32(const Field<float> &U, const Geom &G, const double *params, int twist,
                                              const Crd &c, double (&v)[4])
{
    const Crd cx = step_plus(G, c, 0), cy = step_plus(G, c, 1), cz = step_plus(G, c, 2), ct = step_plus(G, c, 3);
    auto ld = [&](const Crd &q, int mu) { return load_as<NC, float, float>(U, G, q, mu, params, twist); };
    const M3<float> m1 = ld(c, 0), m4 = ld(c, 1), m5 = ld(c, 2), m6 = ld(c, 3);
    const double bet = (double)param_real<float>(params[0]);
    double rs, rt;
    rs  = (double)retr4f(m1, ld(cx, 1), ld(cy, 0), m4);
    rs += (double)retr4f(m1, ld(cx, 2), ld(cz, 0), m5);
    rt  = (double)retr4f(m1, ld(cx, 3), ld(ct, 0), m6);
    rs += (double)retr4f(m4, ld(cy, 2), ld(cz, 1), m5);
    rt += (double)retr4f(m4, ld(cy, 3), ld(ct, 1), m6);
    rt += (double)retr4f(m5, ld(cz, 3), ld(ct, 2), m6);
    v[0] = rs; v[1] = rt;
    v[2] = bet * (3.0 * NC - rs);
    v[3] = bet * (3.0 * NC - rt);
}

template <int NC, typename Real>
__device__ __forceinline__ void plaq_site(const Field<Real> &U, const Geom &G, const double *params, int twist,
                                          uint32_t s, double (&v)[4])
{
    plaq_site_c<NC, Real>(U, G, params, twist, lex2crd(G, s), v);
}

// lattice_polyakov (polyakov.cl:54-140) at spatial site c (c.t = 0):
// ordered product of the N4 T-links in link precision, traces in FP64;
// v = Re P, Im P, |P|^2, |P|^4
template <int NC, typename Real>
__device__ __forceinline__ void poly_site_c(const Field<Real> &U, const Geom &G, Crd c, double (&v)[4])
{
    double pr, pi;
    c.t = 0;
    if (NC == 3) {
        M3<Real> v0 = expand(U.ldg3(3, cb_index(G, c, parity_of(c))));
        for (int k = 1; k < G.n[3]; k++) {
            c.t = k;
            M3<Real> v1 = expand(U.ldg3(3, cb_index(G, c, parity_of(c))));
            v0 = mulf(v0, v1);
        }
        pr = (double)v0.m[0][0].re + (double)v0.m[1][1].re + (double)v0.m[2][2].re;
        pi = (double)v0.m[0][0].im + (double)v0.m[1][1].im + (double)v0.m[2][2].im;
    } else {
        S2<Real> v0 = rec2(U.ldg2(3, cb_index(G, c, parity_of(c))));
        for (int k = 1; k < G.n[3]; k++) {
            c.t = k;
            S2<Real> v1 = rec2(U.ldg2(3, cb_index(G, c, parity_of(c))));
            v0 = mul2(v0, v1);
        }
        pr = (double)v0.u1.re + (double)v0.v2.re;
        pi = (double)v0.u1.im + (double)v0.v2.im;
    }
    double q2 = pr * pr + pi * pi;
    v[0] = pr; v[1] = pi; v[2] = q2; v[3] = q2 * q2;
}
// the same at spatial index i = y + N2 (z + N3 x)
template <int NC, typename Real>
__device__ __forceinline__ void poly_site(const Field<Real> &U, const Geom &G, uint32_t i, double (&v)[4])
{
    Crd c;
    c.y = (int)(i % (uint32_t)G.n[1]);
    uint32_t r = i / (uint32_t)G.n[1];
    c.z = (int)(r % (uint32_t)G.n[2]);
    c.x = (int)(r / (uint32_t)G.n[2]);
    c.t = 0;
    poly_site_c<NC, Real>(U, G, c, v);
}

// ------------------------------------------------- F_munu and profiles
// the plaquette matrix a b c^+ d^+ in FP64 (lattice_retrace_plaquette3_F,
// su3_measurements_cl.cl:555-586)
__device__ __forceinline__ M3<double> plaq_matrix(const M3<double> &a, const M3<double> &b, const M3<double> &c,
                                                  const M3<double> &d)
{
    M3<double> ab = mulf(a, b), abc, r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) abc.m[i][j] = dotc3(&ab.m[i][0], 1, &c.m[j][0], 1);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.m[i][j] = dotc3(&abc.m[i][0], 1, &d.m[j][0], 1);
    return r;
}

// -i Tr(P T_a): T_a = lambda_a / 2 (SU(3), a = 1..8; trace_lambda1..8_double,
// su3_measurements_cl.cl:355-460) or sigma_a / 2 (SU(2), a = 1..3, real
// part only; trace_sigma1..3_double, su2_measurements_cl.cl:89-124) -- the
// generator's two (three) non-zero entries picked out of P
template <int NC>
__device__ __forceinline__ void gen_proj(const M3<double> &P, int a, double &re, double &im)
{
    const CX<double> u1 = P.m[0][0], u2 = P.m[0][1], u3 = P.m[0][2];
    const CX<double> v1 = P.m[1][0], v2 = P.m[1][1], v3 = P.m[1][2];
    const CX<double> w1 = P.m[2][0], w2 = P.m[2][1], w3 = P.m[2][2];
    re = 0; im = 0;
    if (NC == 2) {
        re = a == 1 ? u2.im : a == 2 ? u2.re : u1.im;
        return;
    }
    switch (a) {
    case 1: re = u2.im + v1.im; im = -u2.re - v1.re; break;
    case 2: re = u2.re - v1.re; im = u2.im - v1.im; break;
    case 3: re = u1.im - v2.im; im = -u1.re + v2.re; break;
    case 4: re = u3.im + w1.im; im = -u3.re - w1.re; break;
    case 5: re = u3.re - w1.re; im = u3.im - w1.im; break;
    case 6: re = v3.im + w2.im; im = -v3.re - w2.re; break;
    case 7: re = v3.re - w2.re; im = v3.im - w2.im; break;
    default:
        re = (u1.im + v2.im - 2.0 * w3.im) * 0.57735026918962576451;
        im = (-u1.re - v2.re + 2.0 * w3.re) * 0.57735026918962576451;
        break;
    }
    re /= 2; im /= 2;
}

// the FMUNU / F0MU plaquette kernels (sun_measurements_cl.cl:712-1175) at
// site s: for plane p of {xy, xz, yz} (field 0) or {xt, yt, zt} (field 1)
// v[2p], v[2p+1] = -i Tr(P T_i1), v[6+2p], v[7+2p] = -i Tr(P T_i2)
template <int NC, typename Real>
__device__ __forceinline__ void fmunu_site(const Field<Real> &U, const Geom &G, const double *params, int twist,
                                           uint32_t s, int field, int i1, int i2, double (&v)[12])
{
    const Crd c = lex2crd(G, s);
#pragma unroll
    for (int p = 0; p < 3; p++) {
        const int m = field ? p : (p == 2 ? 1 : 0);
        const int n = field ? 3 : (p == 0 ? 1 : 2);
        const Crd cm = step_plus(G, c, m), cn = step_plus(G, c, n);
        const M3<double> P = plaq_matrix(load_d<NC, Real>(U, G, c, m, params, twist),
                                         load_d<NC, Real>(U, G, cm, n, params, twist),
                                         load_d<NC, Real>(U, G, cn, m, params, twist),
                                         load_d<NC, Real>(U, G, c, n, params, twist));
        double re, im;
        gen_proj<NC>(P, i1, re, im);
        v[2 * p] = re; v[2 * p + 1] = im;
        gen_proj<NC>(P, i2, re, im);
        v[6 + 2 * p] = re; v[7 + 2 * p] = im;
    }
}

// the j-th site of slice k of coordinate `axis`: the other coordinates
// enumerated with y fastest, then z, t, x (the link table's lexicographic
// order, so consecutive j are mostly consecutive addresses); with
// spatial = true t is 0 and only x, y, z are enumerated
__device__ __forceinline__ Crd slice_site(const Geom &G, int axis, int k, uint32_t j, bool spatial)
{
    Crd c;
    if (axis == 1) { c.y = k; } else { c.y = (int)(j % (uint32_t)G.n[1]); j /= (uint32_t)G.n[1]; }
    if (axis == 2) { c.z = k; } else { c.z = (int)(j % (uint32_t)G.n[2]); j /= (uint32_t)G.n[2]; }
    if (spatial) { c.t = 0; } else { c.t = (int)(j % (uint32_t)G.n[3]); j /= (uint32_t)G.n[3]; }
    if (axis == 0) { c.x = k; } else { c.x = (int)j; }
    return c;
}

// lattice_GramSchmidt (suncl.cl:350-396) of the four links stored at
// checkerboard element i; Acc = double for the FP64 pass on FP32 links
template <int NC, typename Real, typename Acc>
__device__ __forceinline__ void gs_site(const Field<Real> &U, uint32_t i)
{
    for (int mu = 0; mu < 4; mu++) {
        if (NC == 3) {
            U.st3(mu, i, gs3<Acc>(U.ld3(mu, i)));
        } else {
            R4<Real> m = U.ld2(mu, i);
            Acc x = m.x, y = m.y, z = m.z, w = m.w;
            Acc det = sqrt(x * x + y * y + z * z + w * w);
            U.st2(mu, i, R4<Real>{ (Real)(x / det), (Real)(y / det), (Real)(z / det), (Real)(w / det) });
        }
    }
}

// one block's fixed-order sum of nblocks partials of ncomp components
// (the second pass of every reduction; deterministic run to run); any
// multiple of 32 threads up to 1024; out may be null (the sums are then
// dropped)
__device__ __forceinline__ void reduce_partials(const double *partials, uint32_t nblocks, int ncomp, double *out)
{
    __shared__ double sh[32];
    for (int k = 0; k < ncomp; k++) {
        double x = 0;
        for (uint32_t b = threadIdx.x; b < nblocks; b += blockDim.x) x += partials[(size_t)b * ncomp + k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x < 32) {
            x = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;   // only the block's warps wrote sh
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (threadIdx.x == 0 && out) out[k] = x;
        }
        __syncthreads();
    }
}

}  // namespace qg
