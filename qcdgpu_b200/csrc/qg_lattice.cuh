// qg_lattice.cuh -- lattice geometry, checkerboarded link storage and
// per-thread PRN sources for the sm_100a sweep kernels.
//
// Site numbering follows the reference (SU(N)/suncl/sun_common.cl:41-66):
// s = y + N2*z + N2*N3*t + N2*N3*N4*x, y fastest, x slowest.
//
// HBM layout of the link field (this library's own): 12 planes (SU(3)) or 4
// planes (SU(2)) of 4-vectors in the reference's plane order (plane
// dir + 4*k, k = row part), but inside each plane the sites are
// checkerboarded: element (parity, s>>1) at parity*cb + (s>>1).  A phase
// kernel then touches contiguous runs of one parity and every 4-vector load
// of a warp is a fully used 512-byte (FP32) or 1 KiB (FP64) segment.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "qg_su.cuh"

namespace qg {

// unsigned division by a run-time constant: round-up multiply-high method
// (Granlund & Montgomery, PLDI 1994)
struct FastDiv {
    uint32_t d, m, l;
    __device__ __forceinline__ uint32_t div(uint32_t n) const
    {
        if (d == 1) return n;
        uint32_t hi = __umulhi(n, m);
        return (hi + ((n - hi) >> 1)) >> (l - 1);
    }
};

inline FastDiv make_fastdiv(uint32_t d)
{
    FastDiv f;
    f.d = d;
    f.m = 0;
    f.l = 0;
    if (d > 1) {
        uint32_t l = 0;
        while ((1ull << l) < d) l++;
        f.l = l;
        f.m = (uint32_t)((((unsigned __int128)1 << 32) * (((uint64_t)1 << l) - d)) / d + 1);
    }
    return f;
}

struct Geom {
    int n[4];             // N1..N4 (x, y, z, t)
    uint32_t V, half;     // sites, sites/2
    uint32_t cb;          // checkerboard half stride (elements)
    uint32_t pstride;     // plane stride = 2*cb
    uint32_t n2n3, n2n3n4;
    FastDiv d2, d23, d234;
};

struct Crd { int x, y, z, t; };

__device__ __forceinline__ Crd lex2crd(const Geom &G, uint32_t s)
{
    Crd c;
    uint32_t x = G.d234.div(s);
    uint32_t r = s - x * G.n2n3n4;
    uint32_t t = G.d23.div(r);
    r -= t * G.n2n3;
    uint32_t z = G.d2.div(r);
    c.x = (int)x; c.t = (int)t; c.z = (int)z; c.y = (int)(r - z * (uint32_t)G.n[1]);
    return c;
}
__device__ __forceinline__ uint32_t crd2lex(const Geom &G, const Crd &c)
{
    return (uint32_t)c.y + (uint32_t)c.z * (uint32_t)G.n[1] + (uint32_t)c.t * G.n2n3 + (uint32_t)c.x * G.n2n3n4;
}
__device__ __forceinline__ Crd step_plus(const Geom &G, Crd c, int d)
{
    switch (d) {
    case 0: c.x = (c.x + 1 == G.n[0]) ? 0 : c.x + 1; break;
    case 1: c.y = (c.y + 1 == G.n[1]) ? 0 : c.y + 1; break;
    case 2: c.z = (c.z + 1 == G.n[2]) ? 0 : c.z + 1; break;
    default: c.t = (c.t + 1 == G.n[3]) ? 0 : c.t + 1; break;
    }
    return c;
}
__device__ __forceinline__ Crd step_minus(const Geom &G, Crd c, int d)
{
    switch (d) {
    case 0: c.x = (c.x == 0) ? G.n[0] - 1 : c.x - 1; break;
    case 1: c.y = (c.y == 0) ? G.n[1] - 1 : c.y - 1; break;
    case 2: c.z = (c.z == 0) ? G.n[2] - 1 : c.z - 1; break;
    default: c.t = (c.t == 0) ? G.n[3] - 1 : c.t - 1; break;
    }
    return c;
}
__device__ __forceinline__ int parity_of(const Crd &c) { return (c.x + c.y + c.z + c.t) & 1; }
// checkerboard element index of a site whose parity is known
__device__ __forceinline__ uint32_t cb_index(const Geom &G, const Crd &c, int par)
{
    return (uint32_t)par * G.cb + (crd2lex(G, c) >> 1);
}

// ------------------------------------------------------------ link access
template <typename Real> struct V4;
template <> struct V4<float> { using T = float4; };
template <> struct V4<double> { using T = double4; };

__device__ __forceinline__ R4<float> ldg4(const float4 *p)
{
    float4 v = __ldg(p);
    return { v.x, v.y, v.z, v.w };
}
__device__ __forceinline__ R4<double> ldg4(const double4 *p)
{
    const double2 *q = reinterpret_cast<const double2 *>(p);
    double2 a = __ldg(q), b = __ldg(q + 1);
    return { a.x, a.y, b.x, b.y };
}
__device__ __forceinline__ R4<float> ld4(const float4 *p)
{
    float4 v = *p;
    return { v.x, v.y, v.z, v.w };
}
__device__ __forceinline__ R4<double> ld4(const double4 *p)
{
    const double2 *q = reinterpret_cast<const double2 *>(p);
    double2 a = q[0], b = q[1];
    return { a.x, a.y, b.x, b.y };
}
__device__ __forceinline__ void st4(float4 *p, const R4<float> &v) { *p = make_float4(v.x, v.y, v.z, v.w); }
__device__ __forceinline__ void st4(double4 *p, const R4<double> &v)
{
    double2 *q = reinterpret_cast<double2 *>(p);
    q[0] = make_double2(v.x, v.y);
    q[1] = make_double2(v.z, v.w);
}

template <typename Real>
struct Field {
    typename V4<Real>::T *p;
    uint32_t pstride;
    __device__ __forceinline__ G3<Real> ldg3(int dir, uint32_t e) const
    {
        G3<Real> m;
        m.uv1 = ldg4(p + (size_t)dir * pstride + e);
        m.uv2 = ldg4(p + (size_t)(dir + 4) * pstride + e);
        m.uv3 = ldg4(p + (size_t)(dir + 8) * pstride + e);
        return m;
    }
    __device__ __forceinline__ G3<Real> ld3(int dir, uint32_t e) const
    {
        G3<Real> m;
        m.uv1 = ld4(p + (size_t)dir * pstride + e);
        m.uv2 = ld4(p + (size_t)(dir + 4) * pstride + e);
        m.uv3 = ld4(p + (size_t)(dir + 8) * pstride + e);
        return m;
    }
    __device__ __forceinline__ void st3(int dir, uint32_t e, const G3<Real> &m) const
    {
        st4(p + (size_t)dir * pstride + e, m.uv1);
        st4(p + (size_t)(dir + 4) * pstride + e, m.uv2);
        st4(p + (size_t)(dir + 8) * pstride + e, m.uv3);
    }
    __device__ __forceinline__ R4<Real> ldg2(int dir, uint32_t e) const { return ldg4(p + (size_t)dir * pstride + e); }
    __device__ __forceinline__ R4<Real> ld2(int dir, uint32_t e) const { return ld4(p + (size_t)dir * pstride + e); }
    __device__ __forceinline__ void st2(int dir, uint32_t e, const R4<Real> &m) const { st4(p + (size_t)dir * pstride + e, m); }
};

// ------------------------------------------------------------ PRN sources
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}
// 32-bit word -> odd multiple of 2^-24 in (0,1), exact in float
__device__ __forceinline__ float u32_to_unit(uint32_t w) { return (float)((w >> 8) | 1u) * 5.9604644775390625e-8f; }

// reference layout: the thread reads float4 prns[GID + k*PRNGSTEP]
// (indprng, su3_update_cl.cl:613-617,644-648,667)
template <typename Real>
struct PrnBuffer {
    static constexpr bool GID = false;
    const float4 *prns;
    uint32_t idx, step;
    __device__ __forceinline__ R4<Real> next()
    {
        float4 q = __ldg(prns + idx);
        idx += step;
        return { (Real)q.x, (Real)q.y, (Real)q.z, (Real)q.w };
    }
    __device__ __forceinline__ R4<Real> try_quad() { return next(); }
    __device__ __forceinline__ R4<Real> dir_quad() { return next(); }
    __device__ __forceinline__ void skip() { idx += step; }
};

// in-register counter stream: quad k of thread t in phase p is
// Philox4x32-10 of (t, k, p_lo, p_hi) under the run's key
template <typename Real>
struct PrnPhilox {
    static constexpr bool GID = false;
    uint2 key;
    uint32_t t, k, plo, phi;
    __device__ __forceinline__ R4<Real> next()
    {
        uint4 w = philox4x32_10(make_uint4(t, k, plo, phi), key);
        k++;
        return { (Real)u32_to_unit(w.x), (Real)u32_to_unit(w.y), (Real)u32_to_unit(w.z), (Real)u32_to_unit(w.w) };
    }
    __device__ __forceinline__ R4<Real> try_quad() { return next(); }
    __device__ __forceinline__ R4<Real> dir_quad() { return next(); }
    __device__ __forceinline__ void skip() { k++; }
};

// INTS=2 deterministic "random" numbers from the site index
// (su3_update_cl.cl:598-611,631-642; su2_update_cl.cl:463-476,495-506)
template <typename Real>
struct PrnGid {
    static constexpr bool GID = true;
    double g, V;
    int nhit;
    __device__ __forceinline__ R4<Real> try_quad()
    {
        double a = 0.005 * (1 + nhit);
        return { (Real)fabs(sin((a + 270.0 / V) * g)), (Real)fabs(cos((a + 60.0 / V) * g)),
                 (Real)fabs(sin((a - 150.0 / V) * g)), (Real)fabs(cos((a - 380.0 / V) * g)) };
    }
    __device__ __forceinline__ R4<Real> dir_quad()
    {
        return { (Real)fabs(cos((0.08 - 270.0 / V) * g)), (Real)fabs(sin((0.08 - 60.0 / V) * g)),
                 (Real)fabs(cos((0.08 + 150.0 / V) * g)), (Real)fabs(sin((0.08 + 380.0 / V) * g)) };
    }
    __device__ __forceinline__ void skip() {}
};

}  // namespace qg
