// qg_fields.cu -- whole-field kernels: start configurations, global
// reunitarisation, reference-layout <-> checkerboard conversion and the
// observables (plaquette/action, Polyakov loop, Wilson loops) with
// deterministic two-pass FP64 reductions.
#include "qg_internal.h"
#include "qg_observe.cuh"

namespace qg {

Geom make_geom(const int n[4])
{
    Geom G;
    for (int i = 0; i < 4; i++) G.n[i] = n[i];
    G.V = (uint32_t)n[0] * n[1] * n[2] * n[3];
    G.half = G.V / 2;
    G.cb = (G.half + 127u) & ~127u;
    G.pstride = 2 * G.cb;
    G.n2n3 = (uint32_t)n[1] * n[2];
    G.n2n3n4 = G.n2n3 * n[3];
    G.d2 = make_fastdiv((uint32_t)n[1]);
    G.d23 = make_fastdiv(G.n2n3);
    G.d234 = make_fastdiv(G.n2n3n4);
    return G;
}

static __device__ __forceinline__ uint32_t native_index(const Geom &G, uint32_t s, const Crd &c)
{
    return (uint32_t)parity_of(c) * G.cb + (s >> 1);
}

// ---------------------------------------------------------------- starts
// lattice_init_cold (suncl.cl:164-187)
template <int NC, typename Real>
__global__ void k_init_cold(Field<Real> U, Geom G)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= G.V) return;
    Crd c = lex2crd(G, s);
    uint32_t e = native_index(G, s, c);
    for (int mu = 0; mu < 4; mu++) {
        if (NC == 3) {
            G3<Real> m;
            m.uv1 = { 1, 0, 0, 0 }; m.uv2 = { 0, 0, 0, 0 }; m.uv3 = { 0, 1, 0, 0 };
            U.st3(mu, e, m);
        } else {
            U.st2(mu, e, R4<Real>{ 1, 0, 0, 0 });
        }
    }
}

// lattice_init_gid (suncl.cl:190-347): closed-form field, GS in Real
template <int NC, typename Real>
__global__ void k_init_gid(Field<Real> U, Geom G)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= G.V) return;
    Crd c = lex2crd(G, s);
    uint32_t e = native_index(G, s, c);
    const double V = (double)G.V, g = (double)s;
    for (int mu = 0; mu < 4; mu++) {
        const double o = (mu == 0) ? 0.001 : (mu == 1) ? 0.002 : (mu == 2) ? 0.003 : 0.004;
        if (NC == 3) {
            G3<Real> m;
            m.uv1 = { (Real)(sin((o + 10.0 / V) * g) / 2.0), (Real)(sin((o - 18.0 / V) * g) / 4.0),
                      (Real)(sin((o - 12.0 / V) * g) / 3.0), (Real)(sin((o - 16.0 / V) * g) / 3.0) };
            m.uv2 = { (Real)(cos((o - 10.0 / V) * g) / 3.0), (Real)(cos((o + 12.0 / V) * g) / 4.0),
                      (Real)(cos((o - 15.0 / V) * g) / 2.0), (Real)(cos((o - 18.0 / V) * g) / 2.0) };
            m.uv3 = { (Real)(sin((o + 15.0 / V) * g) / 3.0), (Real)(sin((o - 11.0 / V) * g) / 3.0),
                      (Real)(cos((o - 11.0 / V) * g) / 4.0), (Real)(cos((o + 16.0 / V) * g) / 2.0) };
            U.st3(mu, e, gs3<Real>(m));
        } else {
            double f1 = sin((o + 10.0 / V) * g) / 2.0;
            double f2 = cos((o - 10.0 / V) * g) / 3.0;
            double f3 = sin((o - 18.0 / V) * g) / 4.0;
            double f4 = sqrt(1.0 - f1 * f1 - f2 * f2 - f3 * f3);
            U.st2(mu, e, R4<Real>{ (Real)f1, (Real)f3, (Real)f4, (Real)f2 });
        }
    }
}

// lattice_random3 / lattice_random2 from three (one) PRN quads (not Haar;
// su3_update_cl.cl:165-225, su2_update_cl.cl:110-146)
template <int NC, typename Real>
__device__ __forceinline__ void random_link(const R4<Real> r[3], G3<Real> &m3, R4<Real> &m2)
{
    if (NC == 3) {
        Real a0[4], a1[4], a2[4], a3[4];
        const Real R1[4] = { r[0].x, r[0].y, r[0].z, r[0].w }, R2[4] = { r[1].x, r[1].y, r[1].z, r[1].w },
                   R3[4] = { r[2].x, r[2].y, r[2].z, r[2].w };
#pragma unroll
        for (int k = 0; k < 3; k++) {
            Real alpha = RC<Real>::PI * R1[k], phi = RC<Real>::PI2 * R2[k];
            Real costh = (Real)2 * R3[k] - (Real)1;
            Real sinth = RC<Real>::sq((Real)1 - costh * costh);
            Real sinal = RC<Real>::sn(alpha);
            a0[k] = RC<Real>::cs(alpha);
            Real sinph = RC<Real>::sn(phi), cosph = RC<Real>::cs(phi);
            Real t1 = sinal * sinth;
            a1[k] = t1 * cosph; a2[k] = t1 * sinph; a3[k] = sinal * costh;
        }
        const int X = 0, Y = 1, Z = 2;
        m3.uv1.x = a0[X] * a0[Y] - a3[X] * a3[Y];
        m3.uv2.x = a0[Y] * a3[X] + a0[X] * a3[Y];
        m3.uv1.y = -a0[X] * a1[Y] * a1[Z] + a0[Z] * a2[X] - a0[X] * a2[Y] * a2[Z] - a1[Z] * a2[Y] * a3[X] + a1[Y] * a2[Z] * a3[X] - a1[X] * a3[Z];
        m3.uv2.y = a0[Z] * a1[X] + a0[X] * a1[Z] * a2[Y] - a0[X] * a1[Y] * a2[Z] - a1[Y] * a1[Z] * a3[X] - a2[Y] * a2[Z] * a3[X] + a2[X] * a3[Z];
        m3.uv1.z = -a1[X] * a1[Z] + a0[X] * a0[Z] * a2[Y] + a2[X] * a2[Z] - a0[Z] * a1[Y] * a3[X] + a0[X] * a1[Y] * a3[Z] + a2[Y] * a3[X] * a3[Z];
        m3.uv2.z = a0[X] * a0[Z] * a1[Y] + a1[Z] * a2[X] + a1[X] * a2[Z] + a0[Z] * a2[Y] * a3[X] - a0[X] * a2[Y] * a3[Z] + a1[Y] * a3[X] * a3[Z];
        m3.uv1.w = -a0[Z] * a1[X] * a1[Y] - a0[Z] * a2[X] * a2[Y] + a0[X] * a2[Z] + a1[Z] * a3[X] - a1[Y] * a2[X] * a3[Z] + a1[X] * a2[Y] * a3[Z];
        m3.uv2.w = a0[X] * a1[Z] - a0[Z] * a1[Y] * a2[X] + a0[Z] * a1[X] * a2[Y] - a2[Z] * a3[X] + a1[X] * a1[Y] * a3[Z] + a2[X] * a2[Y] * a3[Z];
        m3.uv3.x = -a0[Y] * a2[X] - a1[X] * a3[Y];
        m3.uv3.z = a0[Y] * a1[X] - a2[X] * a3[Y];
        m3.uv3.y = a0[X] * a0[Z] + a1[Y] * a1[Z] * a2[X] - a1[X] * a1[Z] * a2[Y] + a1[X] * a1[Y] * a2[Z] + a2[X] * a2[Y] * a2[Z] + a3[X] * a3[Z];
        m3.uv3.w = -a1[X] * a1[Y] * a1[Z] - a1[Z] * a2[X] * a2[Y] + a1[Y] * a2[X] * a2[Z] - a1[X] * a2[Y] * a2[Z] - a0[Z] * a3[X] + a0[X] * a3[Z];
    } else {
        Real alpha = RC<Real>::PI * r[0].x, phi = RC<Real>::PI2 * r[0].y;
        Real costh = (Real)2 * r[0].z - (Real)1;
        Real sinth = RC<Real>::sq((Real)1 - costh * costh);
        Real sinal = RC<Real>::sn(alpha), a0 = RC<Real>::cs(alpha);
        Real sinph = RC<Real>::sn(phi), cosph = RC<Real>::cs(phi);
        Real t1 = sinal * sinth;
        m2 = { a0, t1 * sinph, sinal * costh, t1 * cosph };
    }
}

// lattice_init_hot_{X,Y,Z,T} (suncl.cl:56-161): quads GID + {0,1,2}*ROWSIZE
// of the reference-layout batch, one direction per launch
template <int NC, typename Real>
__global__ void k_init_hot_ref(Field<Real> U, Geom G, int mu, const float4 *prns, uint32_t rowsize)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= G.V) return;
    Crd c = lex2crd(G, s);
    uint32_t e = native_index(G, s, c);
    R4<Real> r[3];
    for (int j = 0; j < 3; j++) {
        float4 q = prns[s + (size_t)j * rowsize];
        r[j] = { (Real)q.x, (Real)q.y, (Real)q.z, (Real)q.w };
    }
    G3<Real> m3; R4<Real> m2;
    random_link<NC, Real>(r, m3, m2);
    if (NC == 3) U.st3(mu, e, m3); else U.st2(mu, e, m2);
}

// same start from the counter stream: quad j of (site, dir) is
// Philox(site, 4*j + dir, ~0, ~0)
template <int NC, typename Real>
__global__ void k_init_hot_philox(Field<Real> U, Geom G, uint2 key)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= G.V) return;
    Crd c = lex2crd(G, s);
    uint32_t e = native_index(G, s, c);
    for (int mu = 0; mu < 4; mu++) {
        R4<Real> r[3];
        for (int j = 0; j < 3; j++) {
            uint4 w = philox4x32_10(make_uint4(s, 4u * j + mu, 0xFFFFFFFFu, 0xFFFFFFFFu), key);
            r[j] = { (Real)u32_to_unit(w.x), (Real)u32_to_unit(w.y), (Real)u32_to_unit(w.z), (Real)u32_to_unit(w.w) };
        }
        G3<Real> m3; R4<Real> m2;
        random_link<NC, Real>(r, m3, m2);
        if (NC == 3) U.st3(mu, e, m3); else U.st2(mu, e, m2);
    }
}

// Haar-distributed start: SU(2) = normalised 4-vector of Gaussians; SU(3) =
// Gram-Schmidt of two complex Gaussian rows (third row by conj cross
// product), Gaussians by Box-Muller from the counter stream (~1, ~0 tag).
template <int NC, typename Real>
__global__ void k_init_haar(Field<Real> U, Geom G, uint2 key)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= G.V) return;
    Crd c = lex2crd(G, s);
    uint32_t e = native_index(G, s, c);
    for (int mu = 0; mu < 4; mu++) {
        double gz[12];
        for (int j = 0; j < 3; j++) {
            uint4 w = philox4x32_10(make_uint4(s, 4u * j + mu, 0xFFFFFFFEu, 0xFFFFFFFFu), key);
            double u1 = u32_to_unit(w.x), u2 = u32_to_unit(w.y), u3 = u32_to_unit(w.z), u4 = u32_to_unit(w.w);
            double r1 = sqrt(-2.0 * log(u1)), r2 = sqrt(-2.0 * log(u3));
            gz[4 * j + 0] = r1 * cos(6.283185307179586 * u2);
            gz[4 * j + 1] = r1 * sin(6.283185307179586 * u2);
            gz[4 * j + 2] = r2 * cos(6.283185307179586 * u4);
            gz[4 * j + 3] = r2 * sin(6.283185307179586 * u4);
        }
        if (NC == 3) {
            G3<double> m;
            m.uv1 = { gz[0], gz[2], gz[4], gz[11] };
            m.uv2 = { gz[1], gz[3], gz[5], gz[10] };
            m.uv3 = { gz[6], gz[8], gz[7], gz[9] };
            G3<double> q = gs3<double>(m);
            G3<Real> r;
            r.uv1 = { (Real)q.uv1.x, (Real)q.uv1.y, (Real)q.uv1.z, (Real)q.uv1.w };
            r.uv2 = { (Real)q.uv2.x, (Real)q.uv2.y, (Real)q.uv2.z, (Real)q.uv2.w };
            r.uv3 = { (Real)q.uv3.x, (Real)q.uv3.y, (Real)q.uv3.z, (Real)q.uv3.w };
            U.st3(mu, e, r);
        } else {
            double n = sqrt(gz[0] * gz[0] + gz[1] * gz[1] + gz[2] * gz[2] + gz[3] * gz[3]);
            U.st2(mu, e, R4<Real>{ (Real)(gz[0] / n), (Real)(gz[1] / n), (Real)(gz[2] / n), (Real)(gz[3] / n) });
        }
    }
}

template <int NC, typename Real>
static cudaError_t init_T(const Geom &G, void *links, int kind, int dir, const float4 *prns, uint32_t rowsize,
                          uint2 key, cudaStream_t s)
{
    Field<Real> U;
    U.p = reinterpret_cast<typename V4<Real>::T *>(links);
    U.pstride = G.pstride;
    unsigned nb = (G.V + 127) / 128;
    switch (kind) {
    case INIT_COLD: k_init_cold<NC, Real><<<nb, 128, 0, s>>>(U, G); break;
    case INIT_GID: k_init_gid<NC, Real><<<nb, 128, 0, s>>>(U, G); break;
    case INIT_HOT_REF: k_init_hot_ref<NC, Real><<<nb, 128, 0, s>>>(U, G, dir, prns, rowsize); break;
    case INIT_HOT_PHILOX: k_init_hot_philox<NC, Real><<<nb, 128, 0, s>>>(U, G, key); break;
    default: k_init_haar<NC, Real><<<nb, 128, 0, s>>>(U, G, key); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_init(const Geom &G, void *links, int group, int prec, int kind, int dir, const float4 *prns,
                        uint32_t rowsize, uint2 key, cudaStream_t s)
{
    if (group == 3)
        return prec ? init_T<3, double>(G, links, kind, dir, prns, rowsize, key, s)
                    : init_T<3, float>(G, links, kind, dir, prns, rowsize, key, s);
    return prec ? init_T<2, double>(G, links, kind, dir, prns, rowsize, key, s)
                : init_T<2, float>(G, links, kind, dir, prns, rowsize, key, s);
}

// ------------------------------------------------------- reunitarisation
// lattice_GramSchmidt kernel (suncl.cl:350-396); Acc = double for the FP64
// variant on FP32 links
template <int NC, typename Real, typename Acc>
__global__ void k_gramschmidt(Field<Real> U, Geom G)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * G.cb) return;
    uint32_t h = (i < G.cb) ? i : i - G.cb;
    if (h >= G.half) return;
    gs_site<NC, Real, Acc>(U, i);
}

cudaError_t launch_gramschmidt(const Geom &G, void *links, int group, int prec, int fp64, cudaStream_t s)
{
    unsigned nb = (2 * G.cb + 127) / 128;
    if (prec) {
        Field<double> U{ reinterpret_cast<double4 *>(links), G.pstride };
        if (group == 3) k_gramschmidt<3, double, double><<<nb, 128, 0, s>>>(U, G);
        else k_gramschmidt<2, double, double><<<nb, 128, 0, s>>>(U, G);
    } else {
        Field<float> U{ reinterpret_cast<float4 *>(links), G.pstride };
        if (group == 3) {
            if (fp64) k_gramschmidt<3, float, double><<<nb, 128, 0, s>>>(U, G);
            else k_gramschmidt<3, float, float><<<nb, 128, 0, s>>>(U, G);
        } else {
            if (fp64) k_gramschmidt<2, float, double><<<nb, 128, 0, s>>>(U, G);
            else k_gramschmidt<2, float, float><<<nb, 128, 0, s>>>(U, G);
        }
    }
    return cudaGetLastError();
}

// ------------------------------------------------------------ field check
// links (thread = element of both parities, blockIdx.y = direction) whose
// stored rows are not finite, not of unit norm or not orthogonal to within
// tol: a counter the host reads (qg_field_check)
template <int NC, typename Real>
__global__ void k_field_check(Field<Real> U, Geom G, double tol, unsigned long long *bad)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const int mu = blockIdx.y;
    if (i >= 2 * G.cb) return;
    const uint32_t h = (i < G.cb) ? i : i - G.cb;
    if (h >= G.half) return;
    bool ok;
    if (NC == 3) {
        const G3<Real> m = U.ld3(mu, i);
        // row 1 = (uv1.x, uv1.y, uv1.z) + i (uv2.x, uv2.y, uv2.z); row 2 =
        // (uv3.x + i uv3.z, uv3.y + i uv3.w, uv1.w + i uv2.w)
        const double ar[3] = { m.uv1.x, m.uv1.y, m.uv1.z }, ai[3] = { m.uv2.x, m.uv2.y, m.uv2.z };
        const double br[3] = { m.uv3.x, m.uv3.y, m.uv1.w }, bi[3] = { m.uv3.z, m.uv3.w, m.uv2.w };
        double n1 = 0, n2 = 0, ore = 0, oim = 0;
        for (int k = 0; k < 3; k++) {
            n1 += ar[k] * ar[k] + ai[k] * ai[k];
            n2 += br[k] * br[k] + bi[k] * bi[k];
            ore += ar[k] * br[k] + ai[k] * bi[k];
            oim += ai[k] * br[k] - ar[k] * bi[k];
        }
        ok = isfinite(n1) && isfinite(n2) && isfinite(ore) && isfinite(oim) && fabs(n1 - 1.0) <= tol &&
             fabs(n2 - 1.0) <= tol && ore * ore + oim * oim <= tol * tol;
    } else {
        const R4<Real> q = U.ld2(mu, i);
        const double n = (double)q.x * q.x + (double)q.y * q.y + (double)q.z * q.z + (double)q.w * q.w;
        ok = isfinite(n) && fabs(n - 1.0) <= tol;
    }
    if (!ok) atomicAdd(bad, 1ull);
}

cudaError_t launch_field_check(const Geom &G, const void *links, int group, int prec, double tol,
                               unsigned long long *bad, cudaStream_t s)
{
    const dim3 grid((2 * G.cb + 127) / 128, 4);
    if (prec) {
        Field<double> U{ (double4 *)links, G.pstride };
        if (group == 3) k_field_check<3, double><<<grid, 128, 0, s>>>(U, G, tol, bad);
        else k_field_check<2, double><<<grid, 128, 0, s>>>(U, G, tol, bad);
    } else {
        Field<float> U{ (float4 *)links, G.pstride };
        if (group == 3) k_field_check<3, float><<<grid, 128, 0, s>>>(U, G, tol, bad);
        else k_field_check<2, float><<<grid, 128, 0, s>>>(U, G, tol, bad);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------- layout convert
template <typename V>
__global__ void k_to_native(Geom G, const V *ref, V *nat, int planes, uint32_t rowsize)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= G.V) return;
    Crd c = lex2crd(G, s);
    uint32_t e = native_index(G, s, c);
    for (int k = 0; k < planes; k++) nat[(size_t)k * G.pstride + e] = ref[s + (size_t)k * rowsize];
}
template <typename V>
__global__ void k_to_ref(Geom G, const V *nat, V *ref, int planes, uint32_t rowsize)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= G.V) return;
    Crd c = lex2crd(G, s);
    uint32_t e = native_index(G, s, c);
    for (int k = 0; k < planes; k++) ref[s + (size_t)k * rowsize] = nat[(size_t)k * G.pstride + e];
}

cudaError_t launch_to_native(const Geom &G, const void *ref, void *links, int group, int prec, uint32_t rowsize,
                             cudaStream_t s)
{
    unsigned nb = (G.V + 127) / 128;
    int planes = group == 3 ? 12 : 4;
    if (prec) k_to_native<double4><<<nb, 128, 0, s>>>(G, (const double4 *)ref, (double4 *)links, planes, rowsize);
    else k_to_native<float4><<<nb, 128, 0, s>>>(G, (const float4 *)ref, (float4 *)links, planes, rowsize);
    return cudaGetLastError();
}
cudaError_t launch_to_ref(const Geom &G, const void *links, void *ref, int group, int prec, uint32_t rowsize,
                          cudaStream_t s)
{
    unsigned nb = (G.V + 127) / 128;
    int planes = group == 3 ? 12 : 4;
    if (prec) k_to_ref<double4><<<nb, 128, 0, s>>>(G, (const double4 *)links, (double4 *)ref, planes, rowsize);
    else k_to_ref<float4><<<nb, 128, 0, s>>>(G, (const float4 *)links, (float4 *)ref, planes, rowsize);
    return cudaGetLastError();
}

// ------------------------------------------------------------ observables
// lattice_measurement_plq + lattice_measurement (sun_measurements_cl.cl:
// 55-184,1178-1311): per-site plaquette and action sums, block partials
// TW: twisted boundaries possible; without it the per-link twist tests
// fold away at compile time
template <int NC, typename Real, bool TW>
__global__ void __launch_bounds__(256) k_plaquette(Field<Real> U, Geom G, const double *params, int twist,
                                                    double *partials)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    double v[4] = { 0, 0, 0, 0 };
    if (s < G.V) plaq_site<NC, Real>(U, G, params, TW ? twist : 0, s, v);
    block_sum_store<4>(v, partials);
}

uint32_t plaq_blocks(const Geom &G) { return (G.V + 255) / 256; }

cudaError_t launch_plaquette(const Geom &G, const void *links, int group, int prec, const double *params, int twist,
                             double *partials, double *out, cudaStream_t s)
{
    uint32_t nb = plaq_blocks(G);
    if (prec) {
        Field<double> U{ (double4 *)links, G.pstride };
#define QG_PLQ(NC, R) (twist ? k_plaquette<NC, R, true><<<nb, 256, 0, s>>>(U, G, params, twist, partials) \
                             : k_plaquette<NC, R, false><<<nb, 256, 0, s>>>(U, G, params, twist, partials))
        if (group == 3) QG_PLQ(3, double);
        else QG_PLQ(2, double);
    } else {
        Field<float> U{ (float4 *)links, G.pstride };
        if (group == 3) QG_PLQ(3, float);
        else QG_PLQ(2, float);
    }
#undef QG_PLQ
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_reduce(partials, nb, 4, out, s);
}

// the plaquette with FP32 products (QG_MEAS_PLAQUETTE_F32): same blocks,
// partials and reduction as k_plaquette; FP64 links take k_plaquette
template <int NC, bool TW>
__global__ void __launch_bounds__(256) k_plaquette_f32(Field<float> U, Geom G, const double *params, int twist,
                                                        double *partials)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    double v[4] = { 0, 0, 0, 0 };
    if (s < G.V) plaq_site_f32<NC>(U, G, params, TW ? twist : 0, lex2crd(G, s), v);
    block_sum_store<4>(v, partials);
}

cudaError_t launch_plaquette_f32(const Geom &G, const void *links, int group, int prec, const double *params,
                                 int twist, double *partials, double *out, cudaStream_t s)
{
    if (prec) return launch_plaquette(G, links, group, prec, params, twist, partials, out, s);
    uint32_t nb = plaq_blocks(G);
    Field<float> U{ (float4 *)links, G.pstride };
    if (group == 3) {
        if (twist) k_plaquette_f32<3, true><<<nb, 256, 0, s>>>(U, G, params, twist, partials);
        else k_plaquette_f32<3, false><<<nb, 256, 0, s>>>(U, G, params, twist, partials);
    } else {
        if (twist) k_plaquette_f32<2, true><<<nb, 256, 0, s>>>(U, G, params, twist, partials);
        else k_plaquette_f32<2, false><<<nb, 256, 0, s>>>(U, G, params, twist, partials);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_reduce(partials, nb, 4, out, s);
}

// lattice_polyakov (polyakov.cl:54-140): one thread per spatial site
template <int NC, typename Real>
__global__ void __launch_bounds__(256) k_polyakov(Field<Real> U, Geom G, double *partials)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[4] = { 0, 0, 0, 0 };
    if (i < (uint32_t)G.n[0] * G.n[1] * G.n[2]) poly_site<NC, Real>(U, G, i, v);
    block_sum_store<4>(v, partials);
}

uint32_t poly_blocks(const Geom &G) { return ((uint32_t)G.n[0] * G.n[1] * G.n[2] + 255) / 256; }

cudaError_t launch_polyakov(const Geom &G, const void *links, int group, int prec, double *partials, double *out,
                            cudaStream_t s)
{
    uint32_t nb = poly_blocks(G);
    if (prec) {
        Field<double> U{ (double4 *)links, G.pstride };
        if (group == 3) k_polyakov<3, double><<<nb, 256, 0, s>>>(U, G, partials);
        else k_polyakov<2, double><<<nb, 256, 0, s>>>(U, G, partials);
    } else {
        Field<float> U{ (float4 *)links, G.pstride };
        if (group == 3) k_polyakov<3, float><<<nb, 256, 0, s>>>(U, G, partials);
        else k_polyakov<2, float><<<nb, 256, 0, s>>>(U, G, partials);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_reduce(partials, nb, 4, out, s);
}

// One-pass measurements: the per-site work once, the totals exactly as
// k_plaquette / k_polyakov (same blocks, same reduction), the site values
// kept in a device buffer, then the per-slice sums of every axis from that
// buffer in k_profile's order -- so the numbers equal the separate
// qg_measure / qg_measure_*_profile calls bit for bit.
template <int NC, typename Real, bool TW>
__global__ void __launch_bounds__(256) k_plaq_sites(Field<Real> U, Geom G, const double *params, int twist,
                                                     double *partials, double *sites)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    double v[4] = { 0, 0, 0, 0 };
    if (s < G.V) {
        plaq_site<NC, Real>(U, G, params, TW ? twist : 0, s, v);
        sites[s] = v[2];                                 // spatial action of the site
        sites[(size_t)G.V + s] = v[3];                   // temporal
    }
    block_sum_store<4>(v, partials);
}
template <int NC, typename Real>
__global__ void __launch_bounds__(256) k_poly_sites(Field<Real> U, Geom G, double *partials, double *sites)
{
    const uint32_t Vs = (uint32_t)G.n[0] * G.n[1] * G.n[2];
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[4] = { 0, 0, 0, 0 };
    if (i < Vs) {
        poly_site<NC, Real>(U, G, i, v);
        sites[i] = v[0];
        sites[(size_t)Vs + i] = v[1];
    }
    block_sum_store<4>(v, partials);
}
// k_profile's loop over the stored site values (KIND 0: action per lattice
// site, lexicographic index; KIND 1: Polyakov trace per spatial site,
// i = y + N2 (z + N3 x))
template <int KIND>
__global__ void __launch_bounds__(256) k_bin_sites(const double *sites, Geom G, int axis, uint32_t per_slice,
                                                    uint32_t chunks, double *partials)
{
    const int k = (int)(blockIdx.x / chunks);
    const uint32_t j0 = (blockIdx.x % chunks) * 1024u;
    const uint32_t j1 = min(per_slice, j0 + 1024u);
    const size_t n = KIND == 0 ? (size_t)G.V : (size_t)G.n[0] * G.n[1] * G.n[2];
    double acc[2] = { 0, 0 };
    for (uint32_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        const Crd c = slice_site(G, axis, k, j, KIND == 1);
        const size_t s = KIND == 0 ? crd2lex(G, c) : (size_t)c.y + (size_t)G.n[1] * (c.z + (size_t)G.n[2] * c.x);
        acc[0] += sites[s];
        acc[1] += sites[n + s];
    }
    block_sum_store<2>(acc, partials);
}

// F_munu (FMUNU / F0MU lattice_measurement_plq, sun_measurements_cl.cl:
// 712-1175 and reduce_measurement_plq_double2 :1313-1357): 12 sums
template <int NC, typename Real, bool TW>
__global__ void __launch_bounds__(256) k_fmunu(Field<Real> U, Geom G, const double *params, int twist, int field,
                                                int i1, int i2, double *partials)
{
    if (!TW) twist = 0;                  // untwisted: the twist tests fold away
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    double v[12] = { 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0 };
    if (s < G.V) fmunu_site<NC, Real>(U, G, params, twist, s, field, i1, i2, v);
    block_sum_store<12>(v, partials);
}

uint32_t fmunu_partials(const Geom &G) { return plaq_blocks(G) * 12; }

cudaError_t launch_fmunu(const Geom &G, const void *links, int group, int prec, const double *params, int twist,
                         int field, int i1, int i2, double *partials, double *out, cudaStream_t s)
{
    uint32_t nb = plaq_blocks(G);
    if (prec) {
        Field<double> U{ (double4 *)links, G.pstride };
        if (group == 3) (twist ? k_fmunu<3, double, true><<<nb, 256, 0, s>>>(U, G, params, twist, field, i1, i2, partials) : k_fmunu<3, double, false><<<nb, 256, 0, s>>>(U, G, params, twist, field, i1, i2, partials));
        else (twist ? k_fmunu<2, double, true><<<nb, 256, 0, s>>>(U, G, params, twist, field, i1, i2, partials) : k_fmunu<2, double, false><<<nb, 256, 0, s>>>(U, G, params, twist, field, i1, i2, partials));
    } else {
        Field<float> U{ (float4 *)links, G.pstride };
        if (group == 3) (twist ? k_fmunu<3, float, true><<<nb, 256, 0, s>>>(U, G, params, twist, field, i1, i2, partials) : k_fmunu<3, float, false><<<nb, 256, 0, s>>>(U, G, params, twist, field, i1, i2, partials));
        else (twist ? k_fmunu<2, float, true><<<nb, 256, 0, s>>>(U, G, params, twist, field, i1, i2, partials) : k_fmunu<2, float, false><<<nb, 256, 0, s>>>(U, G, params, twist, field, i1, i2, partials));
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_reduce(partials, nb, 12, out, s);
}

// Profiles along x, y or z (lattice_action_diff_{x,y,z},
// sun_measurements_cl.cl:187-615 + reduce_action_diff_*_double2 :629-710;
// lattice_polyakov_diff_{x,y,z}, polyakov.cl:142-402 + reduce :434-569):
// block b covers kProfileChunk consecutive sites of slice b / chunks, and
// the second pass sums each slice's chunks in order (deterministic).
// KIND 0: spatial and temporal action over all sites of the slice;
// KIND 1: Re, Im Polyakov trace over the spatial sites of the slice.
constexpr uint32_t kProfileChunk = 1024;

template <int NC, typename Real, int KIND, bool TW>
__global__ void __launch_bounds__(256) k_profile(Field<Real> U, Geom G, const double *params, int twist, int axis,
                                                  uint32_t per_slice, uint32_t chunks, double *partials)
{
    if (!TW) twist = 0;                  // untwisted: the twist tests fold away
    const int k = (int)(blockIdx.x / chunks);
    const uint32_t j0 = (blockIdx.x % chunks) * kProfileChunk;
    const uint32_t j1 = min(per_slice, j0 + kProfileChunk);
    double acc[2] = { 0, 0 };
    for (uint32_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        const Crd c = slice_site(G, axis, k, j, KIND == 1);
        double v[4];
        if (KIND == 0) {
            plaq_site_c<NC, Real>(U, G, params, twist, c, v);
            acc[0] += v[2]; acc[1] += v[3];
        } else {
            poly_site_c<NC, Real>(U, G, c, v);
            acc[0] += v[0]; acc[1] += v[1];
        }
    }
    block_sum_store<2>(acc, partials);
}
__global__ void __launch_bounds__(256) k_profile_reduce(const double *partials, uint32_t chunks, double *out)
{
    reduce_partials(partials + (size_t)blockIdx.x * chunks * 2, chunks, 2, out + 2 * blockIdx.x);
}

static uint32_t profile_per_slice(const Geom &G, int axis, int kind)
{
    uint32_t n = (uint32_t)G.n[0] * G.n[1] * G.n[2] * (kind == 0 ? G.n[3] : 1);
    return n / (uint32_t)G.n[axis];
}
uint32_t profile_partials(const Geom &G)
{
    uint32_t m = 0;
    for (int axis = 0; axis < 3; axis++)
        for (int kind = 0; kind < 2; kind++) {
            uint32_t chunks = (profile_per_slice(G, axis, kind) + kProfileChunk - 1) / kProfileChunk;
            m = max(m, chunks * (uint32_t)G.n[axis] * 2);
        }
    return m;
}

template <int NC, typename Real>
static void profile_kernel(int kind, uint32_t nb, const Field<Real> &U, const Geom &G, const double *params,
                           int twist, int axis, uint32_t per, uint32_t chunks, double *partials, cudaStream_t s)
{
    if (kind == 0 && twist) k_profile<NC, Real, 0, true><<<nb, 256, 0, s>>>(U, G, params, twist, axis, per, chunks, partials);
    else if (kind == 0) k_profile<NC, Real, 0, false><<<nb, 256, 0, s>>>(U, G, params, twist, axis, per, chunks, partials);
    else k_profile<NC, Real, 1, false><<<nb, 256, 0, s>>>(U, G, params, twist, axis, per, chunks, partials);
}

cudaError_t launch_profile(const Geom &G, const void *links, int group, int prec, const double *params, int twist,
                           int kind, int axis, double *partials, double *out, cudaStream_t s)
{
    const uint32_t per = profile_per_slice(G, axis, kind);
    const uint32_t chunks = (per + kProfileChunk - 1) / kProfileChunk;
    const uint32_t nb = chunks * (uint32_t)G.n[axis];
    if (prec) {
        Field<double> U{ (double4 *)links, G.pstride };
        if (group == 3) profile_kernel<3, double>(kind, nb, U, G, params, twist, axis, per, chunks, partials, s);
        else profile_kernel<2, double>(kind, nb, U, G, params, twist, axis, per, chunks, partials, s);
    } else {
        Field<float> U{ (float4 *)links, G.pstride };
        if (group == 3) profile_kernel<3, float>(kind, nb, U, G, params, twist, axis, per, chunks, partials, s);
        else profile_kernel<2, float>(kind, nb, U, G, params, twist, axis, per, chunks, partials, s);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_profile_reduce<<<G.n[axis], 256, 0, s>>>(partials, chunks, out);
    return cudaGetLastError();
}

size_t sites_buffer_doubles(const Geom &G) { return 2 * (size_t)G.V; }

cudaError_t launch_measure_all(const Geom &G, const void *links, int group, int prec, const double *params, int twist,
                               int kind, double *partials, double *ppartials, double *sites, double *out,
                               cudaStream_t s)
{
    // totals into out[0..3], site values into `sites`
    const uint32_t Vs = (uint32_t)G.n[0] * G.n[1] * G.n[2];
    const uint32_t nb = kind == 0 ? plaq_blocks(G) : (Vs + 255) / 256;
#define QG_SITES(NC, R)                                                                                 \
    do {                                                                                                \
        Field<R> U{ (typename V4<R>::T *)links, G.pstride };                                            \
        if (kind == 0 && twist) k_plaq_sites<NC, R, true><<<nb, 256, 0, s>>>(U, G, params, twist, partials, sites); \
        else if (kind == 0) k_plaq_sites<NC, R, false><<<nb, 256, 0, s>>>(U, G, params, twist, partials, sites); \
        else k_poly_sites<NC, R><<<nb, 256, 0, s>>>(U, G, partials, sites);                            \
    } while (0)
    if (prec) { if (group == 3) QG_SITES(3, double); else QG_SITES(2, double); }
    else { if (group == 3) QG_SITES(3, float); else QG_SITES(2, float); }
#undef QG_SITES
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if ((e = launch_reduce(partials, nb, 4, out, s)) != cudaSuccess) return e;
    // per-slice sums along x, y, z into out[4 ..]
    double *o = out + 4;
    for (int axis = 0; axis < 3; axis++) {
        const uint32_t per = profile_per_slice(G, axis, kind);
        const uint32_t chunks = (per + kProfileChunk - 1) / kProfileChunk;
        const uint32_t nbk = chunks * (uint32_t)G.n[axis];
        if (kind == 0) k_bin_sites<0><<<nbk, 256, 0, s>>>(sites, G, axis, per, chunks, ppartials);
        else k_bin_sites<1><<<nbk, 256, 0, s>>>(sites, G, axis, per, chunks, ppartials);
        k_profile_reduce<<<G.n[axis], 256, 0, s>>>(ppartials, chunks, o);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        o += 2 * G.n[axis];
    }
    return cudaSuccess;
}

// lattice_measurement_wilson (wilson_loop.cl:55-454): per site and i in
// {x,y,z}, Re Tr(L_t^T(x) L_i^R(x+T t) L_t^T(x+R i)^+ L_i^R(x)^+) in FP64
template <int NC, typename Real, bool TW>
__global__ void __launch_bounds__(128) k_wilson(Field<Real> U, Geom G, int R, int T, const double *params, int twist,
                                                 double *partials)
{
    if (!TW) twist = 0;                  // untwisted: the twist tests fold away
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    double v[1] = { 0 };
    if (s < G.V) {
        const Crd c1 = lex2crd(G, s);
        Crd co = c1;
        M3<double> m1 = load_d<NC, Real>(U, G, co, 3, params, twist);
        for (int k = 1; k < T; k++) { co = step_plus(G, co, 3); m1 = mulf(m1, load_d<NC, Real>(U, G, co, 3, params, twist)); }
        const Crd c2 = step_plus(G, co, 3);
        double acc = 0;
        for (int i = 0; i < 3; i++) {
            Crd a = c1, b = c2;
            M3<double> m4 = load_d<NC, Real>(U, G, a, i, params, twist);
            M3<double> m2 = load_d<NC, Real>(U, G, b, i, params, twist);
            for (int k = 1; k < R; k++) {
                a = step_plus(G, a, i); b = step_plus(G, b, i);
                m4 = mulf(m4, load_d<NC, Real>(U, G, a, i, params, twist));
                m2 = mulf(m2, load_d<NC, Real>(U, G, b, i, params, twist));
            }
            Crd c4 = step_plus(G, a, i);
            M3<double> m3 = load_d<NC, Real>(U, G, c4, 3, params, twist);
            for (int k = 1; k < T; k++) { c4 = step_plus(G, c4, 3); m3 = mulf(m3, load_d<NC, Real>(U, G, c4, 3, params, twist)); }
            acc += retr4(m1, m2, m3, m4);
        }
        v[0] = acc;
    }
    block_sum_store<1>(v, partials);
}

cudaError_t launch_wilson(const Geom &G, const void *links, int group, int prec, int R, int T, const double *params,
                          int twist, double *partials, double *out, cudaStream_t s)
{
    uint32_t nb = (G.V + 127) / 128;
    if (prec) {
        Field<double> U{ (double4 *)links, G.pstride };
        if (group == 3) (twist ? k_wilson<3, double, true><<<nb, 128, 0, s>>>(U, G, R, T, params, twist, partials) : k_wilson<3, double, false><<<nb, 128, 0, s>>>(U, G, R, T, params, twist, partials));
        else (twist ? k_wilson<2, double, true><<<nb, 128, 0, s>>>(U, G, R, T, params, twist, partials) : k_wilson<2, double, false><<<nb, 128, 0, s>>>(U, G, R, T, params, twist, partials));
    } else {
        Field<float> U{ (float4 *)links, G.pstride };
        if (group == 3) (twist ? k_wilson<3, float, true><<<nb, 128, 0, s>>>(U, G, R, T, params, twist, partials) : k_wilson<3, float, false><<<nb, 128, 0, s>>>(U, G, R, T, params, twist, partials));
        else (twist ? k_wilson<2, float, true><<<nb, 128, 0, s>>>(U, G, R, T, params, twist, partials) : k_wilson<2, float, false><<<nb, 128, 0, s>>>(U, G, R, T, params, twist, partials));
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_reduce(partials, nb, 1, out, s);
}

// All planar Wilson loops R x T, R <= Rmax, T <= Tmax (<= 16), in one
// launch: block (bx, R-1, i) walks sites bx, bx + gridDim.x, ... and for each
// site x builds the spatial line L_i^R(x) once and extends the time lines
// L_t^T(x), L_t^T(x+R i) one link per T, so that every T <= Tmax costs only
// the top line L_i^R(x+T t).  Products in P: FP64 as k_wilson, or FP32 on
// FP32 links (traces still summed in FP64); per-block sums of the Tmax
// traces, then k_wilson_all_reduce in a fixed order.
constexpr int kWilsonMax = 16;

// All planar Wilson loops R x T (R <= Rmax, T <= Tmax) in one launch
// (lattice_measurement_wilson, wilson_loop.cl:55-454, for every R x T at
// once), products in precision P, sums in FP64.  One thread per time
// column: thread (spatial site, i, R) walks t0 = 0 .. N4-1 and keeps the
// spatial lines S(t) = L_i^R(x + t t) of the last Tmax + 1 time slices in
// a private ring in shared memory, so each line is built once per column
// (not once per (t0, T)); each term Re Tr(L_t^T(x) S(t0+T) L_t^T(x+R i)^+
// S(t0)^+) is taken as Re Tr(S(t0+T) Z_T) with Z_T = L_t^T(x+R i)^+ S(t0)^+
// L_t^T(x), which grows by one time link on each side per T (two products
// per T, no product for the term itself).  The per-thread sums w[T] live
// in shared memory.  Dynamic shared
// memory: (Tmax+1) ring entries and Tmax doubles per thread.  A ring entry
// holds the 2 x 2 block for SU(2); for SU(3) the full line in FP64, or
// with FP32 products rows 1, 2 only (row 3 rebuilt on reading; rebuilding
// an FP64 product of FP32 links would move it by their ~1e-7 departure
// from unitarity, more than FP64 products are meant to carry).
template <int NC, typename P> constexpr int kRingFloats = NC == 2 ? 8 : (sizeof(P) == 8 ? 18 : 12);

template <int NC, typename Real, typename P, bool TW>
__global__ void __launch_bounds__(128) k_wilson_cols(Field<Real> U, Geom G, int Tmax, const double *params,
                                                      int twist, double *partials)
{
    if (!TW) twist = 0;                  // untwisted: the twist tests fold away
    extern __shared__ __align__(16) unsigned char wsm[];
    constexpr int RF = kRingFloats<NC, P>;
    constexpr int ROWS = RF == 18 ? 3 : 2;        // rows stored
    const int R = blockIdx.y + 1, i = blockIdx.z;
    const int nb = blockDim.x, tid = threadIdx.x, slots = Tmax + 1;
    double *wsum = reinterpret_cast<double *>(wsm);                          // [Tmax][nb]
    P *ring = reinterpret_cast<P *>(wsm + sizeof(double) * Tmax * nb);       // [slots][RF][nb]
    auto put = [&](int slot, const M3<P> &m) {
        P *q = ring + (size_t)slot * RF * nb + tid;
#pragma unroll
        for (int a = 0; a < ROWS; a++)
#pragma unroll
            for (int b = 0; b < NC; b++) {
                q[(2 * (a * NC + b)) * nb] = m.m[a][b].re;
                q[(2 * (a * NC + b) + 1) * nb] = m.m[a][b].im;
            }
    };
    auto get = [&](int slot) {
        const P *q = ring + (size_t)slot * RF * nb + tid;
        M3<P> m;
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) m.m[a][b] = { (P)0, (P)0 };
#pragma unroll
        for (int a = 0; a < ROWS; a++)
#pragma unroll
            for (int b = 0; b < NC; b++) m.m[a][b] = { q[(2 * (a * NC + b)) * nb], q[(2 * (a * NC + b) + 1) * nb] };
        if (NC == 3 && ROWS == 2) fill_row3(m);
        return m;
    };
    for (int k = 0; k < Tmax; k++) wsum[k * nb + tid] = 0.0;
    const uint32_t Vs = (uint32_t)G.n[0] * G.n[1] * G.n[2];
    const int nt = G.n[3];
    for (uint32_t xs = blockIdx.x * blockDim.x + tid; xs < Vs; xs += gridDim.x * blockDim.x) {
        Crd c0;
        c0.y = (int)(xs % (uint32_t)G.n[1]);
        const uint32_t r = xs / (uint32_t)G.n[1];
        c0.z = (int)(r % (uint32_t)G.n[2]);
        c0.x = (int)(r / (uint32_t)G.n[2]);
        c0.t = 0;
        auto line = [&](int t) {
            Crd a = c0;
            a.t = t;
            M3<P> m = load_as<NC, Real, P>(U, G, a, i, params, twist);
            for (int k = 1; k < R; k++) { a = step_plus(G, a, i); m = mulf(m, load_as<NC, Real, P>(U, G, a, i, params, twist)); }
            return m;
        };
        Crd cy0 = c0;
        for (int k = 0; k < R; k++) cy0 = step_plus(G, cy0, i);     // x + R i
        for (int t = 0; t < Tmax; t++) put(t, line(t % nt));
        // Re Tr(L_t^T(x) S(t0+T) L_t^T(x+Ri)^+ S(t0)^+) = Re Tr(S(t0+T) Z_T)
        // with Z_T = L_t^T(x+Ri)^+ S(t0)^+ L_t^T(x), grown by one link on each
        // side per T: Z_T = b_T^+ Z_(T-1) a_T, Z_0 = S(t0)^+ (a_T, b_T the T-th
        // time links of the two columns).  Per T two products and a 9-term
        // trace; the bottom line S(t0) enters once per t0
        auto hmul = [](const M3<P> &a, const M3<P> &b) {        // a^+ b
            M3<P> r;
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) r.m[i][j] = cdot3(&a.m[0][i], 3, &b.m[0][j], 3);
            return r;
        };
        auto retr_p = [](const M3<P> &a, const M3<P> &b) {      // Re Tr(a b), summed in FP64
            double tr = 0.0;
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    tr = fma((double)a.m[k][j].re, (double)b.m[j][k].re, tr);
                    tr = fma(-(double)a.m[k][j].im, (double)b.m[j][k].im, tr);
                }
            return tr;
        };
#pragma unroll 1
        for (int t0 = 0; t0 < nt; t0++) {
            put((t0 + Tmax) % slots, line((t0 + Tmax) % nt));   // the slot of t0 - 1
            Crd cx = c0, cy = cy0;
            cx.t = t0;
            cy.t = t0;
            M3<P> z = hmul(load_as<NC, Real, P>(U, G, cy, 3, params, twist),
                           hmul(get(t0 % slots), load_as<NC, Real, P>(U, G, cx, 3, params, twist)));
#pragma unroll 1
            for (int T = 1; T <= Tmax; T++) {
                if (T > 1) {
                    cx = step_plus(G, cx, 3);
                    cy = step_plus(G, cy, 3);
                    z = mulf(hmul(load_as<NC, Real, P>(U, G, cy, 3, params, twist), z),
                             load_as<NC, Real, P>(U, G, cx, 3, params, twist));
                }
                wsum[(T - 1) * nb + tid] += retr_p(get((t0 + T) % slots), z);
            }
        }
    }
    double w[kWilsonMax];
#pragma unroll
    for (int k = 0; k < kWilsonMax; k++) w[k] = k < Tmax ? wsum[k * nb + tid] : 0.0;
    block_sum_store<kWilsonMax>(w, partials, (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x);
}

static size_t wilson_cols_smem(int group, int psize, int Tmax, int nb)
{
    const int rf = group == 2 ? 8 : (psize == 8 ? 18 : 12);
    return (size_t)nb * (sizeof(double) * Tmax + (size_t)psize * rf * (Tmax + 1));
}

static int wilson_cols_blocks(const Geom &G, int nb);

template <int NC, typename Real, typename P>
static cudaError_t wilson_cols(const Field<Real> &U, const Geom &G, int Rmax, int Tmax, const double *params,
                               int twist, double *partials, int &nbx, cudaStream_t s)
{
    const int nbk = wilson_cols_smem(NC, sizeof(P), Tmax, 128) <= 80 * 1024 ? 128 : 64;
    const size_t sm = wilson_cols_smem(NC, sizeof(P), Tmax, nbk);
    dim3 gc((unsigned)wilson_cols_blocks(G, nbk), Rmax, 3);
    nbx = (int)gc.x;
    if (twist) {
        cudaFuncSetAttribute(k_wilson_cols<NC, Real, P, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_wilson_cols<NC, Real, P, true><<<gc, nbk, sm, s>>>(U, G, Tmax, params, twist, partials);
    } else {
        cudaFuncSetAttribute(k_wilson_cols<NC, Real, P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_wilson_cols<NC, Real, P, false><<<gc, nbk, sm, s>>>(U, G, Tmax, params, twist, partials);
    }
    return cudaGetLastError();
}

// out[(R-1) Tmax + T-1] = sum over i and blocks (in that order)
__global__ void k_wilson_all_reduce(const double *partials, int nbx, int Rmax, int Tmax, double *out)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Rmax * Tmax) return;
    const int R = q / Tmax + 1, T = q % Tmax + 1;
    double s = 0.0;
    for (int i = 0; i < 3; i++)
        for (int b = 0; b < nbx; b++) s += partials[((size_t)(i * Rmax + R - 1) * nbx + b) * kWilsonMax + T - 1];
    out[q] = s;
}

int wilson_all_blocks(const Geom &G) { return (int)min((G.V + 127u) / 128u, 296u); }
// column kernel: spatial sites per (R, i) over blocks of nb threads, at most
// as many blocks as the site kernel uses (the partials are sized for that)
static int wilson_cols_blocks(const Geom &G, int nb)
{
    const uint32_t Vs = (uint32_t)G.n[0] * G.n[1] * G.n[2];
    return (int)min((Vs + nb - 1) / (uint32_t)nb, (uint32_t)wilson_all_blocks(G));
}
size_t wilson_all_partials(int nbx, int Rmax) { return (size_t)3 * Rmax * nbx * kWilsonMax; }

cudaError_t launch_wilson_all(const Geom &G, const void *links, int group, int prec, int Rmax, int Tmax,
                              int fp64_products, const double *params, int twist, double *partials, double *out,
                              cudaStream_t s)
{
    int nbx = 0;
    cudaError_t e;
    if (prec) {
        Field<double> U{ (double4 *)links, G.pstride };
        e = group == 3 ? wilson_cols<3, double, double>(U, G, Rmax, Tmax, params, twist, partials, nbx, s)
                       : wilson_cols<2, double, double>(U, G, Rmax, Tmax, params, twist, partials, nbx, s);
    } else {
        Field<float> U{ (float4 *)links, G.pstride };
        if (fp64_products)
            e = group == 3 ? wilson_cols<3, float, double>(U, G, Rmax, Tmax, params, twist, partials, nbx, s)
                           : wilson_cols<2, float, double>(U, G, Rmax, Tmax, params, twist, partials, nbx, s);
        else
            e = group == 3 ? wilson_cols<3, float, float>(U, G, Rmax, Tmax, params, twist, partials, nbx, s)
                           : wilson_cols<2, float, float>(U, G, Rmax, Tmax, params, twist, partials, nbx, s);
    }
    if (e != cudaSuccess) return e;
    k_wilson_all_reduce<<<(Rmax * Tmax + 127) / 128, 128, 0, s>>>(partials, nbx, Rmax, Tmax, out);
    return cudaGetLastError();
}

// final pass: one block sums the partials in a fixed order (deterministic)
__global__ void __launch_bounds__(1024) k_reduce(const double *partials, uint32_t nblocks, int ncomp, double *out)
{
    reduce_partials(partials, nblocks, ncomp, out);
}

cudaError_t launch_reduce(const double *partials, uint32_t nblocks, int ncomp, double *out, cudaStream_t s)
{
    k_reduce<<<1, 1024, 0, s>>>(partials, nblocks, ncomp, out);
    return cudaGetLastError();
}

__global__ void k_add_u64(uint64_t *p, uint64_t v)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *p += v;
}
// the copies of a slab halo exchange (qg_slab_halo2): blockIdx.y picks
// the copy, threads stride over its 16-byte words (coalesced both sides)
__global__ void k_slab_copy(SlabCopy c)
{
    const int k = blockIdx.y;
    const uint4 *src = c.src[k];
    uint4 *dst = c.dst[k];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.words; i += gridDim.x * blockDim.x)
        dst[i] = src[i];
}

cudaError_t launch_slab_copy(const SlabCopy &c, cudaStream_t s)
{
    if (c.n <= 0 || c.n > 6 || c.words == 0) return cudaErrorInvalidValue;
    const unsigned bx = (unsigned)min((c.words + 255u) / 256u, 148u * 4u);
    k_slab_copy<<<dim3(bx, (unsigned)c.n), 256, 0, s>>>(c);
    return cudaGetLastError();
}

cudaError_t launch_add_u64(uint64_t *p, uint64_t v, cudaStream_t s)
{
    k_add_u64<<<1, 32, 0, s>>>(p, v);
    return cudaGetLastError();
}

}  // namespace qg
