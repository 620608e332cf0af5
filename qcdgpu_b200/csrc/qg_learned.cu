// qg_learned.cu -- learned local proposal for SU(3) with an exact
// Wilson-action Metropolis step (new; the reference has only the heatbath).
//
// Move.  For link U = U_mu(x) with staple A (A does not contain U or any
// other link of the same (parity, mu) phase) each hit proposes, in turn in
// the SU(2) subgroups (1,2), (1,3), (2,3), U' = X U with
// X = exp(i eps a.sigma) embedded in the subgroup, a ~ N(0, 1)^3, and
// accepts with probability min(1, exp(-dS)), dS = -(beta/N) Re Tr((X-1) U A).
// The step eps = eps_max sigmoid(f(x)) comes from a 3-layer, 32-channel
// network f on 8 gauge-invariant features of the staple alone -- its
// norm Tr AA^+, Tr (AA^+)^2, det A and the 1x2 loop traces Tr F_nu B_nu^+
// of the forward and backward staple terms of each plane -- so eps is the
// same for U and U' and the proposal is symmetric (X and X^-1 equally
// likely): the chain is exact whatever the weights are.  A constant eps
// (all weights zero, output bias set) is the same kernel without a network.
//
// Training maximises the expected squared jump distance
// E[min(1, exp(-dS)) (eps |a|)^2] per subgroup proposal from the current
// link; its derivative in eps is analytic, and the network's backward pass,
// the block sums of the weight gradients (fixed order, deterministic) and
// the Adam step are kernels here.  Weights are stored in BF16 for the
// kernels and in FP32 for the optimiser; all sums accumulate in FP32 (the
// per-link acceptance arithmetic in FP64).
#include "qg_internal.h"
#include "qg_update.cuh"

namespace qg {

constexpr int kNF = QG_NET_FEATURES, kNH = QG_NET_HIDDEN;
constexpr int kW1 = 0, kB1 = kW1 + kNH * kNF, kW2 = kB1 + kNH, kB2 = kW2 + kNH * kNH, kW3 = kB2 + kNH,
              kB3 = kW3 + kNH, kNP = kB3 + 1;
static_assert(kNP == QG_NET_PARAMS, "parameter count");
constexpr int kTrainBlock = 64;

__device__ __forceinline__ float bf16_bits_to_float(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }
// round to nearest even (finite inputs)
__device__ __forceinline__ uint16_t float_to_bf16_bits(float f)
{
    uint32_t u = __float_as_uint(f);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

// Tr(F B^+) in the fixed order (row-major over the 9 entries)
__device__ __forceinline__ CX<float> tr_fbh(const M3<float> &F, const M3<float> &B)
{
    CX<float> r;
    r.re = F.m[0][0].re * B.m[0][0].re;
    r.re = FMA(F.m[0][0].im, B.m[0][0].im, r.re);
    r.im = F.m[0][0].im * B.m[0][0].re;
    r.im = FMA(-F.m[0][0].re, B.m[0][0].im, r.im);
#pragma unroll
    for (int q = 1; q < 9; q++) {
        const CX<float> &f = F.m[q / 3][q % 3], &b = B.m[q / 3][q % 3];
        r.re = FMA(f.re, b.re, r.re);
        r.re = FMA(f.im, b.im, r.re);
        r.im = FMA(f.im, b.re, r.im);
        r.im = FMA(-f.re, b.im, r.im);
    }
    return r;
}

// a*b - c*d (complex)
__device__ __forceinline__ CX<float> cmsub(const CX<float> &a, const CX<float> &b, const CX<float> &c,
                                           const CX<float> &d)
{
    CX<float> r;
    r.re = a.re * b.re;
    r.re = FMA(-a.im, b.im, r.re);
    r.re = FMA(-c.re, d.re, r.re);
    r.re = FMA(c.im, d.im, r.re);
    r.im = a.re * b.im;
    r.im = FMA(a.im, b.re, r.im);
    r.im = FMA(-c.re, d.im, r.im);
    r.im = FMA(-c.im, d.re, r.im);
    return r;
}

// the staple of U_mu(x) (staple3's terms and summation order) and the 8
// network features
template <int mu>
__device__ __forceinline__ void staple_features(const Field<float> &U, const Geom &G, uint32_t t, const Nbr &n,
                                                int p, M3<float> &st, float (&x)[kNF])
{
    const uint32_t own = (uint32_t)p * G.cb + t, opp = (uint32_t)(p ^ 1) * G.cb + t;
    M3<float> s2;
    float rr[3], qq[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const int nu = nu_of(mu, i);
        M3<float> fw = staple_fwd3(U.ldg3(nu, opp + n.dp[mu]), U.ldg3(mu, opp + n.dp[nu]), U.ldg3(nu, own));
        M3<float> bw = staple_bwd3(U.ldg3(nu, own + n.dm[nu] + n.dp[mu]), U.ldg3(mu, opp + n.dm[nu]),
                                   U.ldg3(nu, opp + n.dm[nu]));
        const CX<float> tr = tr_fbh(fw, bw);
        rr[i] = tr.re / 3.0f;
        qq[i] = tr.im / 3.0f;
        if (i == 0) {
            add3(st, fw, bw);
        } else {
            add3(s2, st, fw);
            add3(st, bw, s2);
        }
    }
    const M3<float> &A = st;
    float tn = A.m[0][0].re * A.m[0][0].re;
    tn = FMA(A.m[0][0].im, A.m[0][0].im, tn);
#pragma unroll
    for (int q = 1; q < 9; q++) {
        tn = FMA(A.m[q / 3][q % 3].re, A.m[q / 3][q % 3].re, tn);
        tn = FMA(A.m[q / 3][q % 3].im, A.m[q / 3][q % 3].im, tn);
    }
    float t2 = 0.0f;
#pragma unroll
    for (int q = 0; q < 9; q++) {
        const CX<float> m = dotc3(&A.m[q / 3][0], 1, &A.m[q % 3][0], 1);
        t2 = (q == 0) ? m.re * m.re : FMA(m.re, m.re, t2);
        t2 = FMA(m.im, m.im, t2);
    }
    const CX<float> c0 = cmsub(A.m[1][1], A.m[2][2], A.m[1][2], A.m[2][1]);
    const CX<float> c1 = cmsub(A.m[1][0], A.m[2][2], A.m[1][2], A.m[2][0]);
    const CX<float> c2 = cmsub(A.m[1][0], A.m[2][1], A.m[1][1], A.m[2][0]);
    float dre = A.m[0][0].re * c0.re;
    dre = FMA(-A.m[0][0].im, c0.im, dre);
    dre = FMA(-A.m[0][1].re, c1.re, dre);
    dre = FMA(A.m[0][1].im, c1.im, dre);
    dre = FMA(A.m[0][2].re, c2.re, dre);
    dre = FMA(-A.m[0][2].im, c2.im, dre);
    float dim = A.m[0][0].re * c0.im;
    dim = FMA(A.m[0][0].im, c0.re, dim);
    dim = FMA(-A.m[0][1].re, c1.im, dim);
    dim = FMA(-A.m[0][1].im, c1.re, dim);
    dim = FMA(A.m[0][2].re, c2.im, dim);
    dim = FMA(A.m[0][2].im, c2.re, dim);
    const float s = tn / 3.0f, n3 = s * sqrtf(s);
    x[0] = tn / 108.0f;
    x[1] = (tn > 0.0f) ? t2 / (tn * tn) : 1.0f;
    x[2] = (n3 > 0.0f) ? dre / n3 : 0.0f;
    x[3] = (n3 > 0.0f) ? dim / n3 : 0.0f;
    x[4] = ((rr[0] + rr[1]) + rr[2]) / 3.0f;
    x[5] = FMA(rr[2], rr[2], FMA(rr[1], rr[1], rr[0] * rr[0])) / 3.0f;
    x[6] = ((qq[0] + qq[1]) + qq[2]) / 3.0f;
    x[7] = FMA(qq[2], qq[2], FMA(qq[1], qq[1], qq[0] * qq[0])) / 3.0f;
}

// the network's output o (weights w in shared memory, FP32)
__device__ __forceinline__ float mlp_out(const float *w, const float (&x)[kNF])
{
    float h1[kNH];
#pragma unroll
    for (int j = 0; j < kNH; j++) {
        float z = w[kB1 + j];
#pragma unroll
        for (int k = 0; k < kNF; k++) z = FMA(w[kW1 + j * kNF + k], x[k], z);
        h1[j] = z > 0.0f ? z : 0.0f;
    }
    float o = w[kB3];
    for (int j = 0; j < kNH; j++) {
        float z = w[kB2 + j];
#pragma unroll
        for (int k = 0; k < kNH; k++) z = FMA(w[kW2 + j * kNH + k], h1[k], z);
        o = FMA(w[kW3 + j], z > 0.0f ? z : 0.0f, o);
    }
    return o;
}

__device__ __forceinline__ double sigmoid_d(float o) { return 1.0 / (1.0 + qg_exp(-(double)o)); }

// three standard normals from one quad (Box-Muller on (x,y) and (z,w))
__device__ __forceinline__ void normals3(const R4<float> &q, double &a0, double &a1, double &a2)
{
    const double l1 = sqrt(-2.0 * qg_log((double)q.x)), l3 = sqrt(-2.0 * qg_log((double)q.z));
    double s1, c1, s3, c3;
    qg_sincos(6.283185307179586 * (double)q.y, &s1, &c1);
    qg_sincos(6.283185307179586 * (double)q.w, &s3, &c3);
    a0 = l1 * c1;
    a1 = l1 * s1;
    a2 = l3 * c3;
}

// coefficients of Re Tr((X - 1) w) for the 2x2 block w = (u1 u2; v1 v2) of
// W = U A: (x0 - 1) c0 + x1 c1 + x2 c2 + x3 c3 for X = (x0 + i x3, x2 + i x1;
// -x2 + i x1, x0 - i x3)
__device__ __forceinline__ void block_coeffs(const S2<float> &w, double &c0, double &c1, double &c2, double &c3)
{
    c0 = (double)w.u1.re + (double)w.v2.re;
    c1 = -((double)w.v1.im + (double)w.u2.im);
    c2 = (double)w.v1.re - (double)w.u2.re;
    c3 = -((double)w.u1.im - (double)w.v2.im);
}

// the 2x2 block (rows i, j; columns i, j) of W = U A from rows picked by
// selects (no runtime indexing of register arrays)
__device__ __forceinline__ S2<float> w_block(const CX<float> (&ri)[3], const CX<float> (&rj)[3], const M3<float> &A,
                                             int i, int j)
{
    CX<float> ci[3], cj[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        ci[k] = pick3(A.m[k][0], A.m[k][1], A.m[k][2], i);
        cj[k] = pick3(A.m[k][0], A.m[k][1], A.m[k][2], j);
    }
    S2<float> w;
    w.u1 = dot3(ri, 1, ci, 1);
    w.u2 = dot3(ri, 1, cj, 1);
    w.v1 = dot3(rj, 1, ci, 1);
    w.v2 = dot3(rj, 1, cj, 1);
    return w;
}

template <int mu>
__global__ void __launch_bounds__(128) k_mh_phase(Field<float> U, Geom G, PhaseArgs A, const uint16_t *wq,
                                                  double eps_max, int nhit, unsigned long long *acc_count,
                                                  double *jump_sum)
{
    __shared__ float w[kNP];
    for (int i = threadIdx.x; i < kNP; i += blockDim.x) w[i] = bf16_bits_to_float(wq[i]);
    __syncthreads();
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned acc = 0;
    double jump = 0.0;
    if (t < G.half) {
        const int p = A.parity;
        Crd c = lex2crd(G, 2 * t);
        if (parity_of(c) != p) c.y += 1;
        const uint32_t e0 = (uint32_t)p * G.cb + t;
        const Nbr nb = neighbours(G, c);
        const double bn = (double)(float)A.params[0];          // (float)(BETA/N), as the heatbath
        M3<float> st;
        float x[kNF];
        staple_features<mu>(U, G, t, nb, p, st, x);
        const float eps = (float)(eps_max * sigmoid_d(mlp_out(w, x)));
        M3<float> Um = expand(U.ld3(mu, e0));
        const uint64_t phase = *A.phase_base + A.phase_offset;
        PrnPhilox<float> prn;
        prn.key = A.key; prn.t = t; prn.k = 0; prn.plo = (uint32_t)phase; prn.phi = (uint32_t)(phase >> 32);
        for (int h = 0; h < nhit; h++) {
#pragma unroll 1
            for (int sg = 0; sg < 3; sg++) {
                const int i = (sg == 2) ? 1 : 0, j = (sg == 0) ? 1 : 2;
                const R4<float> q1 = prn.next(), q2 = prn.next();
                double a0, a1, a2;
                normals3(q1, a0, a1, a2);
                const double r = sqrt(FMA(a2, a2, FMA(a1, a1, a0 * a0)));
                const double th = (double)eps * r;
                double sn, cs;
                qg_sincos(th, &sn, &cs);
                const double sr = (r > 0.0) ? sn / r : 0.0;
                const float x0 = (float)cs, x1 = (float)(sr * a0), x2 = (float)(sr * a1), x3 = (float)(sr * a2);
                CX<float> ri[3], rj[3];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    ri[k] = pick3(Um.m[0][k], Um.m[1][k], Um.m[2][k], i);
                    rj[k] = pick3(Um.m[0][k], Um.m[1][k], Um.m[2][k], j);
                }
                double c0, c1, c2, c3;
                block_coeffs(w_block(ri, rj, st, i, j), c0, c1, c2, c3);
                const double dS =
                    -bn * FMA((double)x0 - 1.0, c0, FMA((double)x1, c1, FMA((double)x2, c2, (double)x3 * c3)));
                if (qg_log((double)q2.x) <= -dS) {
                    S2<float> V;
                    V.u1 = { x0, x3 }; V.u2 = { x2, x1 }; V.v1 = { -x2, x1 }; V.v2 = { x0, -x3 };
                    M3<float> R;
#pragma unroll
                    for (int k = 0; k < 3; k++) { R.m[0][k] = ri[k]; R.m[1][k] = rj[k]; }
                    rotate_rows(R, 0, 1, V);
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        if (i == 0) Um.m[0][k] = R.m[0][k]; else Um.m[1][k] = R.m[0][k];
                        if (j == 1) Um.m[1][k] = R.m[1][k]; else Um.m[2][k] = R.m[1][k];
                    }
                    acc++;
                    jump += th * th;
                }
            }
        }
        U.st3(mu, e0, gs3<float>(compress(Um)));
    }
    for (int o = 16; o > 0; o >>= 1) {
        acc += __shfl_down_sync(0xffffffffu, acc, o);
        jump += __shfl_down_sync(0xffffffffu, jump, o);
    }
    if ((threadIdx.x & 31) == 0 && acc_count) {
        atomicAdd(acc_count, (unsigned long long)acc);
        atomicAdd(jump_sum, jump);
    }
}

// Gradient of the loss L = -(1/links) sum_links sum_subgroups
// min(1, exp(-dS)) (eps |a|)^2 over the links of one phase, for proposals
// drawn from the current links (the field is not changed).  Block b writes
// its sums of the per-link weight gradients (in thread order) and of
// (loss, ESJD, acceptance, links) to partials[b][kNP + 4].
template <int mu>
__global__ void __launch_bounds__(kTrainBlock) k_mh_grad(Field<float> U, Geom G, int parity, const double *params,
                                                         const uint16_t *wq, double eps_max, uint2 key,
                                                         uint64_t phase, float *partials)
{
    __shared__ float w[kNP];
    __shared__ float sx[kTrainBlock][kNF], sh1[kTrainBlock][kNH], sh2[kTrainBlock][kNH], sd1[kTrainBlock][kNH],
        sd2[kTrainBlock][kNH], sgo[kTrainBlock], sst[kTrainBlock][4];
    for (int i = threadIdx.x; i < kNP; i += blockDim.x) w[i] = bf16_bits_to_float(wq[i]);
    __syncthreads();
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const int me = threadIdx.x;
    float x[kNF], z1[kNH], z2[kNH];
#pragma unroll
    for (int k = 0; k < kNF; k++) x[k] = 0.0f;
#pragma unroll
    for (int k = 0; k < kNH; k++) { z1[k] = 0.0f; z2[k] = 0.0f; }
    float go = 0.0f, loss = 0.0f, esjd = 0.0f, accm = 0.0f, one = 0.0f;
    if (t < G.half) {
        Crd c = lex2crd(G, 2 * t);
        if (parity_of(c) != parity) c.y += 1;
        const uint32_t e0 = (uint32_t)parity * G.cb + t;
        const Nbr nb = neighbours(G, c);
        const double bn = (double)(float)params[0];
        M3<float> st;
        staple_features<mu>(U, G, t, nb, parity, st, x);
        // forward, keeping the pre-activations
#pragma unroll
        for (int j = 0; j < kNH; j++) {
            float z = w[kB1 + j];
#pragma unroll
            for (int k = 0; k < kNF; k++) z = FMA(w[kW1 + j * kNF + k], x[k], z);
            z1[j] = z;
        }
        float o = w[kB3];
#pragma unroll
        for (int j = 0; j < kNH; j++) {
            float z = w[kB2 + j];
#pragma unroll
            for (int k = 0; k < kNH; k++) z = FMA(w[kW2 + j * kNH + k], z1[k] > 0.0f ? z1[k] : 0.0f, z);
            z2[j] = z;
            o = FMA(w[kW3 + j], z > 0.0f ? z : 0.0f, o);
        }
        const double sg = sigmoid_d(o);
        const double eps = eps_max * sg;
        const M3<float> Um = expand(U.ld3(mu, e0));
        PrnPhilox<float> prn;
        prn.key = key; prn.t = t; prn.k = 0; prn.plo = (uint32_t)phase; prn.phi = (uint32_t)(phase >> 32);
        double geps = 0.0, ls = 0.0, es = 0.0, ac = 0.0;
#pragma unroll 1
        for (int s = 0; s < 3; s++) {
            const int i = (s == 2) ? 1 : 0, j = (s == 0) ? 1 : 2;
            double a0, a1, a2;
            normals3(prn.next(), a0, a1, a2);
            const double r = sqrt(FMA(a2, a2, FMA(a1, a1, a0 * a0)));
            const double th = eps * r;
            double sn, cs;
            qg_sincos(th, &sn, &cs);
            CX<float> ri[3], rj[3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                ri[k] = pick3(Um.m[0][k], Um.m[1][k], Um.m[2][k], i);
                rj[k] = pick3(Um.m[0][k], Um.m[1][k], Um.m[2][k], j);
            }
            double c0, c1, c2, c3;
            block_coeffs(w_block(ri, rj, st, i, j), c0, c1, c2, c3);
            const double ac_ = (r > 0.0) ? (a0 * c1 + a1 * c2 + a2 * c3) / r : 0.0;   // a-hat . c
            const double dS = -bn * ((cs - 1.0) * c0 + sn * ac_);
            const double dSde = -bn * r * (-sn * c0 + cs * ac_);
            const double a = (dS <= 0.0) ? 1.0 : qg_exp(-dS);
            const double dade = (dS <= 0.0) ? 0.0 : -a * dSde;
            es += a * th * th;
            ac += a;
            geps -= dade * th * th + a * 2.0 * eps * r * r;
        }
        ls = -es;
        go = (float)(geps * eps_max * sg * (1.0 - sg));
        loss = (float)ls;
        esjd = (float)es;
        accm = (float)(ac / 3.0);
        one = 1.0f;
    }
    // backward of one link into shared memory
#pragma unroll
    for (int k = 0; k < kNF; k++) sx[me][k] = x[k];
    float dz2[kNH];
#pragma unroll
    for (int j = 0; j < kNH; j++) {
        sh2[me][j] = z2[j] > 0.0f ? z2[j] : 0.0f;
        dz2[j] = z2[j] > 0.0f ? go * w[kW3 + j] : 0.0f;
        sd2[me][j] = dz2[j];
        sh1[me][j] = z1[j] > 0.0f ? z1[j] : 0.0f;
    }
#pragma unroll 1
    for (int k = 0; k < kNH; k++) {           // dz1[k] = relu'(z1[k]) sum_j W2[j][k] dz2[j]
        float d = 0.0f;
#pragma unroll
        for (int j = 0; j < kNH; j++) d = FMA(w[kW2 + j * kNH + k], dz2[j], d);
        sd1[me][k] = sh1[me][k] > 0.0f ? d : 0.0f;
    }
    sgo[me] = go;
    sst[me][0] = loss; sst[me][1] = esjd; sst[me][2] = accm; sst[me][3] = one;
    __syncthreads();
    // block sums in thread order
    float *out = partials + (size_t)blockIdx.x * (kNP + 4);
    for (int q = threadIdx.x; q < kNP + 4; q += blockDim.x) {
        float acc = 0.0f;
        if (q < kB1) {                                   // W1[j][k] = sum dz1[j] x[k]
            const int j = (q - kW1) / kNF, k = (q - kW1) % kNF;
            for (int u = 0; u < kTrainBlock; u++) acc = FMA(sd1[u][j], sx[u][k], acc);
        } else if (q < kW2) {                            // b1[j]
            for (int u = 0; u < kTrainBlock; u++) acc += sd1[u][q - kB1];
        } else if (q < kB2) {                            // W2[j][k] = sum dz2[j] h1[k]
            const int j = (q - kW2) / kNH, k = (q - kW2) % kNH;
            for (int u = 0; u < kTrainBlock; u++) acc = FMA(sd2[u][j], sh1[u][k], acc);
        } else if (q < kW3) {                            // b2[j]
            for (int u = 0; u < kTrainBlock; u++) acc += sd2[u][q - kB2];
        } else if (q < kB3) {                            // w3[k] = sum go h2[k]
            for (int u = 0; u < kTrainBlock; u++) acc = FMA(sgo[u], sh2[u][q - kW3], acc);
        } else if (q == kB3) {
            for (int u = 0; u < kTrainBlock; u++) acc += sgo[u];
        } else {
            for (int u = 0; u < kTrainBlock; u++) acc += sst[u][q - kNP];
        }
        out[q] = acc;
    }
}

// grad[q] = (sum over blocks in order) / links, stats = raw sums
__global__ void k_mh_grad_reduce(const float *partials, uint32_t nblocks, float *grad)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kNP + 4) return;
    double s = 0.0, n = 0.0;
    for (uint32_t b = 0; b < nblocks; b++) {
        s += (double)partials[(size_t)b * (kNP + 4) + q];
        n += (double)partials[(size_t)b * (kNP + 4) + kNP + 3];
    }
    grad[q] = (q < kNP) ? (float)(n > 0.0 ? s / n : 0.0) : (float)s;
}

// Adam on the FP32 master weights; writes the BF16 copy the kernels read
__global__ void k_adam(float *master, float *m, float *v, const float *grad, uint16_t *wq, float lr, float b1,
                       float b2, float c1, float c2, float epsa)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kNP) return;
    const float g = grad[q];
    const float mq = b1 * m[q] + (1.0f - b1) * g, vq = b2 * v[q] + (1.0f - b2) * g * g;
    m[q] = mq;
    v[q] = vq;
    const float p = master[q] - lr * (mq / c1) / (sqrtf(vq / c2) + epsa);
    master[q] = p;
    wq[q] = float_to_bf16_bits(p);
}

__global__ void k_to_bf16(const float *master, uint16_t *wq)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < kNP) wq[q] = float_to_bf16_bits(master[q]);
}

// ------------------------------------------------------------- launchers
cudaError_t launch_mh_phase(const Geom &G, void *links, const PhaseArgs &a, const uint16_t *wq, double eps_max,
                            int nhit, unsigned long long *acc_count, double *jump_sum, cudaStream_t s)
{
    Field<float> U{ (float4 *)links, G.pstride };
    const unsigned nb = (G.half + 127) / 128;
    switch (a.dir) {
    case 0: k_mh_phase<0><<<nb, 128, 0, s>>>(U, G, a, wq, eps_max, nhit, acc_count, jump_sum); break;
    case 1: k_mh_phase<1><<<nb, 128, 0, s>>>(U, G, a, wq, eps_max, nhit, acc_count, jump_sum); break;
    case 2: k_mh_phase<2><<<nb, 128, 0, s>>>(U, G, a, wq, eps_max, nhit, acc_count, jump_sum); break;
    default: k_mh_phase<3><<<nb, 128, 0, s>>>(U, G, a, wq, eps_max, nhit, acc_count, jump_sum); break;
    }
    return cudaGetLastError();
}

uint32_t mh_grad_blocks(const Geom &G) { return (G.half + kTrainBlock - 1) / kTrainBlock; }

cudaError_t launch_mh_grad(const Geom &G, const void *links, int parity, int dir, const double *params,
                           const uint16_t *wq, double eps_max, uint2 key, uint64_t phase, float *partials,
                           float *grad, cudaStream_t s)
{
    Field<float> U{ (float4 *)links, G.pstride };
    const unsigned nb = mh_grad_blocks(G);
    switch (dir) {
    case 0: k_mh_grad<0><<<nb, kTrainBlock, 0, s>>>(U, G, parity, params, wq, eps_max, key, phase, partials); break;
    case 1: k_mh_grad<1><<<nb, kTrainBlock, 0, s>>>(U, G, parity, params, wq, eps_max, key, phase, partials); break;
    case 2: k_mh_grad<2><<<nb, kTrainBlock, 0, s>>>(U, G, parity, params, wq, eps_max, key, phase, partials); break;
    default: k_mh_grad<3><<<nb, kTrainBlock, 0, s>>>(U, G, parity, params, wq, eps_max, key, phase, partials); break;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_mh_grad_reduce<<<(kNP + 4 + 255) / 256, 256, 0, s>>>(partials, nb, grad);
    return cudaGetLastError();
}

cudaError_t launch_adam(float *master, float *m, float *v, const float *grad, uint16_t *wq, float lr, float b1,
                        float b2, float c1, float c2, float epsa, cudaStream_t s)
{
    k_adam<<<(kNP + 255) / 256, 256, 0, s>>>(master, m, v, grad, wq, lr, b1, b2, c1, c2, epsa);
    return cudaGetLastError();
}

cudaError_t launch_to_bf16(const float *master, uint16_t *wq, cudaStream_t s)
{
    k_to_bf16<<<(kNP + 255) / 256, 256, 0, s>>>(master, wq);
    return cudaGetLastError();
}

}  // namespace qg
