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
// the block sums of the weight gradients and the Adam step are kernels
// here.  Weights are stored in BF16 for the kernels and in FP32 for the
// optimiser; the per-link acceptance arithmetic is FP64.
//
// Tensor cores.  The network runs on the fifth-generation tensor cores
// (tcgen05, qg_tc.cuh): a CTA of 128 threads holds 128 links, the MMA's M
// rows.  Forward: the features (BF16, K = 16 with 8 zero columns) times W1
// (N = 32) accumulate in FP32 in tensor memory; each thread reads its link's
// row back (tcgen05.ld), adds the bias, applies the ReLU and stores the
// hidden layer as BF16 for the second MMA (K = 32, N = 32); the output layer
// (32 -> 1) is an FP32 dot product in the thread.  Training adds two MMAs:
// the back-propagated dz1 = W2^T dz2 per link (M = 128 links, N = 32, K = 32)
// and all weight and bias gradients of the block in one product over the
// link dimension (M = 128 rows [dz2^T; dz1^T; dL/do], N = 80 columns
// [h1^T; h2^T; x^T; 1], K = 128 links).  Activations and back-propagated
// values enter the MMAs rounded to BF16; products and sums are FP32.
#include "qg_internal.h"
#include "qg_tc.cuh"
#include "qg_update.cuh"

namespace qg {

constexpr int kNF = QG_NET_FEATURES, kNH = QG_NET_HIDDEN;
constexpr int kW1 = 0, kB1 = kW1 + kNH * kNF, kW2 = kB1 + kNH, kB2 = kW2 + kNH * kNH, kW3 = kB2 + kNH,
              kB3 = kW3 + kNH, kNP = kB3 + 1;
static_assert(kNP == QG_NET_PARAMS, "parameter count");

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

constexpr int kMHBlock = 128;                  // links per CTA = the MMA's M
constexpr uint32_t kWaitPolls = 1u << 22;       // mbarrier polls before a wait gives up
constexpr uint32_t kIdesc32 = tc::idesc_bf16_f32(128, 32), kIdesc80 = tc::idesc_bf16_f32(128, 80);
constexpr int kGN = 80;                         // columns of the weight-gradient MMA
constexpr uint16_t kBF16One = 0x3F80u;

// the network's operands in shared memory (tcgen05 K-major layout)
struct NetOps {
    alignas(128) uint8_t a1[kMHBlock * 16 * 2];   // features, BF16, K = 16 (columns 8..15 zero)
    alignas(128) uint8_t a2[kMHBlock * 32 * 2];   // hidden layer 1 (training: then dz2), BF16, K = 32
    alignas(128) uint8_t b1[kNH * 16 * 2];        // W1[j][k], K = 16
    alignas(128) uint8_t b2[kNH * kNH * 2];       // W2[j][k], K = 32
    float bias1[kNH], bias2[kNH], w3[kNH], b3;
    uint64_t mbar;
    uint32_t tmem;
};
// the training kernel's extra operands
struct GradOps {
    alignas(128) uint8_t b2t[kNH * kNH * 2];      // W2^T: [k][j], K = 32
    alignas(128) uint8_t ga[128 * kMHBlock * 2];  // rows: dz2^T (0..31), dz1^T (32..63), dL/do (64), 0; K = links
    alignas(128) uint8_t gb[kGN * kMHBlock * 2];  // rows: h1^T (0..31), h2^T (32..63), x^T (64..71), 1 (72), 0
    float sst[kMHBlock][4];
};

__device__ __forceinline__ void st_bf16(uint8_t *base, uint32_t off, uint16_t v)
{
    *reinterpret_cast<uint16_t *>(base + off) = v;
}
// 8 floats as BF16 into one 16-byte chunk (row m, columns c .. c+7)
__device__ __forceinline__ void st_bf16x8(uint8_t *base, uint32_t off, const float *v)
{
    uint4 q;
    q.x = (uint32_t)float_to_bf16_bits(v[0]) | ((uint32_t)float_to_bf16_bits(v[1]) << 16);
    q.y = (uint32_t)float_to_bf16_bits(v[2]) | ((uint32_t)float_to_bf16_bits(v[3]) << 16);
    q.z = (uint32_t)float_to_bf16_bits(v[4]) | ((uint32_t)float_to_bf16_bits(v[5]) << 16);
    q.w = (uint32_t)float_to_bf16_bits(v[6]) | ((uint32_t)float_to_bf16_bits(v[7]) << 16);
    *reinterpret_cast<uint4 *>(base + off) = q;
}

// weights into the operand layout, the mbarrier, ncols TMEM columns
__device__ __forceinline__ void net_setup(NetOps &S, const uint16_t *wq, uint32_t ncols)
{
    for (int i = threadIdx.x; i < kNH * 16; i += blockDim.x) {
        const int j = i >> 4, k = i & 15;
        st_bf16(S.b1, tc::kmajor_off(j, k, 16), k < kNF ? wq[kW1 + j * kNF + k] : (uint16_t)0);
    }
    for (int i = threadIdx.x; i < kNH * kNH; i += blockDim.x) {
        const int j = i >> 5, k = i & 31;
        st_bf16(S.b2, tc::kmajor_off(j, k, 32), wq[kW2 + j * kNH + k]);
    }
    for (int i = threadIdx.x; i < kNH; i += blockDim.x) {
        S.bias1[i] = bf16_bits_to_float(wq[kB1 + i]);
        S.bias2[i] = bf16_bits_to_float(wq[kB2 + i]);
        S.w3[i] = bf16_bits_to_float(wq[kW3 + i]);
    }
    if (threadIdx.x == 0) {
        S.b3 = bf16_bits_to_float(wq[kB3]);
        tc::mbar_init(&S.mbar, 1);
    }
    if (threadIdx.x < 32) tc::tmem_alloc(&S.tmem, ncols);
}
// all threads: make the generic shared-memory writes visible to the tensor
// core, order them (and earlier TMEM reads) before the next MMA
__device__ __forceinline__ void net_sync()
{
    tc::fence_async_shared();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
}
// all threads: wait for the committed MMAs; false (block-uniform) if the
// wait ran out
__device__ __forceinline__ bool net_wait(NetOps &S, uint32_t &phase)
{
    const bool ok = tc::mbar_wait(&S.mbar, phase, kWaitPolls);
    phase ^= 1u;
    const int bad = __syncthreads_or(!ok);
    tc::fence_after_sync();
    return !bad;
}
__device__ __forceinline__ void net_teardown(NetOps &S, uint32_t ncols, bool ok, uint32_t phase)
{
    if (!ok) tc::mbar_wait(&S.mbar, phase, kWaitPolls);      // let a late MMA land before the free
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc::fence_after_sync();
        tc::tmem_free(S.tmem, ncols);
    }
}

// the network for the CTA's 128 links: thread m's features x -> the
// pre-activations z1, z2 and the output o of its link
__device__ __forceinline__ bool net_forward(NetOps &S, uint32_t &phase, const float (&x)[kNF], float (&z1)[kNH],
                                            float (&z2)[kNH], float &o)
{
    const int m = threadIdx.x;
    const float zero8[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
    st_bf16x8(S.a1, tc::kmajor_off(m, 0, 16), x);
    st_bf16x8(S.a1, tc::kmajor_off(m, 8, 16), zero8);
    net_sync();                                  // also publishes the TMEM address and the mbarrier
    const uint32_t lane_base = S.tmem + ((uint32_t)(m & ~31) << 16);
    if (m == 0) {
        tc::mma_bf16(S.tmem, tc::desc_operand(S.a1, 16, 0), tc::desc_operand(S.b1, 16, 0), kIdesc32, 0);
        tc::mma_commit(&S.mbar);
    }
    if (!net_wait(S, phase)) return false;
    float acc[32];
    tc::tmem_ld32(lane_base, acc);
    float h[kNH];
#pragma unroll
    for (int j = 0; j < kNH; j++) {
        z1[j] = acc[j] + S.bias1[j];
        h[j] = z1[j] > 0.0f ? z1[j] : 0.0f;
    }
#pragma unroll
    for (int c = 0; c < 4; c++) st_bf16x8(S.a2, tc::kmajor_off(m, 8 * c, 32), h + 8 * c);
    net_sync();
    if (m == 0) {
        tc::mma_bf16(S.tmem, tc::desc_operand(S.a2, 32, 0), tc::desc_operand(S.b2, 32, 0), kIdesc32, 0);
        tc::mma_bf16(S.tmem, tc::desc_operand(S.a2, 32, 16), tc::desc_operand(S.b2, 32, 16), kIdesc32, 1);
        tc::mma_commit(&S.mbar);
    }
    if (!net_wait(S, phase)) return false;
    tc::tmem_ld32(lane_base, acc);
    float out = S.b3;
#pragma unroll
    for (int j = 0; j < kNH; j++) {
        z2[j] = acc[j] + S.bias2[j];
        out = FMA(S.w3[j], z2[j] > 0.0f ? z2[j] : 0.0f, out);
    }
    o = out;
    return true;
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

// One Metropolis phase; EPS_ONLY: only the step eps of every link of the
// phase into eps_out[t] (the same arithmetic up to eps, the field untouched)
template <int mu, bool EPS_ONLY>
__global__ void __launch_bounds__(kMHBlock) k_mh_phase(Field<float> U, Geom G, PhaseArgs A, const uint16_t *wq,
                                                       double eps_max, int nhit, unsigned long long *acc_count,
                                                       double *jump_sum, float *eps_out, unsigned *err)
{
    __shared__ NetOps S;
    net_setup(S, wq, 32);
    const uint32_t t = blockIdx.x * kMHBlock + threadIdx.x;
    const bool active = t < G.half;
    const int p = A.parity;
    Crd c = lex2crd(G, 2 * (active ? t : 0));
    if (parity_of(c) != p) c.y += 1;
    const uint32_t e0 = (uint32_t)p * G.cb + t;
    const Nbr nb = neighbours(G, c);
    M3<float> st;
    float x[kNF];
#pragma unroll
    for (int k = 0; k < kNF; k++) x[k] = 0.0f;
    if (active) staple_features<mu>(U, G, t, nb, p, st, x);
    uint32_t phase = 0;
    float z1[kNH], z2[kNH], o = 0.0f;
    const bool ok = net_forward(S, phase, x, z1, z2, o);
    net_teardown(S, 32, ok, phase);
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(err, 1u);
        return;
    }
    const float eps = (float)(eps_max * sigmoid_d(o));
    if (EPS_ONLY) {
        if (active) eps_out[t] = eps;
        return;
    }
    unsigned acc = 0;
    double jump = 0.0;
    if (active) {
        const double bn = (double)(float)A.params[0];          // (float)(BETA/N), as the heatbath
        M3<float> Um = expand(U.ld3(mu, e0));
        const uint64_t ph = *A.phase_base + A.phase_offset;
        PrnPhilox<float> prn;
        prn.key = A.key; prn.t = t; prn.k = 0; prn.plo = (uint32_t)ph; prn.phi = (uint32_t)(ph >> 32);
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
    for (int ofs = 16; ofs > 0; ofs >>= 1) {
        acc += __shfl_down_sync(0xffffffffu, acc, ofs);
        jump += __shfl_down_sync(0xffffffffu, jump, ofs);
    }
    if ((threadIdx.x & 31) == 0 && acc_count) {
        atomicAdd(acc_count, (unsigned long long)acc);
        atomicAdd(jump_sum, jump);
    }
}

// Gradient of the loss L = -(1/links) sum_links sum_subgroups
// min(1, exp(-dS)) (eps |a|)^2 over the links of one phase, for proposals
// drawn from the current links (the field is not changed).  Block b writes
// its sums of the per-link weight gradients and of (loss, ESJD,
// acceptance, links) to partials[b][kNP + 4]; the weight and bias sums come
// from one tensor-core product over the block's links (see the file head).
constexpr size_t kGradSmem = sizeof(NetOps) + sizeof(GradOps) + 128;

template <int mu>
__global__ void __launch_bounds__(kMHBlock) k_mh_grad(Field<float> U, Geom G, int parity, const double *params,
                                                      const uint16_t *wq, double eps_max, uint2 key, uint64_t phase,
                                                      float *partials, unsigned *err)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    NetOps &S = *reinterpret_cast<NetOps *>(base);
    GradOps &T = *reinterpret_cast<GradOps *>(base + sizeof(NetOps));
    net_setup(S, wq, 128);
    const int me = threadIdx.x;
    for (int i = me; i < kNH * kNH; i += kMHBlock) {           // W2^T[k][j] = W2[j][k]
        const int k = i >> 5, j = i & 31;
        st_bf16(T.b2t, tc::kmajor_off(k, j, 32), wq[kW2 + j * kNH + k]);
    }
    // rows 64..127 of ga (row groups 8..15) and 72..79 of gb (row group 9) start at zero
    for (int i = me; i < 8 * kMHBlock * 16 / 16; i += kMHBlock)
        reinterpret_cast<uint4 *>(T.ga + tc::kmajor_off(64, 0, kMHBlock))[i] = make_uint4(0, 0, 0, 0);
    for (int i = me; i < kMHBlock * 16 / 16; i += kMHBlock)
        reinterpret_cast<uint4 *>(T.gb + tc::kmajor_off(72, 0, kMHBlock))[i] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    st_bf16(T.gb, tc::kmajor_off(72, me, kMHBlock), kBF16One);

    const uint32_t t = blockIdx.x * kMHBlock + me;
    const bool active = t < G.half;
    float x[kNF];
#pragma unroll
    for (int k = 0; k < kNF; k++) x[k] = 0.0f;
    M3<float> st;
    Crd c = lex2crd(G, 2 * (active ? t : 0));
    if (parity_of(c) != parity) c.y += 1;
    const uint32_t e0 = (uint32_t)parity * G.cb + t;
    if (active) {
        const Nbr nb = neighbours(G, c);
        staple_features<mu>(U, G, t, nb, parity, st, x);
    }
    uint32_t mph = 0;
    float z1[kNH], z2[kNH], o = 0.0f;
    bool ok = net_forward(S, mph, x, z1, z2, o);
    float go = 0.0f, loss = 0.0f, esjd = 0.0f, accm = 0.0f, one = 0.0f;
    if (ok && active) {
        const double bn = (double)(float)params[0];
        const double sg = sigmoid_d(o);
        const double eps = eps_max * sg;
        const M3<float> Um = expand(U.ld3(mu, e0));
        PrnPhilox<float> prn;
        prn.key = key; prn.t = t; prn.k = 0; prn.plo = (uint32_t)phase; prn.phi = (uint32_t)(phase >> 32);
        double geps = 0.0, es = 0.0, ac = 0.0;
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
        go = (float)(geps * eps_max * sg * (1.0 - sg));
        loss = (float)(-es);
        esjd = (float)es;
        accm = (float)(ac / 3.0);
        one = 1.0f;
    }
    if (ok) {
        // back-propagation through the output layer; dz2 as the A operand
        // of dz1 = W2^T dz2 (rows = links, K = 32)
        float dz2[kNH], h[kNH];
#pragma unroll
        for (int j = 0; j < kNH; j++) dz2[j] = z2[j] > 0.0f ? go * S.w3[j] : 0.0f;
#pragma unroll
        for (int q = 0; q < 4; q++) st_bf16x8(S.a2, tc::kmajor_off(me, 8 * q, 32), dz2 + 8 * q);
        // the weight-gradient operands of this link (column me)
#pragma unroll
        for (int j = 0; j < kNH; j++) {
            st_bf16(T.ga, tc::kmajor_off(j, me, kMHBlock), float_to_bf16_bits(dz2[j]));
            h[j] = z1[j] > 0.0f ? z1[j] : 0.0f;
            st_bf16(T.gb, tc::kmajor_off(j, me, kMHBlock), float_to_bf16_bits(h[j]));
            st_bf16(T.gb, tc::kmajor_off(32 + j, me, kMHBlock), float_to_bf16_bits(z2[j] > 0.0f ? z2[j] : 0.0f));
        }
#pragma unroll
        for (int k = 0; k < kNF; k++) st_bf16(T.gb, tc::kmajor_off(64 + k, me, kMHBlock), float_to_bf16_bits(x[k]));
        st_bf16(T.ga, tc::kmajor_off(64, me, kMHBlock), float_to_bf16_bits(go));
        net_sync();
        if (me == 0) {
            tc::mma_bf16(S.tmem, tc::desc_operand(S.a2, 32, 0), tc::desc_operand(T.b2t, 32, 0), kIdesc32, 0);
            tc::mma_bf16(S.tmem, tc::desc_operand(S.a2, 32, 16), tc::desc_operand(T.b2t, 32, 16), kIdesc32, 1);
            tc::mma_commit(&S.mbar);
        }
        ok = net_wait(S, mph);
        if (ok) {
            float d[32];
            tc::tmem_ld32(S.tmem + ((uint32_t)(me & ~31) << 16), d);
#pragma unroll
            for (int k = 0; k < kNH; k++)
                st_bf16(T.ga, tc::kmajor_off(32 + k, me, kMHBlock), float_to_bf16_bits(z1[k] > 0.0f ? d[k] : 0.0f));
            net_sync();
            if (me == 0) {
#pragma unroll 1
                for (int q = 0; q < kMHBlock / 16; q++)
                    tc::mma_bf16(S.tmem, tc::desc_operand(T.ga, kMHBlock, 16 * q),
                                 tc::desc_operand(T.gb, kMHBlock, 16 * q), kIdesc80, q > 0 ? 1u : 0u);
                tc::mma_commit(&S.mbar);
            }
            ok = net_wait(S, mph);
        }
    }
    T.sst[me][0] = loss; T.sst[me][1] = esjd; T.sst[me][2] = accm; T.sst[me][3] = one;
    __syncthreads();
    float *out = partials + (size_t)blockIdx.x * (kNP + 4);
    if (ok) {
        const int w = me >> 5, l = me & 31;
        const uint32_t lanes = S.tmem + ((uint32_t)(w * 32) << 16);
        float d[32], e[32];
        if (w == 0) {                                   // rows j: dW2[j][k] (columns 0..31), db2[j] (column 72)
            tc::tmem_ld32(lanes, d);
            tc::tmem_ld32(lanes + 64, e);
#pragma unroll
            for (int k = 0; k < kNH; k++) out[kW2 + l * kNH + k] = d[k];
            out[kB2 + l] = e[8];
        } else if (w == 1) {                            // rows 32 + j: dW1[j][k] (columns 64..71), db1[j] (72)
            tc::tmem_ld32(lanes + 64, e);
#pragma unroll
            for (int k = 0; k < kNF; k++) out[kW1 + l * kNF + k] = e[k];
            out[kB1 + l] = e[8];
        } else if (w == 2) {                            // row 64: dw3[j] (columns 32..63), db3 (72)
            tc::tmem_ld32(lanes + 32, d);
            tc::tmem_ld32(lanes + 64, e);
            if (l == 0) {
#pragma unroll
                for (int k = 0; k < kNH; k++) out[kW3 + k] = d[k];
                out[kB3] = e[8];
            }
        }
    } else if (me == 0) {
        atomicOr(err, 1u);
    }
    for (int q = me; q < 4; q += kMHBlock) {            // statistics: FP32 sums in thread order
        float a = 0.0f;
        for (int u = 0; u < kMHBlock; u++) a += T.sst[u][q];
        out[kNP + q] = a;
    }
    net_teardown(S, 128, ok, mph);
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
                            int nhit, unsigned long long *acc_count, double *jump_sum, float *eps_out, unsigned *err,
                            cudaStream_t s)
{
    Field<float> U{ (float4 *)links, G.pstride };
    const unsigned nb = (G.half + kMHBlock - 1) / kMHBlock;
#define QG_MH(MU)                                                                                            \
    do {                                                                                                     \
        if (eps_out)                                                                                         \
            k_mh_phase<MU, true><<<nb, kMHBlock, 0, s>>>(U, G, a, wq, eps_max, nhit, acc_count, jump_sum, eps_out, \
                                                          err);                                              \
        else                                                                                                 \
            k_mh_phase<MU, false><<<nb, kMHBlock, 0, s>>>(U, G, a, wq, eps_max, nhit, acc_count, jump_sum,     \
                                                           nullptr, err);                                    \
    } while (0)
    switch (a.dir) {
    case 0: QG_MH(0); break;
    case 1: QG_MH(1); break;
    case 2: QG_MH(2); break;
    default: QG_MH(3); break;
    }
#undef QG_MH
    return cudaGetLastError();
}

uint32_t mh_grad_blocks(const Geom &G) { return (G.half + kMHBlock - 1) / kMHBlock; }

template <int mu>
static cudaError_t grad_launch(unsigned nb, Field<float> U, const Geom &G, int parity, const double *params,
                               const uint16_t *wq, double eps_max, uint2 key, uint64_t phase, float *partials,
                               unsigned *err, cudaStream_t s)
{
    static bool attr = false;               // the dynamic shared memory above 48 KB, once per instantiation
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_mh_grad<mu>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGradSmem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    k_mh_grad<mu><<<nb, kMHBlock, kGradSmem, s>>>(U, G, parity, params, wq, eps_max, key, phase, partials, err);
    return cudaGetLastError();
}

cudaError_t launch_mh_grad(const Geom &G, const void *links, int parity, int dir, const double *params,
                           const uint16_t *wq, double eps_max, uint2 key, uint64_t phase, float *partials,
                           float *grad, unsigned *err, cudaStream_t s)
{
    Field<float> U{ (float4 *)links, G.pstride };
    const unsigned nb = mh_grad_blocks(G);
    cudaError_t e;
    switch (dir) {
    case 0: e = grad_launch<0>(nb, U, G, parity, params, wq, eps_max, key, phase, partials, err, s); break;
    case 1: e = grad_launch<1>(nb, U, G, parity, params, wq, eps_max, key, phase, partials, err, s); break;
    case 2: e = grad_launch<2>(nb, U, G, parity, params, wq, eps_max, key, phase, partials, err, s); break;
    default: e = grad_launch<3>(nb, U, G, parity, params, wq, eps_max, key, phase, partials, err, s); break;
    }
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
