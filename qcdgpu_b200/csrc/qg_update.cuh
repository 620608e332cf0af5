// qg_update.cuh -- the checkerboard phase kernel: one thread per link of
// one (parity, direction) class; staple from the 18 neighbouring links,
// then Cabibbo-Marinari heatbath / overrelaxation (SU(3)) or Kennedy-
// Pendleton heatbath / reflection (SU(2)), stored in place.
// Restates update_{even,odd}_{X,Y,Z,T} (SU(N)/suncl/suncl.cl:399-975),
// lattice_staple_3 / lattice_staple_2 (su3_update_cl.cl:341-565,
// su2_update_cl.cl:206-431).
#pragma once
#include "qg_internal.h"
#include "qg_pair.cuh"

namespace qg {

template <typename Real>
struct Twist {
    int on;
    Real phi, omega;
    int xlast;
};

template <typename Real>
__device__ __forceinline__ G3<Real> load3t(const Field<Real> &U, int dir, uint32_t e, int xc, const Twist<Real> &tw)
{
    G3<Real> m = U.ldg3(dir, e);
    if (tw.on && dir == 1 && xc == tw.xlast) m = twist3(m, tw.phi, tw.omega);
    return m;
}
template <typename Real>
__device__ __forceinline__ R4<Real> load2t(const Field<Real> &U, int dir, uint32_t e, int xc, const Twist<Real> &tw)
{
    R4<Real> m = U.ldg2(dir, e);
    if (tw.on && dir == 1 && xc == tw.xlast) {
        R4<Real> om = { RC<Real>::cs(tw.phi / 2), 0, RC<Real>::sn(tw.phi / 2), 0 };
        m = times2(om, m);
    }
    return m;
}

// the reference's fixed plane order: mu=X: Y,Z,T; Y: X,Z,T; Z: Y,X,T; T: Y,Z,X
__host__ __device__ constexpr int nu_of(int mu, int i)
{
    return (i == 0) ? (mu == 1 ? 0 : 1) : (i == 1) ? (mu == 2 ? 0 : 2) : (mu == 3 ? 0 : 3);
}

// Neighbour offsets in checkerboard half-index space.  With N2 even the
// half index of a site is h = (y>>1) + (N2/2)(z + N3 t + N3 N4 x), so a
// shift along one direction changes h by an amount that depends only on
// that direction's coordinate (and y's parity), and two shifts along
// different directions add: h(x - nu + mu) = h + dm[nu] + dp[mu].
struct Nbr {
    int32_t dp[4], dm[4];
    int x, xp, xm;          // x coordinates of the site and of its x neighbours
};

__device__ __forceinline__ Nbr neighbours(const Geom &G, const Crd &c)
{
    Nbr n;
    const int32_t Y2 = G.n[1] >> 1;
    const int32_t sz = Y2, st = Y2 * G.n[2], sx = st * G.n[3];
    // y: y+1 changes y>>1 by (y odd); the wrap from N2-1 to 0 by -(Y2-1)
    n.dp[1] = (c.y == G.n[1] - 1) ? -(Y2 - 1) : (c.y & 1);
    n.dm[1] = (c.y == 0) ? (Y2 - 1) : -((c.y & 1) ^ 1);
    n.dp[2] = (c.z == G.n[2] - 1) ? -sz * (G.n[2] - 1) : sz;
    n.dm[2] = (c.z == 0) ? sz * (G.n[2] - 1) : -sz;
    n.dp[3] = (c.t == G.n[3] - 1) ? -st * (G.n[3] - 1) : st;
    n.dm[3] = (c.t == 0) ? st * (G.n[3] - 1) : -st;
    n.dp[0] = (c.x == G.n[0] - 1) ? -sx * (G.n[0] - 1) : sx;
    n.dm[0] = (c.x == 0) ? sx * (G.n[0] - 1) : -sx;
    n.x = c.x;
    n.xp = (c.x == G.n[0] - 1) ? 0 : c.x + 1;
    n.xm = (c.x == 0) ? G.n[0] - 1 : c.x - 1;
    return n;
}

// staple of U_mu(x), lattice_staple_3 (su3_update_cl.cl:341-565): per
// plane nu the forward term U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+ and the
// backward term U_nu(x-nu+mu)^+ U_mu(x-nu)^+ U_nu(x-nu), summed as
// st = f0 + b0; st = b_i + (st + f_i)
template <int mu, typename Real>
__device__ __forceinline__ M3<Real> staple3(const Field<Real> &U, const Geom &G, uint32_t t, const Nbr &n, int p,
                                           const Twist<Real> &tw)
{
    const uint32_t own = (uint32_t)p * G.cb + t, opp = (uint32_t)(p ^ 1) * G.cb + t;
    const int xmu = (mu == 0) ? n.xp : n.x;
    M3<Real> st, s2;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const int nu = nu_of(mu, i);
        const int xnp = (nu == 0) ? n.xp : n.x, xnm = (nu == 0) ? n.xm : n.x;
        const int xnmmu = (nu == 0) ? n.xm : xmu;
        M3<Real> fw = staple_fwd3(load3t(U, nu, opp + n.dp[mu], xmu, tw), load3t(U, mu, opp + n.dp[nu], xnp, tw),
                                  load3t(U, nu, own, n.x, tw));
        M3<Real> bw = staple_bwd3(load3t(U, nu, own + n.dm[nu] + n.dp[mu], xnmmu, tw),
                                  load3t(U, mu, opp + n.dm[nu], xnm, tw), load3t(U, nu, opp + n.dm[nu], xnm, tw));
        if (i == 0) {
            add3(st, fw, bw);
        } else {
            add3(s2, st, fw);
            add3(st, bw, s2);
        }
    }
    return st;
}

template <int mu, typename Real>
__device__ __forceinline__ S2<Real> staple2(const Field<Real> &U, const Geom &G, uint32_t t, const Nbr &n, int p,
                                           const Twist<Real> &tw)
{
    const uint32_t own = (uint32_t)p * G.cb + t, opp = (uint32_t)(p ^ 1) * G.cb + t;
    const int xmu = (mu == 0) ? n.xp : n.x;
    S2<Real> st, s2;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const int nu = nu_of(mu, i);
        const int xnp = (nu == 0) ? n.xp : n.x, xnm = (nu == 0) ? n.xm : n.x;
        const int xnmmu = (nu == 0) ? n.xm : xmu;
        S2<Real> fw = staple_fwd2(load2t(U, nu, opp + n.dp[mu], xmu, tw), load2t(U, mu, opp + n.dp[nu], xnp, tw),
                                  load2t(U, nu, own, n.x, tw));
        S2<Real> bw = staple_bwd2(load2t(U, nu, own + n.dm[nu] + n.dp[mu], xnmmu, tw),
                                  load2t(U, mu, opp + n.dm[nu], xnm, tw), load2t(U, nu, opp + n.dm[nu], xnm, tw));
        if (i == 0) {
            st = add2(fw, bw);
        } else {
            s2 = add2(st, fw);
            st = add2(bw, s2);
        }
    }
    return st;
}

// ------------------------------------------ staple links through shared memory
// The staged form of staple3 (SU(3), FP32 links): each staple term's three
// links (nine 16-byte plane entries per thread) are copied global -> shared
// with cp.async two terms ahead of their use, so a warp keeps the next
// term's loads in flight while it multiplies the current one instead of
// holding them in registers.  A thread only reads back what it copied
// itself, so no block barrier is needed; the arithmetic is staple3's.
constexpr int kPhaseBlock = 128;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// slots of 16 bytes x kPhaseBlock threads: two term buffers of 9 slots
// (3 links x 3 planes); the updated link itself goes into the forward
// buffer once the last forward term has been read (36 KB per block, so
// five blocks fit an SM with room to spare)
constexpr int kTermSlots = 9, kOwnSlot = 0, kStageSlots = 2 * kTermSlots;
using StageBuf = float4[kStageSlots][kPhaseBlock];

__device__ __forceinline__ void stage_link(const Field<float> &U, int dir, uint32_t e, StageBuf &sb, int slot)
{
#pragma unroll
    for (int c = 0; c < 3; c++) cp_async16(&sb[slot + c][threadIdx.x], U.p + (size_t)(dir + 4 * c) * U.pstride + e);
}
__device__ __forceinline__ G3<float> unstage_link(const StageBuf &sb, int slot)
{
    G3<float> m;
    float4 a = sb[slot][threadIdx.x], b = sb[slot + 1][threadIdx.x], d = sb[slot + 2][threadIdx.x];
    m.uv1 = { a.x, a.y, a.z, a.w };
    m.uv2 = { b.x, b.y, b.z, b.w };
    m.uv3 = { d.x, d.y, d.z, d.w };
    return m;
}

// the plane-nu neighbour offsets for a runtime nu (selects, no local memory)
__device__ __forceinline__ int32_t pick4(const int32_t (&a)[4], int k)
{
    return k == 0 ? a[0] : k == 1 ? a[1] : k == 2 ? a[2] : a[3];
}

// staple3 with staged loads, as a loop over the three planes (one copy of
// the forward and backward term code, so the kernel's instruction stream
// stays small); also brings in the updated link U_mu(x).  Term buffer 0
// holds the forward term of the plane, buffer 1 the backward term; the
// next plane's copies are issued as soon as a buffer has been read; on the
// last plane the forward buffer receives U_mu(x) instead, so its copy runs
// under the last backward term.  Every iteration commits one group per
// buffer (the last backward group is empty) so that wait_group 1 always
// means "this buffer has landed".
template <int mu>
__device__ __forceinline__ M3<float> staple3_staged(const Field<float> &U, const Geom &G, uint32_t t, const Nbr &n,
                                                   int p, const Twist<float> &tw, StageBuf &sb, G3<float> &m0)
{
    const uint32_t own = (uint32_t)p * G.cb + t, opp = (uint32_t)(p ^ 1) * G.cb + t;
    const int xmu = (mu == 0) ? n.xp : n.x;
    auto fwd_copy = [&](int nu) {
        stage_link(U, nu, opp + n.dp[mu], sb, 0);
        stage_link(U, mu, opp + pick4(n.dp, nu), sb, 3);
        stage_link(U, nu, own, sb, 6);
    };
    auto bwd_copy = [&](int nu) {
        const int32_t dmn = pick4(n.dm, nu);
        stage_link(U, nu, own + dmn + n.dp[mu], sb, kTermSlots);
        stage_link(U, mu, opp + dmn, sb, kTermSlots + 3);
        stage_link(U, nu, opp + dmn, sb, kTermSlots + 6);
    };
    auto get = [&](int slot, int dir, int xc) {
        G3<float> m = unstage_link(sb, slot);
        if (tw.on && dir == 1 && xc == tw.xlast) m = twist3(m, tw.phi, tw.omega);
        return m;
    };
    fwd_copy(nu_of(mu, 0));
    cp_async_commit();
    bwd_copy(nu_of(mu, 0));
    cp_async_commit();
    MR3 st, s2;
#pragma unroll 1
    for (int i = 0; i < 3; i++) {
        const int nu = nu_of(mu, i);
        const int xnp = (nu == 0) ? n.xp : n.x, xnm = (nu == 0) ? n.xm : n.x;
        const int xnmmu = (nu == 0) ? n.xm : xmu;
        cp_async_wait<1>();
        MR3 fw = staple_fwd3_rows(get(0, nu, xmu), get(3, mu, xnp), get(6, nu, n.x));
        if (i < 2)
            fwd_copy(nu_of(mu, i + 1));
        else
            stage_link(U, mu, own, sb, kOwnSlot);
        cp_async_commit();
        cp_async_wait<1>();
        MR3 bw = staple_bwd3_rows(get(kTermSlots, nu, xnmmu), get(kTermSlots + 3, mu, xnm),
                                  get(kTermSlots + 6, nu, xnm));
        if (i < 2) bwd_copy(nu_of(mu, i + 1));
        cp_async_commit();
        if (i == 0) {
            mr_add(st, fw, bw);
        } else {
            mr_add(s2, st, fw);
            mr_add(st, bw, s2);
        }
    }
    cp_async_wait<0>();
    m0 = unstage_link(sb, kOwnSlot);
    return mr_unpack(st);
}

// PRN source of thread t (PMODE 0 = RANLUX buffer, 1 = Philox, 2 = gid)
template <typename Real, int PMODE> struct PrnOf;
template <typename Real> struct PrnOf<Real, 0> {
    using T = PrnBuffer<Real>;
    __device__ static T make(const PhaseArgs &A, uint32_t t, uint32_t, uint64_t, const Geom &)
    {
        T p; p.prns = A.prns; p.idx = t; p.step = A.prngstep; return p;
    }
};
template <typename Real> struct PrnOf<Real, 1> {
    using T = PrnPhilox<Real>;
    __device__ static T make(const PhaseArgs &A, uint32_t t, uint32_t, uint64_t phase, const Geom &)
    {
        T p; p.key = A.key; p.t = (uint32_t)((int32_t)t + A.t_prn); p.k = 0; p.plo = (uint32_t)phase;
        p.phi = (uint32_t)(phase >> 32); return p;
    }
};
template <typename Real> struct PrnOf<Real, 2> {
    using T = PrnGid<Real>;
    __device__ static T make(const PhaseArgs &A, uint32_t, uint32_t site, uint64_t, const Geom &G)
    {
        T p; p.g = (double)(float)site; p.V = (double)G.V; p.nhit = A.nhit; return p;
    }
};

// MINB: minimum resident blocks of 128 threads per SM asked of the
// compiler (0 = its own register choice); the launch shapes the tuner picks
// The update of link U_mu(x) for thread t of a (parity, mu) phase: the
// body of update_{even,odd}_{X,Y,Z,T}.  STAGED: staple links through
// shared memory (staple3_staged; SU(3) FP32 links).
// TW: twisted boundaries possible (the launch has A.twist set); without it
// every twist test folds away at compile time (4 % of the phase's time)
// sb: the block's staging buffer (STAGED; declared by the kernel, so that a
// kernel running several directions holds one)
template <int NC, typename Real, int PMODE, bool OR, int mu, bool STAGED, bool TW = false>
__device__ __forceinline__ void phase_site(const Field<Real> &U, const Geom &G, const PhaseArgs &A, uint32_t t,
                                           StageBuf *sb)
{
    const int p = A.parity;
    Crd c = lex2crd(G, 2 * t);
    if (parity_of(c) != p) c.y += 1;                 // lattice_{even,odd}_gid
    const uint32_t site = 2 * t + (uint32_t)(c.y & 1);
    const uint32_t e0 = (uint32_t)p * G.cb + t;
    const Nbr nb = neighbours(G, c);
    Twist<Real> tw;
    tw.on = TW ? A.twist : 0;
    tw.xlast = G.n[0] - 1;
    tw.phi = (Real)(float)A.params[1]; tw.omega = (Real)(float)A.params[2];
    if (sizeof(Real) == 8) { tw.phi = (Real)A.params[1]; tw.omega = (Real)A.params[2]; }
    const Real beta = (Real)A.params[0];            // lattice_parameters[0] = BETA/N
    const uint64_t phase = (PMODE == 1) ? (*A.phase_base + A.phase_offset) : 0;
    auto prn = PrnOf<Real, PMODE>::make(A, t, site, phase, G);
    if (NC == 3) {
        G3<Real> m0;
        M3<Real> st;
        if constexpr (STAGED) {
            st = staple3_staged<mu>(U, G, t, nb, p, tw, *sb, m0);
        } else {
            m0 = U.ld3(mu, e0);
            st = staple3<mu>(U, G, t, nb, p, tw);
        }
        if (tw.on && mu == 1 && c.x == tw.xlast) m0 = twist3(m0, tw.phi, tw.omega);
        G3<Real> mU;
        if constexpr (STAGED && OR)
            mU = cm3_or_rows(st, m0, A.nhitpar);
        else
            mU = cm3<Real, OR, decltype(prn), STAGED && !OR>(st, m0, beta, prn, A.nhit, A.nhitpar);
        U.st3(mu, e0, mU);
    } else {
        R4<Real> m0 = U.ld2(mu, e0);
        if (tw.on && mu == 1 && c.x == tw.xlast) {
            R4<Real> om = { RC<Real>::cs(tw.phi / 2), 0, RC<Real>::sn(tw.phi / 2), 0 };
            m0 = times2(om, m0);
        }
        S2<Real> st = staple2<mu>(U, G, t, nb, p, tw);
        if (!OR) {
            S2<Real> a = st;
            if (kp_step<Real, false>(a, beta, prn, A.nhit))
                U.st2(mu, e0, R4<Real>{ a.u1.re, a.u2.re, a.u1.im, a.u2.im });
            else
                U.st2(mu, e0, m0);
        } else {
            Real Mx = st.u1.re + st.v2.re, My = st.u1.im - st.v2.im;
            Real Mz = st.u2.re - st.v1.re, Mw = st.u2.im + st.v1.im;
            Real n2 = Mx * Mx;
            n2 = FMA(My, My, n2); n2 = FMA(Mz, Mz, n2); n2 = FMA(Mw, Mw, n2);
            Real id = (Real)1 / RC<Real>::sq(n2);
            R4<Real> aH = { Mx * id, -Mz * id, -My * id, -Mw * id };
            U.st2(mu, e0, times2(times2(aH, herm2(m0)), aH));
        }
    }
}

template <int NC, typename Real, int PMODE, bool OR, int mu, int MINB, bool STAGED, bool TW>
__global__ void __launch_bounds__(kPhaseBlock, MINB) k_phase(Field<Real> U, Geom G, PhaseArgs A)
{
    const uint32_t t = A.t_begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.t_end) return;
    if constexpr (STAGED) {
        __shared__ __align__(16) StageBuf sb;
        phase_site<NC, Real, PMODE, OR, mu, STAGED, TW>(U, G, A, t, &sb);
    } else {
        phase_site<NC, Real, PMODE, OR, mu, STAGED, TW>(U, G, A, t, nullptr);
    }
}

// Overrelaxation of two links per thread (t and t + ceil(half/2)) with the
// packed FP32 algebra of qg_pair.cuh: each lane performs the scalar
// kernel's operations in the same order (bit-identical results) while one
// FFMA2 issue serves both links.  SU(3), FP32 links, periodic boundaries;
// the running staple sum is kept as s2 = st + f_i (f_0 alone for the first
// plane), then st = b_i + s2 -- the scalar order, with the first sum
// written b_0 + f_0 (addition commutes exactly).
template <int mu>
__global__ void __launch_bounds__(kPhaseBlock, 1) k_phase_or_pair(Field<float> U, Geom G, PhaseArgs A)
{
    const uint32_t H = (G.half + 1) >> 1;
    const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (t0 >= H) return;
    uint32_t t1 = t0 + H;
    const bool two = t1 < G.half;
    if (!two) t1 = t0;
    const int p = A.parity;
    Crd c0 = lex2crd(G, 2 * t0);
    if (parity_of(c0) != p) c0.y += 1;
    Crd c1 = lex2crd(G, 2 * t1);
    if (parity_of(c1) != p) c1.y += 1;
    const Nbr n0 = neighbours(G, c0), n1 = neighbours(G, c1);
    const uint32_t own0 = (uint32_t)p * G.cb + t0, opp0 = (uint32_t)(p ^ 1) * G.cb + t0;
    const uint32_t own1 = (uint32_t)p * G.cb + t1, opp1 = (uint32_t)(p ^ 1) * G.cb + t1;
    M32 st, s2;
#pragma unroll 1
    for (int i = 0; i < 3; i++) {
        const int nu = nu_of(mu, i);
        const int32_t dpn0 = pick4(n0.dp, nu), dpn1 = pick4(n1.dp, nu);
        const int32_t dmn0 = pick4(n0.dm, nu), dmn1 = pick4(n1.dm, nu);
        {
            M32 fw = pstaple_fwd3(gpair(U.ldg3(nu, opp0 + n0.dp[mu]), U.ldg3(nu, opp1 + n1.dp[mu])),
                                  gpair(U.ldg3(mu, opp0 + dpn0), U.ldg3(mu, opp1 + dpn1)),
                                  gpair(U.ldg3(nu, own0), U.ldg3(nu, own1)));
            if (i == 0) s2 = fw;
            else padd3(s2, st, fw);
        }
        M32 bw = pstaple_bwd3(gpair(U.ldg3(nu, own0 + dmn0 + n0.dp[mu]), U.ldg3(nu, own1 + dmn1 + n1.dp[mu])),
                              gpair(U.ldg3(mu, opp0 + dmn0), U.ldg3(mu, opp1 + dmn1)),
                              gpair(U.ldg3(nu, opp0 + dmn0), U.ldg3(nu, opp1 + dmn1)));
        padd3(st, bw, s2);
    }
    const G32 r = pcm3_or(st, gpair(U.ld3(mu, own0), U.ld3(mu, own1)), A.nhitpar);
    G3<float> r0, r1;
    gsplit(r, r0, r1);
    U.st3(mu, own0, r0);
    if (two) U.st3(mu, own1, r1);
}

template <typename Real>
cudaError_t launch_phase_T(const Geom &G, void *links, int group, const PhaseArgs &a, cudaStream_t s)
{
    Field<Real> U;
    U.p = reinterpret_cast<typename V4<Real>::T *>(links);
    U.pstride = G.pstride;
    const int bs = kPhaseBlock;
    const unsigned nb = (a.t_end - a.t_begin + bs - 1) / bs;
    const int pm = a.prn_mode;   // -1 selects overrelaxation (no PRNs)
    // shapes 3, 4 stage the staple through shared memory where that form
    // exists (SU(3), FP32 links); elsewhere they run shapes 0, 1
    constexpr bool kStage = sizeof(Real) == 4;
    // shape 5: overrelaxation two links per thread (SU(3), FP32, periodic,
    // the whole lattice); otherwise it runs shape 4
    if constexpr (sizeof(Real) == 4) {
        if (a.variant == 5 && group == 3 && pm == -1 && !a.twist && a.t_begin == 0 && a.t_end == G.half) {
            const unsigned nbp = ((G.half + 1) / 2 + bs - 1) / bs;
            switch (a.dir) {
            case 0: k_phase_or_pair<0><<<nbp, bs, 0, s>>>(U, G, a); break;
            case 1: k_phase_or_pair<1><<<nbp, bs, 0, s>>>(U, G, a); break;
            case 2: k_phase_or_pair<2><<<nbp, bs, 0, s>>>(U, G, a); break;
            default: k_phase_or_pair<3><<<nbp, bs, 0, s>>>(U, G, a); break;
            }
            return cudaGetLastError();
        }
    }
    // twisted boundaries: shape 0's form with the twist tests compiled in
    // (any shape computes the same sequence); the others are compiled
    // without them
#define QG_LAUNCH2(NC, PM, OR, MU, MB, ST) k_phase<NC, Real, PM, OR, MU, MB, ST, false><<<nb, bs, 0, s>>>(U, G, a)
#define QG_LAUNCH1(NC, PM, OR, MU)                                                  \
    do {                                                                            \
        if (a.twist) k_phase<NC, Real, PM, OR, MU, 0, false, true><<<nb, bs, 0, s>>>(U, G, a); \
        else if (a.variant == 1) QG_LAUNCH2(NC, PM, OR, MU, 5, false);              \
        else if (a.variant == 2) QG_LAUNCH2(NC, PM, OR, MU, 6, false);              \
        else if (a.variant == 3) QG_LAUNCH2(NC, PM, OR, MU, 0, NC == 3 && kStage);  \
        else if (a.variant >= 4) QG_LAUNCH2(NC, PM, OR, MU, 5, NC == 3 && kStage);  \
        else QG_LAUNCH2(NC, PM, OR, MU, 0, false);                                  \
    } while (0)
#define QG_LAUNCH(NC, PM, OR)                                     \
    do {                                                          \
        switch (a.dir) {                                          \
        case 0: QG_LAUNCH1(NC, PM, OR, 0); break;                 \
        case 1: QG_LAUNCH1(NC, PM, OR, 1); break;                 \
        case 2: QG_LAUNCH1(NC, PM, OR, 2); break;                 \
        default: QG_LAUNCH1(NC, PM, OR, 3); break;                \
        }                                                         \
    } while (0)
    if (group == 3) {
        if (pm == -1) QG_LAUNCH(3, 0, true);
        else if (pm == 0) QG_LAUNCH(3, 0, false);
        else if (pm == 1) QG_LAUNCH(3, 1, false);
        else QG_LAUNCH(3, 2, false);
    } else {
        if (pm == -1) QG_LAUNCH(2, 0, true);
        else if (pm == 0) QG_LAUNCH(2, 0, false);
        else if (pm == 1) QG_LAUNCH(2, 1, false);
        else QG_LAUNCH(2, 2, false);
    }
#undef QG_LAUNCH
#undef QG_LAUNCH1
#undef QG_LAUNCH2
    return cudaGetLastError();
}

}  // namespace qg
