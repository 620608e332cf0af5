// qg_update.cuh -- the checkerboard phase kernel: one thread per link of
// one (parity, direction) class; staple from the 18 neighbouring links,
// then Cabibbo-Marinari heatbath / overrelaxation (SU(3)) or Kennedy-
// Pendleton heatbath / reflection (SU(2)), stored in place.
// Restates update_{even,odd}_{X,Y,Z,T} (SU(N)/suncl/suncl.cl:399-975),
// lattice_staple_3 / lattice_staple_2 (su3_update_cl.cl:341-565,
// su2_update_cl.cl:206-431).
#pragma once
#include "qg_internal.h"

namespace qg {

template <typename Real>
struct Twist {
    int on;
    Real phi, omega;
    int xlast;
};

template <typename Real>
__device__ __forceinline__ G3<Real> load3t(const Field<Real> &U, int dir, uint32_t e, const Crd &c, const Twist<Real> &tw)
{
    G3<Real> m = U.ldg3(dir, e);
    if (tw.on && dir == 1 && c.x == tw.xlast) m = twist3(m, tw.phi, tw.omega);
    return m;
}
template <typename Real>
__device__ __forceinline__ R4<Real> load2t(const Field<Real> &U, int dir, uint32_t e, const Crd &c, const Twist<Real> &tw)
{
    R4<Real> m = U.ldg2(dir, e);
    if (tw.on && dir == 1 && c.x == tw.xlast) {
        R4<Real> om = { RC<Real>::cs(tw.phi / 2), 0, RC<Real>::sn(tw.phi / 2), 0 };
        m = times2(om, m);
    }
    return m;
}

// the reference's fixed plane order: mu=X: Y,Z,T; Y: X,Z,T; Z: Y,X,T; T: Y,Z,X
__device__ __forceinline__ int nu_of(int mu, int i)
{
    return (i == 0) ? (mu == 1 ? 0 : 1) : (i == 1) ? (mu == 2 ? 0 : 2) : (mu == 3 ? 0 : 3);
}

template <typename Real>
__device__ __forceinline__ M3<Real> staple3(const Field<Real> &U, const Geom &G, const Crd &c, int p, int mu,
                                           const Twist<Real> &tw)
{
    const Crd cp = step_plus(G, c, mu);
    const uint32_t e_cp = cb_index(G, cp, p ^ 1);
    const uint32_t e_c = (uint32_t)p * G.cb + (crd2lex(G, c) >> 1);
    M3<Real> st, s2;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const int nu = nu_of(mu, i);
        const Crd cn = step_plus(G, c, nu);
        const Crd cm = step_minus(G, c, nu);
        const Crd cmp = step_plus(G, cm, mu);
        const uint32_t e_cn = cb_index(G, cn, p ^ 1), e_cm = cb_index(G, cm, p ^ 1), e_cmp = cb_index(G, cmp, p);
        M3<Real> fw = staple_fwd3(load3t(U, nu, e_cp, cp, tw), load3t(U, mu, e_cn, cn, tw), load3t(U, nu, e_c, c, tw));
        M3<Real> bw = staple_bwd3(load3t(U, nu, e_cmp, cmp, tw), load3t(U, mu, e_cm, cm, tw), load3t(U, nu, e_cm, cm, tw));
        if (i == 0) {
            add3(st, fw, bw);
        } else {
            add3(s2, st, fw);
            add3(st, bw, s2);
        }
    }
    return st;
}

template <typename Real>
__device__ __forceinline__ S2<Real> staple2(const Field<Real> &U, const Geom &G, const Crd &c, int p, int mu,
                                           const Twist<Real> &tw)
{
    const Crd cp = step_plus(G, c, mu);
    const uint32_t e_cp = cb_index(G, cp, p ^ 1);
    const uint32_t e_c = (uint32_t)p * G.cb + (crd2lex(G, c) >> 1);
    S2<Real> st, s2;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const int nu = nu_of(mu, i);
        const Crd cn = step_plus(G, c, nu);
        const Crd cm = step_minus(G, c, nu);
        const Crd cmp = step_plus(G, cm, mu);
        const uint32_t e_cn = cb_index(G, cn, p ^ 1), e_cm = cb_index(G, cm, p ^ 1), e_cmp = cb_index(G, cmp, p);
        S2<Real> fw = staple_fwd2(load2t(U, nu, e_cp, cp, tw), load2t(U, mu, e_cn, cn, tw), load2t(U, nu, e_c, c, tw));
        S2<Real> bw = staple_bwd2(load2t(U, nu, e_cmp, cmp, tw), load2t(U, mu, e_cm, cm, tw), load2t(U, nu, e_cm, cm, tw));
        if (i == 0) {
            st = add2(fw, bw);
        } else {
            s2 = add2(st, fw);
            st = add2(bw, s2);
        }
    }
    return st;
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
        T p; p.key = A.key; p.t = t; p.k = 0; p.plo = (uint32_t)phase; p.phi = (uint32_t)(phase >> 32); return p;
    }
};
template <typename Real> struct PrnOf<Real, 2> {
    using T = PrnGid<Real>;
    __device__ static T make(const PhaseArgs &A, uint32_t, uint32_t site, uint64_t, const Geom &G)
    {
        T p; p.g = (double)(float)site; p.V = (double)G.V; p.nhit = A.nhit; return p;
    }
};

template <int NC, typename Real, int PMODE, bool OR>
__global__ void __launch_bounds__(128) k_phase(Field<Real> U, Geom G, PhaseArgs A)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= G.half) return;
    const int p = A.parity, mu = A.dir;
    Crd c = lex2crd(G, 2 * t);
    if (parity_of(c) != p) c.y += 1;                 // lattice_{even,odd}_gid
    const uint32_t site = crd2lex(G, c);
    const uint32_t e0 = (uint32_t)p * G.cb + t;
    Twist<Real> tw;
    tw.on = A.twist; tw.xlast = G.n[0] - 1;
    tw.phi = (Real)(float)A.params[1]; tw.omega = (Real)(float)A.params[2];
    if (sizeof(Real) == 8) { tw.phi = (Real)A.params[1]; tw.omega = (Real)A.params[2]; }
    const Real beta = (Real)A.params[0];            // lattice_parameters[0] = BETA/N
    const uint64_t phase = (PMODE == 1) ? (*A.phase_base + A.phase_offset) : 0;
    auto prn = PrnOf<Real, PMODE>::make(A, t, site, phase, G);
    if (NC == 3) {
        G3<Real> m0 = U.ld3(mu, e0);
        if (tw.on && mu == 1 && c.x == tw.xlast) m0 = twist3(m0, tw.phi, tw.omega);
        M3<Real> st = staple3(U, G, c, p, mu, tw);
        G3<Real> mU = cm3<Real, OR>(st, m0, beta, prn, A.nhit, A.nhitpar);
        U.st3(mu, e0, mU);
    } else {
        R4<Real> m0 = U.ld2(mu, e0);
        if (tw.on && mu == 1 && c.x == tw.xlast) {
            R4<Real> om = { RC<Real>::cs(tw.phi / 2), 0, RC<Real>::sn(tw.phi / 2), 0 };
            m0 = times2(om, m0);
        }
        S2<Real> st = staple2(U, G, c, p, mu, tw);
        if (!OR) {
            S2<Real> a = st;
            if (kp_step<Real, false>(a, beta, prn, A.nhit))
                U.st2(mu, e0, R4<Real>{ a.u1.re, a.u2.re, a.u1.im, a.u2.im });
            else
                U.st2(mu, e0, m0);
        } else {
            Real Mx = st.u1.re + st.v2.re, My = st.u1.im - st.v2.im;
            Real Mz = st.u2.re - st.v1.re, Mw = st.u2.im + st.v1.im;
            Real det = RC<Real>::sq(Mx * Mx + My * My + Mz * Mz + Mw * Mw);
            R4<Real> aH = { Mx / det, -Mz / det, -My / det, -Mw / det };
            U.st2(mu, e0, times2(times2(aH, herm2(m0)), aH));
        }
    }
}

template <typename Real>
cudaError_t launch_phase_T(const Geom &G, void *links, int group, const PhaseArgs &a, cudaStream_t s)
{
    Field<Real> U;
    U.p = reinterpret_cast<typename V4<Real>::T *>(links);
    U.pstride = G.pstride;
    const int bs = 128;
    const unsigned nb = (G.half + bs - 1) / bs;
    const int pm = a.prn_mode;   // -1 selects overrelaxation (no PRNs)
#define QG_LAUNCH(NC, PM, OR) k_phase<NC, Real, PM, OR><<<nb, bs, 0, s>>>(U, G, a)
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
    return cudaGetLastError();
}

}  // namespace qg
