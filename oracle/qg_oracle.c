/*
 * qg_oracle.c -- CPU oracle for the SU(2)/SU(3) checkerboard link sweep.
 *
 * TEST INFRASTRUCTURE ONLY.  A plain-C restatement of the QCDGPU reference
 * (vadimdi/QCDGPU, SU(N)/) used by tests/ to check the CUDA product path.
 * The product never links or loads this file.  Each routine names the
 * reference file:line it restates.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "qg_oracle.h"

#define PASTE_(a, b) a##b
#define PASTE(a, b) PASTE_(a, b)

/* ======================================================= RANLUX + seeding */
#define RL_ICONS  2147483563
#define RL_ITWO24 16777216
#define RL_TWOM24 0.000000059604644775390625f
#define RL_TWOM12 0.000244140625f

int ol_sizeof_ranlux(void) { return (int)sizeof(ol_ranlux); }

/* PRNG::initialize -> RL_initialize_CPU -> RL_initialize seeding order
 * (random/random.cpp:228-235, 462-465, 508): srand(series); first rand()
 * (mod 2^31-1) seeds instance 0, the next instances-1 rand() calls seed the
 * other instances.  Uses the C library's own srand/rand, as the reference. */
void ol_glibc_seeds(uint32_t randseries, int instances, uint32_t *seeds)
{
    srand(randseries);
    int jseed = rand() % 2147483647;
    seeds[0] = (uint32_t)jseed;
    for (int i = 1; i < instances; i++) seeds[i] = (uint32_t)rand();
}

/* RL_initialize_CPU (random/random.cpp:504-522) and ranlux_init
 * (random/prngcl_ranlux.cl:97-157): 24 seeds from the 40014/53668 LCG. */
void ol_ranlux_init(ol_ranlux *st, int32_t jseed, int nskip)
{
    int32_t j = jseed;
    for (int i = 0; i < 24; i++) {
        int32_t k = j / 53668;
        j = 40014 * (j - k * 53668) - k * 12211;
        if (j < 0) j += RL_ICONS;
        st->seeds[i] = ((float)(j % RL_ITWO24)) * RL_TWOM24;
    }
    st->i24 = 23; st->j24 = 9; st->in24 = 0; st->nskip = nskip;
    st->carry = (st->seeds[23] == 0) ? RL_TWOM24 : 0.0f;
}

/* RL_produce_one_CPU (random/random.cpp:523-574): subtract-with-borrow with
 * luxury skip every 24 outputs; outputs below 2^-12 get 24 more bits. */
float ol_ranlux_next(ol_ranlux *st)
{
    float uni;
    if (st->in24 == 0) {
        st->in24 = 24;
        for (int isk = 0; isk < st->nskip; isk++) {
            uni = st->seeds[st->j24] - st->seeds[st->i24] - st->carry;
            if (uni < 0.0f) { uni += 1.0f; st->carry = RL_TWOM24; } else st->carry = 0.0f;
            st->seeds[st->i24] = uni;
            if (st->i24 == 0) st->i24 = 24;
            if (st->j24 == 0) st->j24 = 24;
            st->i24--; st->j24--;
        }
    }
    uni = st->seeds[st->j24] - st->seeds[st->i24] - st->carry;
    if (uni < 0.0f) { uni += 1.0f; st->carry = RL_TWOM24; } else st->carry = 0.0f;
    st->seeds[st->i24] = uni;
    if (st->i24 == 0) st->i24 = 24;
    if (st->j24 == 0) st->j24 = 24;
    st->i24--; st->j24--;
    if (uni < RL_TWOM12) {
        uni = uni + RL_TWOM24 * st->seeds[st->j24];
        if (uni == 0.0f) uni = RL_TWOM24 * RL_TWOM24;
    }
    st->in24--;
    return uni;
}

void ol_ranlux_states(const uint32_t *seeds, int instances, int nskip, ol_ranlux *states)
{
    for (int i = 0; i < instances; i++) ol_ranlux_init(&states[i], (int32_t)seeds[i], nskip);
}

/* ranlux kernel (random/prngcl_ranlux.cl:533-563): instance i writes its
 * s-th float4 (four consecutive outputs) to prns[s*instances + i]. */
void ol_ranlux_batch(ol_ranlux *states, int instances, int samples, float *prns)
{
    /* every instance runs its own generator: instances in parallel */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < instances; i++)
        for (int s = 0; s < samples; s++) {
            float *o = prns + ((size_t)s * instances + i) * 4;
            o[0] = ol_ranlux_next(&states[i]);
            o[1] = ol_ranlux_next(&states[i]);
            o[2] = ol_ranlux_next(&states[i]);
            o[3] = ol_ranlux_next(&states[i]);
        }
}

/* ======================================================= Philox4x32-10 */
/* Counter-based generator of Salmon, Moraes, Dror, Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3" (SC'11): 10 rounds of two 32x32->64
 * multiplies with Weyl-sequence key bumps.                                */
void ol_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* fast-mode PRN quad: counter (thread, k, phase lo, phase hi); each 32-bit
 * word becomes ((w>>8)|1) * 2^-24, an odd multiple of 2^-24 in (0,1). */
void ol_philox_prn(const ol_prn *src, uint32_t thread, uint32_t k, float out[4])
{
    uint32_t ctr[4] = { thread, k, (uint32_t)src->phase, (uint32_t)(src->phase >> 32) };
    uint32_t key[2] = { src->key0, src->key1 }, w[4];
    ol_philox4x32(ctr, key, w);
    for (int i = 0; i < 4; i++) out[i] = (float)((w[i] >> 8) | 1u) * RL_TWOM24;
}

/* ======================================================= geometry */
typedef struct { int x, y, z, t; } crd;

static inline int sites_of(const ol_cfg *c) { return c->n[0] * c->n[1] * c->n[2] * c->n[3]; }
static inline int has_twist(const ol_cfg *c) { return !(c->phi == 0.0 && c->omega == 0.0); }

/* lattice_gid_to_coords / lattice_coords_to_gid, sun_common.cl:41-66 */
static inline void gid2c(const ol_cfg *c, unsigned g, crd *o)
{
    unsigned n2 = c->n[1], n2n3 = c->n[1] * c->n[2], n2n3n4 = n2n3 * c->n[3];
    o->x = g / n2n3n4; g -= o->x * n2n3n4;
    o->t = g / n2n3;   g -= o->t * n2n3;
    o->z = g / n2;     o->y = g - o->z * n2;
}
static inline unsigned c2gid(const ol_cfg *c, crd o)
{
    return o.y + o.z * c->n[1] + o.t * c->n[1] * c->n[2] + o.x * c->n[1] * c->n[2] * c->n[3];
}
/* lattice_neighbours_gid(_minus), sun_common.cl:455-513 (periodic) */
static inline crd nb_plus(const ol_cfg *c, crd o, int d)
{
    switch (d) {
    case 0: if (++o.x >= c->n[0]) o.x = 0; break;
    case 1: if (++o.y >= c->n[1]) o.y = 0; break;
    case 2: if (++o.z >= c->n[2]) o.z = 0; break;
    default: if (++o.t >= c->n[3]) o.t = 0; break;
    }
    return o;
}
static inline crd nb_minus(const ol_cfg *c, crd o, int d)
{
    switch (d) {
    case 0: if (o.x <= 0) o.x = c->n[0]; o.x--; break;
    case 1: if (o.y <= 0) o.y = c->n[1]; o.y--; break;
    case 2: if (o.z <= 0) o.z = c->n[2]; o.z--; break;
    default: if (o.t <= 0) o.t = c->n[3]; o.t--; break;
    }
    return o;
}
/* lattice_even_gid / lattice_odd_gid, sun_common.cl:351-381 */
static inline unsigned even_gid(const ol_cfg *c, unsigned t)
{
    crd o; unsigned g = 2 * t; gid2c(c, g, &o);
    return g + ((o.x + o.y + o.z + o.t) & 1);
}
static inline unsigned odd_gid(const ol_cfg *c, unsigned t)
{
    crd o; unsigned g = 2 * t + 1; gid2c(c, g, &o);
    return g - (((o.x + o.y + o.z + o.t) & 1) ^ 1);
}

/* ======================================================= FP64 3x3 helpers */
typedef struct { double re, im; } cdd;
typedef struct { cdd m[3][3]; } cd3;

static void cd_mul(const cd3 *a, const cd3 *b, cd3 *o, int N)
{
    cd3 r;
    memset(&r, 0, sizeof(r));
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            double re = 0, im = 0;
            for (int k = 0; k < N; k++) {
                re += a->m[i][k].re * b->m[k][j].re - a->m[i][k].im * b->m[k][j].im;
                im += a->m[i][k].re * b->m[k][j].im + a->m[i][k].im * b->m[k][j].re;
            }
            r.m[i][j].re = re; r.m[i][j].im = im;
        }
    *o = r;
}
static void cd_herm(const cd3 *a, cd3 *o, int N)
{
    cd3 r;
    memset(&r, 0, sizeof(r));
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) { r.m[i][j].re = a->m[j][i].re; r.m[i][j].im = -a->m[j][i].im; }
    *o = r;
}
static double cd_retr(const cd3 *a, int N)
{
    double s = 0;
    for (int i = 0; i < N; i++) s += a->m[i][i].re;
    return s;
}

static inline int crd_get(crd o, int d) { return d == 0 ? o.x : d == 1 ? o.y : d == 2 ? o.z : o.t; }

/* -i Tr(P T_a), T_a = lambda_a / 2 for SU(3) (a = 1..8; trace_lambda1..8_double,
 * su3_measurements_cl.cl:355-460) or sigma_a / 2 for SU(2) (a = 1..3, real
 * part only; trace_sigma1..3_double, su2_measurements_cl.cl:89-124), from
 * the entries of P written out per generator; out = {Re, Im} */
static void gen_proj(const cd3 *P, int N, int a, double out[2])
{
    const cdd u1 = P->m[0][0], u2 = P->m[0][1], u3 = P->m[0][2];
    const cdd v1 = P->m[1][0], v2 = P->m[1][1], v3 = P->m[1][2];
    const cdd w1 = P->m[2][0], w2 = P->m[2][1], w3 = P->m[2][2];
    double re = 0, im = 0;
    if (N == 2) {
        re = a == 1 ? u2.im : a == 2 ? u2.re : u1.im;
    } else {
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
    out[0] = re; out[1] = im;
}

/* ======================================================= elementary functions */
/* sin/cos for |x| < 16: Cody-Waite reduction by pi/2 (three-part constant)
 * and Taylor polynomials of degree 17 / 18 on [-pi/4, pi/4], Horner with
 * fma; natural log by y = m 2^e, log m = 2 atanh((m-1)/(m+1)) to s^23.
 * The same operation sequence as the CUDA path's routines, so both sides
 * round identically. */
/* float sin/cos for |x| < 1024 (qg_sincosf of the kernels): Cody-Waite
 * reduction by pi/2 with a three-part float constant, Taylor polynomials of
 * degree 9 / 10 on [-pi/4, pi/4] in Horner form, every step in float */
static void ol_sincosf(float x, float *s, float *c)
{
    const float INV_PIO2 = 0.6366197466850281f;
    const float P1 = 1.5707963705062866f, P2 = -4.371138828673793e-08f, P3 = -1.7151245100058819e-15f;
    const float n = rintf(x * INV_PIO2);
    float f = fmaf(-n, P1, x);
    f = fmaf(-n, P2, f);
    f = fmaf(-n, P3, f);
    const float f2 = f * f;
    float ps = 2.7557318844628753e-06f;
    ps = fmaf(ps, f2, -1.9841270113829523e-04f);
    ps = fmaf(ps, f2, 8.333333767950535e-03f);
    ps = fmaf(ps, f2, -1.666666716337204e-01f);
    const float sn = fmaf(ps * f2, f, f);
    float pc = -2.755731998149713e-07f;
    pc = fmaf(pc, f2, 2.4801587642286904e-05f);
    pc = fmaf(pc, f2, -1.3888889225199819e-03f);
    pc = fmaf(pc, f2, 4.16666679084301e-02f);
    pc = fmaf(pc, f2, -0.5f);
    const float cs = fmaf(pc, f2, 1.0f);
    const int q = ((int)n) & 3;
    *s = (q == 0) ? sn : (q == 1) ? cs : (q == 2) ? -sn : -cs;
    *c = (q == 0) ? cs : (q == 1) ? -sn : (q == 2) ? -cs : sn;
}
float ol_sinf_own(float x) { float s, c; ol_sincosf(x, &s, &c); return s; }
float ol_cosf_own(float x) { float s, c; ol_sincosf(x, &s, &c); return c; }

static void ol_sincos(double x, double *s, double *c)
{
    const double INV_PIO2 = 0.63661977236758134308;
    const double P1 = 1.5707963267948966, P2 = 6.123233995736766e-17, P3 = -1.4973849048591698e-33;
    double n = rint(x * INV_PIO2);
    double f = fma(-n, P1, x);
    f = fma(-n, P2, f);
    f = fma(-n, P3, f);
    double f2 = f * f;
    double ps = 2.8114572543455206e-15;
    ps = fma(ps, f2, -7.6471637318198164e-13);
    ps = fma(ps, f2, 1.6059043836821613e-10);
    ps = fma(ps, f2, -2.5052108385441720e-08);
    ps = fma(ps, f2, 2.7557319223985893e-06);
    ps = fma(ps, f2, -1.9841269841269841e-04);
    ps = fma(ps, f2, 8.3333333333333333e-03);
    ps = fma(ps, f2, -1.6666666666666667e-01);
    double sn = fma(ps * f2, f, f);
    double pc = -1.5619206968586225e-16;
    pc = fma(pc, f2, 4.7794773323873853e-14);
    pc = fma(pc, f2, -1.1470745597729725e-11);
    pc = fma(pc, f2, 2.0876756987868099e-09);
    pc = fma(pc, f2, -2.7557319223985888e-07);
    pc = fma(pc, f2, 2.4801587301587302e-05);
    pc = fma(pc, f2, -1.3888888888888889e-03);
    pc = fma(pc, f2, 4.1666666666666667e-02);
    pc = fma(pc, f2, -0.5);
    double cs = fma(pc, f2, 1.0);
    int q = ((int)n) & 3;
    *s = (q == 0) ? sn : (q == 1) ? cs : (q == 2) ? -sn : -cs;
    *c = (q == 0) ? cs : (q == 1) ? -sn : (q == 2) ? -cs : sn;
}

/* natural log of a positive normal y, table-driven (P. T. P. Tang, ACM
 * TOMS 16 (1990) 378-400): y = 2^e m, m in [1, 2); k = the nearest multiple
 * of 1/128 to m - 1 from the top 8 mantissa bits; r = fma(m, c_k, -1),
 * |r| <= 2^-8; log1p(r) by its Taylor terms to r^7; log y = (e ln2_hi +
 * L_hi) + ((e ln2_lo + L_lo) + log1p(r)) with L = -log c_k.  The table is
 * the device routine's (qg_logtab.h), the operations qg_log's in order. */
#include "../qcdgpu_b200/csrc/qg_logtab.h"
static const double ol_log_c[QG_LOG_TABLE_SIZE] = QG_LOG_C_INIT;
static const double ol_log_hi[QG_LOG_TABLE_SIZE] = QG_LOG_LHI_INIT;
static const double ol_log_lo[QG_LOG_TABLE_SIZE] = QG_LOG_LLO_INIT;

static double ol_log(double y)
{
    int64_t b;
    memcpy(&b, &y, sizeof(b));
    const int e = (int)(b >> 52) - 1023;
    const int k = (int)(((b >> 44) & 0xFF) + 1) >> 1;
    const int64_t mb = (b & 0x000FFFFFFFFFFFFFLL) | 0x3FF0000000000000LL;
    double m;
    memcpy(&m, &mb, sizeof(m));
    const double r = fma(m, ol_log_c[k], -1.0);
    double q = 1.0 / 7.0;
    q = fma(q, r, -1.0 / 6.0);
    q = fma(q, r, 1.0 / 5.0);
    q = fma(q, r, -0.25);
    q = fma(q, r, 1.0 / 3.0);
    q = fma(q, r, -0.5);
    const double r2 = r * r;
    const double l1p = fma(r2, q, r);
    const double de = (double)e;
    const double hi = fma(de, QG_LN2_HI, ol_log_hi[k]);
    const double lo = fma(de, QG_LN2_LO, ol_log_lo[k]);
    return hi + (lo + l1p);
}

/* exp(x), |x| <= 700: x = k ln2 + r (Cody-Waite, two-part ln 2), Taylor
 * polynomial of degree 13 in Horner form, scaled by 2^k (exact); the
 * device routine qg_exp performs the same operations */
static double ol_exp(double x)
{
    x = fmin(fmax(x, -700.0), 700.0);
    const double LN2_HI = 6.93147180369123816490e-01, LN2_LO = 1.90821492927058770002e-10;
    const double k = rint(x * 1.44269504088896340736);
    double r = fma(-k, LN2_HI, x);
    r = fma(-k, LN2_LO, r);
    double p = 1.0 / 6227020800.0;
    p = fma(p, r, 1.0 / 479001600.0);
    p = fma(p, r, 1.0 / 39916800.0);
    p = fma(p, r, 1.0 / 3628800.0);
    p = fma(p, r, 1.0 / 362880.0);
    p = fma(p, r, 1.0 / 40320.0);
    p = fma(p, r, 1.0 / 5040.0);
    p = fma(p, r, 1.0 / 720.0);
    p = fma(p, r, 1.0 / 120.0);
    p = fma(p, r, 1.0 / 24.0);
    p = fma(p, r, 1.0 / 6.0);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    return ldexp(p, (int)k);
}
double ol_expd(double x) { return ol_exp(x); }

/* test-only: when set, the Kennedy-Pendleton step evaluates the reference's
 * expression for delta unfused, with the C library's cos / sin / log in
 * place of this build's routines (a measure of how far this build's own
 * arithmetic moves the chain; not what the device does) */
int ol_ref_arith = 0;
void ol_set_reference_arith(int on) { ol_ref_arith = on != 0; }

/* exported for the accuracy tests of the two routines */
double ol_sin(double x) { double s, c; ol_sincos(x, &s, &c); return s; }
double ol_cos(double x) { double s, c; ol_sincos(x, &s, &c); return c; }
double ol_logd(double x) { return ol_log(x); }

/* ======================================================= precision bodies */
#define REAL double
#define SFX _d
#define IS_F 0
#include "qg_oracle_impl.h"
#undef REAL
#undef SFX
#undef IS_F

#define REAL float
#define SFX _f
#define IS_F 1
#include "qg_oracle_impl.h"
#undef REAL
#undef SFX
#undef IS_F

/* ======================================================= public API */
#define DISPATCH(call_f, call_d) do { if (c->precision == 0) { call_f; } else { call_d; } } while (0)

void ol_init_cold(const ol_cfg *c, void *t) { DISPATCH(init_cold_f(c, (float *)t), init_cold_d(c, (double *)t)); }
void ol_init_gid(const ol_cfg *c, void *t)  { DISPATCH(init_gid_f(c, (float *)t), init_gid_d(c, (double *)t)); }
void ol_init_hot_dir(const ol_cfg *c, void *t, int dir, const float *prns)
{
    DISPATCH(init_hot_dir_f(c, (float *)t, dir, prns), init_hot_dir_d(c, (double *)t, dir, prns));
}
void ol_phase_hb(const ol_cfg *c, void *t, int parity, int dir, const ol_prn *src)
{
    DISPATCH(phase_f(c, (float *)t, parity, dir, src, 0), phase_d(c, (double *)t, parity, dir, src, 0));
}
void ol_phase_or(const ol_cfg *c, void *t, int parity, int dir)
{
    ol_prn none;
    memset(&none, 0, sizeof(none));
    DISPATCH(phase_f(c, (float *)t, parity, dir, &none, 1), phase_d(c, (double *)t, parity, dir, &none, 1));
}
void ol_gramschmidt(const ol_cfg *c, void *t) { DISPATCH(gramschmidt_f(c, (float *)t), gramschmidt_d(c, (double *)t)); }

/* FP64 reunitarisation of the stored links (new: REUNIT in double for FP32
 * links); same Gram-Schmidt steps as lattice_GramSchmidt3 in double. */
void ol_gramschmidt_fp64(const ol_cfg *c, void *t)
{
    if (c->precision != 0) { gramschmidt_d(c, (double *)t); return; }
    int V = sites_of(c);
    float *tf = (float *)t;
#pragma omp parallel for schedule(static)
    for (int g = 0; g < V; g++)
        for (int mu = 0; mu < 4; mu++) {
            if (c->group == 3) {
                g3_f a = load3_notwist_f(c, tf, g, mu);
                g3_d b;
                b.uv1.x = a.uv1.x; b.uv1.y = a.uv1.y; b.uv1.z = a.uv1.z; b.uv1.w = a.uv1.w;
                b.uv2.x = a.uv2.x; b.uv2.y = a.uv2.y; b.uv2.z = a.uv2.z; b.uv2.w = a.uv2.w;
                b.uv3.x = a.uv3.x; b.uv3.y = a.uv3.y; b.uv3.z = a.uv3.z; b.uv3.w = a.uv3.w;
                b = gs3_d(b);
                a.uv1.x = (float)b.uv1.x; a.uv1.y = (float)b.uv1.y; a.uv1.z = (float)b.uv1.z; a.uv1.w = (float)b.uv1.w;
                a.uv2.x = (float)b.uv2.x; a.uv2.y = (float)b.uv2.y; a.uv2.z = (float)b.uv2.z; a.uv2.w = (float)b.uv2.w;
                a.uv3.x = (float)b.uv3.x; a.uv3.y = (float)b.uv3.y; a.uv3.z = (float)b.uv3.z; a.uv3.w = (float)b.uv3.w;
                store3_f(c, tf, g, mu, a);
            } else {
                r4_f m = ld4_f(tf, c->rowsize, g, mu);
                double x = m.x, y = m.y, z = m.z, w = m.w;
                double det = sqrt(x * x + y * y + z * z + w * w);
                m.x = (float)(x / det); m.y = (float)(y / det); m.z = (float)(z / det); m.w = (float)(w / det);
                st4_f(tf, c->rowsize, g, mu, m);
            }
        }
}

void ol_plaquette(const ol_cfg *c, const void *t, double out[2])
{
    DISPATCH(plaquette_f(c, (const float *)t, out, NULL), plaquette_d(c, (const double *)t, out, NULL));
}
void ol_plaquette_f32(const ol_cfg *c, const void *t, double out[2])
{
    DISPATCH(plaquette_lp_f(c, (const float *)t, out), plaquette_d(c, (const double *)t, out, NULL));
}
void ol_action(const ol_cfg *c, const void *t, double out[2])
{
    double p[2];
    DISPATCH(plaquette_f(c, (const float *)t, p, out), plaquette_d(c, (const double *)t, p, out));
}
void ol_polyakov(const ol_cfg *c, const void *t, double out[4])
{
    DISPATCH(polyakov_f(c, (const float *)t, out), polyakov_d(c, (const double *)t, out));
}
void ol_fmunu(const ol_cfg *c, const void *t, int field, int i1, int i2, double out[12])
{
    DISPATCH(fmunu_f(c, (const float *)t, field, i1, i2, out), fmunu_d(c, (const double *)t, field, i1, i2, out));
}
void ol_action_profile(const ol_cfg *c, const void *t, int axis, double *out)
{
    DISPATCH(action_profile_f(c, (const float *)t, axis, out), action_profile_d(c, (const double *)t, axis, out));
}
void ol_polyakov_profile(const ol_cfg *c, const void *t, int axis, double *out)
{
    DISPATCH(polyakov_profile_f(c, (const float *)t, axis, out), polyakov_profile_d(c, (const double *)t, axis, out));
}
double ol_wilson(const ol_cfg *c, const void *t, int R, int T)
{
    double r;
    DISPATCH(r = wilson_f(c, (const float *)t, R, T), r = wilson_d(c, (const double *)t, R, T));
    return r;
}
double ol_local_action_link(const ol_cfg *c, const void *t, int gid, int dir)
{
    double r;
    DISPATCH(r = local_action_f(c, (const float *)t, gid, dir), r = local_action_d(c, (const double *)t, gid, dir));
    return r;
}

/* ======================================================= learned proposal */
#include "qg_oracle_learned.h"
