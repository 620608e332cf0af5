/*
 * qg_oracle_impl.h -- precision-generic body of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see qg_oracle.h).  Included twice by qg_oracle.c,
 * once with REAL=float (SFX=_f, IS_F=1) and once with REAL=double (SFX=_d).
 * REAL plays the role of the reference's hgpu_float (SU(N)/kernel/complex.h:69-91);
 * where the reference's float kernels promote to double through a double
 * literal (cl_khr_fp64 is enabled, SU(N)/suncl/model.cl:40-44) this file
 * promotes explicitly with (double).
 *
 * Operation order: every multiply-add is an explicit fma() in a fixed order
 * (the file is compiled with -ffp-contract=off) and sin/cos/log on the
 * update path are the routines ol_sincosf (float links) / ol_sincos (double
 * links) and ol_log of qg_oracle.c, so the roundings this restatement
 * performs are fully specified by the source.
 */

#define R4  PASTE(r4,  SFX)
#define CX  PASTE(cx,  SFX)
#define G3  PASTE(g3,  SFX)
#define M3  PASTE(m3,  SFX)
#define G2  PASTE(g2,  SFX)
#define S2  PASTE(s2,  SFX)
#define FN(n) PASTE(n, SFX)

#if IS_F
#define RPI   3.141592653589793f
#define RPI2  6.283185307179586f
#define RSQRT sqrtf
#define RFMA  fmaf
static float FN(rsin)(float a) { float s, c; ol_sincosf(a, &s, &c); return s; }
static float FN(rcos)(float a) { float s, c; ol_sincosf(a, &s, &c); return c; }
#else
#define RPI   3.1415926535897932384626433832795
#define RPI2  6.2831853071795864769252867665590
#define RSQRT sqrt
#define RFMA  fma
static double FN(rsin)(double a) { double s, c; ol_sincos(a, &s, &c); return s; }
static double FN(rcos)(double a) { double s, c; ol_sincos(a, &s, &c); return c; }
#endif
#define RSIN FN(rsin)
#define RCOS FN(rcos)

typedef struct { REAL x, y, z, w; } R4;
typedef struct { REAL re, im; } CX;
typedef struct { R4 uv1, uv2, uv3; } G3;              /* 12-real compressed SU(3) */
typedef struct { CX m[3][3]; } M3;                    /* full 3x3, row major      */
typedef struct { R4 uv1; } G2;                        /* 4-real SU(2)             */
typedef struct { CX u1, u2, v1, v2; } S2;             /* 2x2 block (u1 u2; v1 v2) */

/* ------------------------------------------------------------------ memory */
/* lattice_table_3 / lattice_store_3: SU(N)/suncl/su3_matrix_memory.cl:43-176 */
static R4 FN(ld4)(const REAL *tab, int rowsize, unsigned site, int plane)
{
    const REAL *p = tab + ((size_t)site + (size_t)plane * rowsize) * 4;
    R4 r = { p[0], p[1], p[2], p[3] };
    return r;
}
static void FN(st4)(REAL *tab, int rowsize, unsigned site, int plane, R4 v)
{
    REAL *p = tab + ((size_t)site + (size_t)plane * rowsize) * 4;
    p[0] = v.x; p[1] = v.y; p[2] = v.z; p[3] = v.w;
}

/* twisted boundary: Y links at x = N1-1 (su3_matrix_memory.cl:57-97):
 * row 1 times exp(i(phi+omega)/2), row 2 times exp(i(omega-phi)/2) */
static G3 FN(twist3)(const ol_cfg *c, G3 m)
{
    REAL phi = (REAL)c->phi, omega = (REAL)c->omega;
    REAL p = (phi + omega) / 2, q = (omega - phi) / 2;
    REAL cp = RCOS(p), sp = RSIN(p), cq = RCOS(q), sq = RSIN(q);
    R4 a = m.uv1, b = m.uv2, d = m.uv3;
    G3 r;
    r.uv1.x = RFMA(-b.x, sp, a.x * cp); r.uv1.y = RFMA(-b.y, sp, a.y * cp);
    r.uv1.z = RFMA(-b.z, sp, a.z * cp); r.uv1.w = RFMA(-b.w, sq, a.w * cq);
    r.uv2.x = RFMA(a.x, sp, b.x * cp);  r.uv2.y = RFMA(a.y, sp, b.y * cp);
    r.uv2.z = RFMA(a.z, sp, b.z * cp);  r.uv2.w = RFMA(a.w, sq, b.w * cq);
    r.uv3.x = RFMA(-d.z, sq, d.x * cq); r.uv3.y = RFMA(-d.w, sq, d.y * cq);
    r.uv3.z = RFMA(d.x, sq, d.z * cq);  r.uv3.w = RFMA(d.y, sq, d.w * cq);
    return r;
}

static G3 FN(load3)(const ol_cfg *c, const REAL *tab, const crd *co, unsigned site, int dir)
{
    G3 m;
    m.uv1 = FN(ld4)(tab, c->rowsize, site, dir);
    m.uv2 = FN(ld4)(tab, c->rowsize, site, dir + 4);
    m.uv3 = FN(ld4)(tab, c->rowsize, site, dir + 8);
    if (dir == 1 && has_twist(c) && co->x == c->n[0] - 1) m = FN(twist3)(c, m);
    return m;
}
static G3 FN(load3_notwist)(const ol_cfg *c, const REAL *tab, unsigned site, int dir)
{
    G3 m;
    m.uv1 = FN(ld4)(tab, c->rowsize, site, dir);
    m.uv2 = FN(ld4)(tab, c->rowsize, site, dir + 4);
    m.uv3 = FN(ld4)(tab, c->rowsize, site, dir + 8);
    return m;
}
static void FN(store3)(const ol_cfg *c, REAL *tab, unsigned site, int dir, G3 m)
{
    FN(st4)(tab, c->rowsize, site, dir, m.uv1);
    FN(st4)(tab, c->rowsize, site, dir + 4, m.uv2);
    FN(st4)(tab, c->rowsize, site, dir + 8, m.uv3);
}

/* SU(2): su2_matrix_memory.cl:56-143 */
static R4 FN(times2)(R4 u, R4 v);
static G2 FN(load2)(const ol_cfg *c, const REAL *tab, const crd *co, unsigned site, int dir)
{
    G2 m;
    m.uv1 = FN(ld4)(tab, c->rowsize, site, dir);
    if (dir == 1 && has_twist(c) && co->x == c->n[0] - 1) {
        REAL phi = (REAL)c->phi;
        R4 om;
        om.x = RCOS(phi / 2); om.y = 0; om.z = RSIN(phi / 2); om.w = 0;
        m.uv1 = FN(times2)(om, m.uv1);
    }
    return m;
}
static void FN(store2)(const ol_cfg *c, REAL *tab, unsigned site, int dir, G2 m)
{
    FN(st4)(tab, c->rowsize, site, dir, m.uv1);
}

/* --------------------------------------------------------------- algebra */
/* sum_k a_k b_k (k = 0,1,2 in order), with a, b strided */
static CX FN(dot3)(const CX *a, int as, const CX *b, int bs)
{
    CX r;
    r.re = a[0].re * b[0].re;
    r.re = RFMA(-a[0].im, b[0].im, r.re);
    r.im = a[0].re * b[0].im;
    r.im = RFMA(a[0].im, b[0].re, r.im);
    for (int k = 1; k < 3; k++) {
        CX x = a[k * as], y = b[k * bs];
        r.re = RFMA(x.re, y.re, r.re);
        r.re = RFMA(-x.im, y.im, r.re);
        r.im = RFMA(x.re, y.im, r.im);
        r.im = RFMA(x.im, y.re, r.im);
    }
    return r;
}
/* sum_k a_k conj(b_k) */
static CX FN(dotc3)(const CX *a, int as, const CX *b, int bs)
{
    CX r;
    r.re = a[0].re * b[0].re;
    r.re = RFMA(a[0].im, b[0].im, r.re);
    r.im = a[0].im * b[0].re;
    r.im = RFMA(-a[0].re, b[0].im, r.im);
    for (int k = 1; k < 3; k++) {
        CX x = a[k * as], y = b[k * bs];
        r.re = RFMA(x.re, y.re, r.re);
        r.re = RFMA(x.im, y.im, r.re);
        r.im = RFMA(x.im, y.re, r.im);
        r.im = RFMA(-x.re, y.im, r.im);
    }
    return r;
}
/* sum_k conj(a_k) b_k */
static CX FN(cdot3)(const CX *a, int as, const CX *b, int bs)
{
    CX r;
    r.re = a[0].re * b[0].re;
    r.re = RFMA(a[0].im, b[0].im, r.re);
    r.im = a[0].re * b[0].im;
    r.im = RFMA(-a[0].im, b[0].re, r.im);
    for (int k = 1; k < 3; k++) {
        CX x = a[k * as], y = b[k * bs];
        r.re = RFMA(x.re, y.re, r.re);
        r.re = RFMA(x.im, y.im, r.re);
        r.im = RFMA(x.re, y.im, r.im);
        r.im = RFMA(-x.im, y.re, r.im);
    }
    return r;
}

/* row 3 = conj(row1 x row2): lattice_reconstruct3, SU(N)/suncl/su3cl.cl:137-165 */
static void FN(fill_row3)(M3 *a)
{
    for (int j = 0; j < 3; j++) {
        int p = (j + 1) % 3, q = (j + 2) % 3;
        CX u1 = a->m[0][p], u2 = a->m[0][q], v1 = a->m[1][p], v2 = a->m[1][q];
        REAL re = u1.re * v2.re;
        re = RFMA(-u1.im, v2.im, re);
        re = RFMA(-u2.re, v1.re, re);
        re = RFMA(u2.im, v1.im, re);
        REAL im = u2.re * v1.im;
        im = RFMA(u2.im, v1.re, im);
        im = RFMA(-u1.re, v2.im, im);
        im = RFMA(-u1.im, v2.re, im);
        a->m[2][j].re = re;
        a->m[2][j].im = im;
    }
}
static M3 FN(expand)(G3 g)
{
    M3 a;
    a.m[0][0].re = g.uv1.x; a.m[0][0].im = g.uv2.x;
    a.m[0][1].re = g.uv1.y; a.m[0][1].im = g.uv2.y;
    a.m[0][2].re = g.uv1.z; a.m[0][2].im = g.uv2.z;
    a.m[1][0].re = g.uv3.x; a.m[1][0].im = g.uv3.z;
    a.m[1][1].re = g.uv3.y; a.m[1][1].im = g.uv3.w;
    a.m[1][2].re = g.uv1.w; a.m[1][2].im = g.uv2.w;
    FN(fill_row3)(&a);
    return a;
}
static G3 FN(compress)(const M3 *a)
{
    G3 g;
    g.uv1.x = a->m[0][0].re; g.uv1.y = a->m[0][1].re; g.uv1.z = a->m[0][2].re; g.uv1.w = a->m[1][2].re;
    g.uv2.x = a->m[0][0].im; g.uv2.y = a->m[0][1].im; g.uv2.z = a->m[0][2].im; g.uv2.w = a->m[1][2].im;
    g.uv3.x = a->m[1][0].re; g.uv3.y = a->m[1][1].re; g.uv3.z = a->m[1][0].im; g.uv3.w = a->m[1][1].im;
    return g;
}
/* full product (matrix_times_su3, su3cl.cl:101-135) */
static M3 FN(mul3)(const M3 *u, const M3 *v)
{
    M3 t;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) t.m[i][j] = FN(dot3)(&u->m[i][0], 1, &v->m[0][j], 3);
    return t;
}

/* staple term U_a U_b^+ U_c^+ (lattice_staple_hermitian3, su3_update_cl.cl:294-307):
 * rows 1,2 of P = A B^+, rows 1,2 of T = P C^+, row 3 of T reconstructed */
static M3 FN(staple_fwd3)(G3 ga, G3 gb, G3 gc)
{
    M3 A = FN(expand)(ga), B = FN(expand)(gb), C = FN(expand)(gc), P, T;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 3; j++) P.m[i][j] = FN(dotc3)(&A.m[i][0], 1, &B.m[j][0], 1);
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 3; j++) T.m[i][j] = FN(dotc3)(&P.m[i][0], 1, &C.m[j][0], 1);
    FN(fill_row3)(&T);
    return T;
}
/* staple term U_a^+ U_b^+ U_c (lattice_staple_hermitian_backward3,
 * su3_update_cl.cl:324-338) as the adjoint of H = C^+ R, R = B A: rows 1,2
 * of R, row 3 of R reconstructed, rows 1,2 of H, row 3 of H reconstructed */
static M3 FN(staple_bwd3)(G3 ga, G3 gb, G3 gc)
{
    M3 A = FN(expand)(ga), B = FN(expand)(gb), C = FN(expand)(gc), R, H, T;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 3; j++) R.m[i][j] = FN(dot3)(&B.m[i][0], 1, &A.m[0][j], 3);
    FN(fill_row3)(&R);
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 3; j++) H.m[i][j] = FN(cdot3)(&C.m[0][i], 3, &R.m[0][j], 3);
    FN(fill_row3)(&H);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            T.m[i][j].re = H.m[j][i].re;
            T.m[i][j].im = -H.m[j][i].im;
        }
    return T;
}
static M3 FN(add3)(const M3 *a, const M3 *b)
{
    M3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            r.m[i][j].re = a->m[i][j].re + b->m[i][j].re;
            r.m[i][j].im = a->m[i][j].im + b->m[i][j].im;
        }
    return r;
}

/* lattice_GramSchmidt3, su3_update_cl.cl:228-291 (in REAL precision) */
static G3 FN(gs3)(G3 g)
{
    REAL u[3][2] = { { g.uv1.x, g.uv2.x }, { g.uv1.y, g.uv2.y }, { g.uv1.z, g.uv2.z } };
    REAL v[3][2] = { { g.uv3.x, g.uv3.z }, { g.uv3.y, g.uv3.w }, { g.uv1.w, g.uv2.w } };
    REAL n2 = u[0][0] * u[0][0];
    n2 = RFMA(u[0][1], u[0][1], n2);
    for (int k = 1; k < 3; k++) { n2 = RFMA(u[k][0], u[k][0], n2); n2 = RFMA(u[k][1], u[k][1], n2); }
    REAL inu = (REAL)1 / RSQRT(n2);
    for (int k = 0; k < 3; k++) { u[k][0] = u[k][0] * inu; u[k][1] = u[k][1] * inu; }
    REAL sr = v[0][0] * u[0][0], si = v[0][1] * u[0][0];
    sr = RFMA(v[0][1], u[0][1], sr);
    si = RFMA(-v[0][0], u[0][1], si);
    for (int k = 1; k < 3; k++) {
        sr = RFMA(v[k][0], u[k][0], sr); sr = RFMA(v[k][1], u[k][1], sr);
        si = RFMA(v[k][1], u[k][0], si); si = RFMA(-v[k][0], u[k][1], si);
    }
    for (int k = 0; k < 3; k++) {
        REAL r = RFMA(-sr, u[k][0], v[k][0]);
        r = RFMA(si, u[k][1], r);
        REAL i = RFMA(-sr, u[k][1], v[k][1]);
        i = RFMA(-si, u[k][0], i);
        v[k][0] = r; v[k][1] = i;
    }
    REAL m2 = v[0][0] * v[0][0];
    m2 = RFMA(v[0][1], v[0][1], m2);
    for (int k = 1; k < 3; k++) { m2 = RFMA(v[k][0], v[k][0], m2); m2 = RFMA(v[k][1], v[k][1], m2); }
    REAL inv = (REAL)1 / RSQRT(m2);
    for (int k = 0; k < 3; k++) { v[k][0] = v[k][0] * inv; v[k][1] = v[k][1] * inv; }
    G3 r;
    r.uv1.x = u[0][0]; r.uv1.y = u[1][0]; r.uv1.z = u[2][0]; r.uv1.w = v[2][0];
    r.uv2.x = u[0][1]; r.uv2.y = u[1][1]; r.uv2.z = u[2][1]; r.uv2.w = v[2][1];
    r.uv3.x = v[0][0]; r.uv3.y = v[1][0]; r.uv3.z = v[0][1]; r.uv3.w = v[1][1];
    return r;
}

/* SU(2) algebra, gpu_su_2 layout (x=Re u11, y=Re u12, z=Im u11, w=Im u12):
 * matrix_times2, su2_matrix_memory.cl:41-53 / su3_update_cl.cl:150-162 */
static R4 FN(times2)(R4 u, R4 v)
{
    R4 a;
    a.x = u.x * v.x; a.x = RFMA(-u.y, v.y, a.x); a.x = RFMA(-u.z, v.z, a.x); a.x = RFMA(-u.w, v.w, a.x);
    a.z = u.x * v.z; a.z = RFMA(u.z, v.x, a.z); a.z = RFMA(u.y, v.w, a.z); a.z = RFMA(-u.w, v.y, a.z);
    a.y = u.x * v.y; a.y = RFMA(u.y, v.x, a.y); a.y = RFMA(u.w, v.z, a.y); a.y = RFMA(-u.z, v.w, a.y);
    a.w = u.x * v.w; a.w = RFMA(u.w, v.x, a.w); a.w = RFMA(u.z, v.y, a.w); a.w = RFMA(-u.y, v.z, a.w);
    return a;
}
static R4 FN(herm2)(R4 u) { R4 r = { u.x, -u.y, -u.z, -u.w }; return r; }
static S2 FN(rec2)(R4 a)
{
    S2 b;
    b.u1.re = a.x;  b.u1.im = a.z;  b.u2.re = a.y;  b.u2.im = a.w;
    b.v1.re = -a.y; b.v1.im = a.w;  b.v2.re = a.x;  b.v2.im = -a.z;
    return b;
}
/* full 2x2 complex product: matrix_times_su2, su2cl.cl:43-60 */
static S2 FN(mul2)(const S2 *u, const S2 *v)
{
    CX U[2][2] = { { u->u1, u->u2 }, { u->v1, u->v2 } }, W[2][2] = { { v->u1, v->u2 }, { v->v1, v->v2 } }, T[2][2];
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            REAL re = U[i][0].re * W[0][j].re;
            re = RFMA(-U[i][0].im, W[0][j].im, re);
            re = RFMA(U[i][1].re, W[1][j].re, re);
            re = RFMA(-U[i][1].im, W[1][j].im, re);
            REAL im = U[i][0].re * W[0][j].im;
            im = RFMA(U[i][0].im, W[0][j].re, im);
            im = RFMA(U[i][1].re, W[1][j].im, im);
            im = RFMA(U[i][1].im, W[1][j].re, im);
            T[i][j].re = re; T[i][j].im = im;
        }
    S2 t;
    t.u1 = T[0][0]; t.u2 = T[0][1]; t.v1 = T[1][0]; t.v2 = T[1][1];
    return t;
}
static S2 FN(add2)(S2 a, S2 b)
{
    S2 r;
    r.u1.re = a.u1.re + b.u1.re; r.u1.im = a.u1.im + b.u1.im;
    r.u2.re = a.u2.re + b.u2.re; r.u2.im = a.u2.im + b.u2.im;
    r.v1.re = a.v1.re + b.v1.re; r.v1.im = a.v1.im + b.v1.im;
    r.v2.re = a.v2.re + b.v2.re; r.v2.im = a.v2.im + b.v2.im;
    return r;
}
/* staple pieces for SU(2): su2_update_cl.cl:158-203 */
static S2 FN(staple_fwd2)(R4 u1, R4 u2, R4 u3)
{
    return FN(rec2)(FN(times2)(FN(times2)(u1, FN(herm2)(u2)), FN(herm2)(u3)));
}
static S2 FN(staple_bwd2)(R4 u1, R4 u2, R4 u3)
{
    return FN(rec2)(FN(times2)(FN(times2)(FN(herm2)(u1), FN(herm2)(u2)), u3));
}

/* ------------------------------------------------------------- PRN source */
typedef struct {
    const ol_prn *src;
    const ol_cfg *cfg;
    uint32_t thread;      /* GID of the phase kernel thread            */
    uint32_t k;           /* PRN quads consumed so far (indprng step)  */
    double gidval;        /* INTS=2: float(gindex)                     */
} FN(prnctx);

static void FN(prn_next)(FN(prnctx) *p, REAL r[4])
{
    float q[4];
    if (p->src->mode == 2) {
        for (int i = 0; i < 4; i++) r[i] = (REAL)ol_ranlux_next(p->src->stream);
        p->k++;
        return;
    }
    if (p->src->mode == 0) {
        size_t idx = (size_t)p->thread + (size_t)p->k * (size_t)p->cfg->prngstep;
        const float *s = p->src->prns + idx * 4;
        q[0] = s[0]; q[1] = s[1]; q[2] = s[2]; q[3] = s[3];
    } else {
        ol_philox_prn(p->src, p->thread, p->k, q);
    }
    p->k++;
    r[0] = (REAL)q[0]; r[1] = (REAL)q[1]; r[2] = (REAL)q[2]; r[3] = (REAL)q[3];
}

/* --------------------------------------------------------------- heatbath */
/* Kennedy-Pendleton step on the SU(2) block a.  Returns 1 when a try was
 * accepted and a is overwritten with c*aH; on rejection the SU(3) caller
 * wants the identity and one extra PRN skip (su3_update_cl.cl:665-668).
 * su3_update_cl.cl:568-669 (SU(3) path) / su2_update_cl.cl:434-531 (SU(2)). */
static int FN(kp_step)(S2 *a, REAL beta, FN(prnctx) *p, int su3_path)
{
    const ol_cfg *c = p->cfg;
    R4 aH, cc, d;
    REAL det, bdet, cosrnd, delta = 0, rnd[4], n2;
    int flag = 0;
    if (su3_path) {
        aH.x =  (a->u1.re + a->v2.re);
        aH.z = -(a->u1.im - a->v2.im);
        aH.y = -(a->u2.re - a->v1.re);
        aH.w = -(a->u2.im + a->v1.im);
        n2 = aH.x * aH.x;
        n2 = RFMA(aH.y, aH.y, n2); n2 = RFMA(aH.z, aH.z, n2); n2 = RFMA(aH.w, aH.w, n2);
        det = RSQRT(n2);
        REAL id = (REAL)1 / det;
        aH.x *= id; aH.z *= id; aH.y *= id; aH.w *= id;
    } else {
        REAL Mx = a->u1.re + a->v2.re, My = a->u1.im - a->v2.im;
        REAL Mz = a->u2.re - a->v1.re, Mw = a->u2.im + a->v1.im;
        n2 = Mx * Mx;
        n2 = RFMA(My, My, n2); n2 = RFMA(Mz, Mz, n2); n2 = RFMA(Mw, Mw, n2);
        det = RSQRT(n2);
        REAL id = (REAL)1 / det;
        aH.x = Mx * id; aH.z = -My * id; aH.y = -Mz * id; aH.w = -Mw * id;
    }
    bdet = beta * det;
    for (int i = 0; i < c->nhit && !flag; i++) {
        if (c->gid_mode) {
            double g = p->gidval, V = (double)sites_of(c);
            double a5 = 0.005 * (1 + c->nhit);
            rnd[0] = (REAL)fabs(sin((a5 + 270.0 / V) * g));
            rnd[1] = (REAL)fabs(cos((a5 +  60.0 / V) * g));
            rnd[2] = (REAL)fabs(sin((a5 - 150.0 / V) * g));
            rnd[3] = (REAL)fabs(cos((a5 - 380.0 / V) * g));
        } else {
            FN(prn_next)(p, rnd);
        }
        if (ol_ref_arith) {
            /* the reference's expression as written (su3_update_cl.cl:619-620):
             * product and sum rounded separately, the C library's cos and log
             * standing in for the OpenCL runtime's (test-only comparison) */
#if IS_F
            cosrnd = cosf(RPI2 * rnd[1]);
#else
            cosrnd = cos(RPI2 * rnd[1]);
#endif
            double lx = log(1.0 - (double)rnd[0]), lz = log(1.0 - (double)rnd[2]);
            delta = (REAL)(-(lx + (double)(cosrnd * cosrnd) * lz) / (double)bdet);
        } else {
            cosrnd = RCOS(RPI2 * rnd[1]);
            double lx = ol_log(1.0 - (double)rnd[0]), lz = ol_log(1.0 - (double)rnd[2]);
            delta = (REAL)(-fma((double)(cosrnd * cosrnd), lz, lx) / (double)bdet);
        }
        if ((double)(rnd[3] * rnd[3]) <= fma(-0.5, (double)delta, 1.0)) flag = 1;
        if (c->gid_mode) { delta = cosrnd * cosrnd / bdet; flag = 1; }
    }
    if (flag) {
        if (c->gid_mode) {
            double g = p->gidval, V = (double)sites_of(c);
            rnd[0] = (REAL)fabs(cos((0.08 - 270.0 / V) * g));
            rnd[1] = (REAL)fabs(sin((0.08 -  60.0 / V) * g));
            rnd[2] = (REAL)fabs(cos((0.08 + 150.0 / V) * g));
            rnd[3] = (REAL)fabs(sin((0.08 + 380.0 / V) * g));
        } else if (p->src->mode == 2) {
            rnd[0] = (REAL)ol_ranlux_next(p->src->stream);   /* update_su2.cpp:101: 2 numbers */
            rnd[1] = (REAL)ol_ranlux_next(p->src->stream);
        } else {
            FN(prn_next)(p, rnd);
        }
        REAL cosal = (REAL)(1.0 - (double)delta);
        REAL costh = (REAL)fma(2.0, (double)rnd[0], -1.0);
        REAL sinth = (REAL)sqrt(1.0 - (double)(costh * costh));
        REAL sinal = (REAL)sqrt(1.0 - (double)(cosal * cosal));
        REAL phi = RPI2 * rnd[1];
        REAL sinphi = RSIN(phi), cosphi = RCOS(phi);
        if (ol_ref_arith) {
#if IS_F
            sinphi = sinf(phi); cosphi = cosf(phi);
#else
            sinphi = sin(phi); cosphi = cos(phi);
#endif
        }
        cc.x = cosal;
        cc.z = sinal * costh;
        cc.y = sinal * sinth * sinphi;
        cc.w = sinal * sinth * cosphi;
        d = FN(times2)(cc, aH);
        *a = FN(rec2)(d);
        return 1;
    }
    if (su3_path) {
        a->u1.re = 1; a->u1.im = 0; a->u2.re = 0; a->u2.im = 0;
        a->v1.re = 0; a->v1.im = 0; a->v2.re = 1; a->v2.im = 0;
        if (!c->gid_mode && p->src->mode != 2) p->k++;
    }
    return 0;
}

/* Microcanonical reflection of the SU(2) block (overrelaxation; absent in
 * the reference, Creutz PRD 36 (1987) 515, Brown-Woch PRL 58 (1987) 2394):
 * with aH = h/|h| the normalised hermitian projection used by the heatbath,
 * the subgroup element aH*aH leaves Re Tr(V W) unchanged and is an
 * involution.  Written in closed form: aH^2 = (x^2 - y^2 - z^2 - w^2,
 * 2xy, 2xz, 2xw) / |h|^2 (one reciprocal, no square root). */
static void FN(or_step)(S2 *a)
{
    REAL hx =  (a->u1.re + a->v2.re);
    REAL hz = -(a->u1.im - a->v2.im);
    REAL hy = -(a->u2.re - a->v1.re);
    REAL hw = -(a->u2.im + a->v1.im);
    REAL n2 = hx * hx;
    n2 = RFMA(hy, hy, n2); n2 = RFMA(hz, hz, n2); n2 = RFMA(hw, hw, n2);
    REAL v0 = hx * hx;
    v0 = RFMA(-hy, hy, v0); v0 = RFMA(-hz, hz, v0); v0 = RFMA(-hw, hw, v0);
    REAL inv = (REAL)1 / n2;
    REAL t = (hx + hx) * inv;
    R4 v;
    v.x = v0 * inv; v.y = hy * t; v.z = hz * t; v.w = hw * t;
    *a = FN(rec2)(v);
}

/* rows i, j of U <- V (rows i, j), V = (u1 u2; v1 v2) */
static void FN(rotate_rows)(M3 *U, int i, int j, const S2 *V)
{
    for (int k = 0; k < 3; k++) {
        CX x = U->m[i][k], y = U->m[j][k];
        REAL re = V->u1.re * x.re; re = RFMA(-V->u1.im, x.im, re); re = RFMA(V->u2.re, y.re, re); re = RFMA(-V->u2.im, y.im, re);
        REAL im = V->u1.re * x.im; im = RFMA(V->u1.im, x.re, im); im = RFMA(V->u2.re, y.im, im); im = RFMA(V->u2.im, y.re, im);
        REAL re2 = V->v1.re * x.re; re2 = RFMA(-V->v1.im, x.im, re2); re2 = RFMA(V->v2.re, y.re, re2); re2 = RFMA(-V->v2.im, y.im, re2);
        REAL im2 = V->v1.re * x.im; im2 = RFMA(V->v1.im, x.re, im2); im2 = RFMA(V->v2.re, y.im, im2); im2 = RFMA(V->v2.im, y.re, im2);
        U->m[i][k].re = re;  U->m[i][k].im = im;
        U->m[j][k].re = re2; U->m[j][k].im = im2;
    }
}

/* Cabibbo-Marinari over the SU(2) subgroups (1,2), (1,3), (2,3); restates
 * lattice_heatbath3, su3_update_cl.cl:672-779: for each subgroup the block
 * of W = U*staple (matrix_times_su3), the Kennedy-Pendleton draw and the
 * subgroup rotation V*U of the two rows; then Gram-Schmidt.
 * kind 0 = heatbath, 1 = overrelaxation. */
static G3 FN(cm3)(const M3 *S, G3 m0, REAL beta, FN(prnctx) *p, int nhitpar, int kind)
{
    G3 reslt = m0;
    M3 U = FN(expand)(m0);
    for (int n = 0; n < nhitpar; n++) {
        for (int sg = 0; sg < 3; sg++) {
            int i = (sg == 2) ? 1 : 0, j = (sg == 0) ? 1 : 2;
            S2 r0;
            r0.u1 = FN(dot3)(&U.m[i][0], 1, &S->m[0][i], 3);
            r0.u2 = FN(dot3)(&U.m[i][0], 1, &S->m[0][j], 3);
            r0.v1 = FN(dot3)(&U.m[j][0], 1, &S->m[0][i], 3);
            r0.v2 = FN(dot3)(&U.m[j][0], 1, &S->m[0][j], 3);
            if (kind == 0) FN(kp_step)(&r0, beta, p, 1); else FN(or_step)(&r0);
            FN(rotate_rows)(&U, i, j, &r0);
        }
        /* Gram-Schmidt after a heatbath update; the reflections keep U
         * unitary to rounding and an overrelaxed link is stored as it is
         * (reunitarised by its next heatbath update and the global pass) */
        reslt = (kind == 0) ? FN(gs3)(FN(compress)(&U)) : FN(compress)(&U);
        U = FN(expand)(reslt);
    }
    return reslt;
}

/* --------------------------------------------------------------- staples */
/* lattice_staple_3, su3_update_cl.cl:341-565: for direction mu the three
 * other directions are visited in the reference's fixed order and summed
 * pairwise as written there (forward+backward per plane, running sum). */
static const int FN(nu_order)[4][3] = { {1, 2, 3}, {0, 2, 3}, {1, 0, 3}, {1, 2, 0} };

static M3 FN(staple3)(const ol_cfg *c, const REAL *tab, unsigned g, int mu)
{
    crd co, cp, cn, cm, cmp;
    gid2c(c, g, &co);
    cp = nb_plus(c, co, mu);
    M3 st, s2;
    for (int i = 0; i < 3; i++) {
        int nu = FN(nu_order)[mu][i];
        cn = nb_plus(c, co, nu);
        cm = nb_minus(c, co, nu);
        cmp = nb_plus(c, cm, mu);
        G3 a = FN(load3)(c, tab, &cp, c2gid(c, cp), nu);
        G3 b = FN(load3)(c, tab, &cn, c2gid(c, cn), mu);
        G3 d = FN(load3)(c, tab, &co, g, nu);
        M3 fw = FN(staple_fwd3)(a, b, d);
        a = FN(load3)(c, tab, &cmp, c2gid(c, cmp), nu);
        b = FN(load3)(c, tab, &cm, c2gid(c, cm), mu);
        d = FN(load3)(c, tab, &cm, c2gid(c, cm), nu);
        M3 bw = FN(staple_bwd3)(a, b, d);
        if (i == 0) {
            st = FN(add3)(&fw, &bw);                   /* staple  = f0 + b0    */
        } else {
            s2 = FN(add3)(&st, &fw);                   /* staple2 = st + f_i   */
            st = FN(add3)(&bw, &s2);                   /* staple  = b_i + s2   */
        }
    }
    return st;
}

static S2 FN(staple2)(const ol_cfg *c, const REAL *tab, unsigned g, int mu)
{
    crd co, cp, cn, cm, cmp;
    gid2c(c, g, &co);
    cp = nb_plus(c, co, mu);
    S2 st, s2;
    for (int i = 0; i < 3; i++) {
        int nu = FN(nu_order)[mu][i];
        cn = nb_plus(c, co, nu);
        cm = nb_minus(c, co, nu);
        cmp = nb_plus(c, cm, mu);
        R4 a = FN(load2)(c, tab, &cp, c2gid(c, cp), nu).uv1;
        R4 b = FN(load2)(c, tab, &cn, c2gid(c, cn), mu).uv1;
        R4 d = FN(load2)(c, tab, &co, g, nu).uv1;
        S2 fw = FN(staple_fwd2)(a, b, d);
        a = FN(load2)(c, tab, &cmp, c2gid(c, cmp), nu).uv1;
        b = FN(load2)(c, tab, &cm, c2gid(c, cm), mu).uv1;
        d = FN(load2)(c, tab, &cm, c2gid(c, cm), nu).uv1;
        S2 bw = FN(staple_bwd2)(a, b, d);
        if (i == 0) {
            st = FN(add2)(fw, bw);
        } else {
            s2 = FN(add2)(st, fw);
            st = FN(add2)(bw, s2);
        }
    }
    return st;
}

/* ----------------------------------------------------------- phase kernel */
/* update_{even,odd}_{X,Y,Z,T}, SU(N)/suncl/suncl.cl:399-975 */
static void FN(phase_link)(const ol_cfg *c, REAL *tab, int parity, int mu, const ol_prn *src, int kind,
                          REAL beta, unsigned t)
{
    {
        unsigned g = parity ? odd_gid(c, t) : even_gid(c, t);
        crd co;
        gid2c(c, g, &co);
        FN(prnctx) p;
        p.src = src; p.cfg = c; p.thread = t; p.k = 0; p.gidval = (double)(float)g;
        if (c->group == 3) {
            G3 m0 = FN(load3)(c, tab, &co, g, mu);
            M3 st = FN(staple3)(c, tab, g, mu);
            G3 mU = FN(cm3)(&st, m0, beta, &p, c->nhitpar, kind);
            FN(store3)(c, tab, g, mu, mU);
        } else {
            G2 m0 = FN(load2)(c, tab, &co, g, mu);
            S2 st = FN(staple2)(c, tab, g, mu);
            if (kind == 0) {
                S2 a = st;
                if (FN(kp_step)(&a, beta, &p, 0)) {
                    G2 r; r.uv1.x = a.u1.re; r.uv1.y = a.u2.re; r.uv1.z = a.u1.im; r.uv1.w = a.u2.im;
                    FN(store2)(c, tab, g, mu, r);
                } else {
                    FN(store2)(c, tab, g, mu, m0);
                }
            } else {
                /* U -> aH U^+ aH with aH = normalised (staple projection)^+ */
                R4 aH;
                REAL Mx = st.u1.re + st.v2.re, My = st.u1.im - st.v2.im;
                REAL Mz = st.u2.re - st.v1.re, Mw = st.u2.im + st.v1.im;
                REAL n2 = Mx * Mx;
                n2 = RFMA(My, My, n2); n2 = RFMA(Mz, Mz, n2); n2 = RFMA(Mw, Mw, n2);
                REAL id = (REAL)1 / RSQRT(n2);
                aH.x = Mx * id; aH.z = -My * id; aH.y = -Mz * id; aH.w = -Mw * id;
                G2 r;
                r.uv1 = FN(times2)(FN(times2)(aH, FN(herm2)(m0.uv1)), aH);
                FN(store2)(c, tab, g, mu, r);
            }
        }
    }
}

static void FN(phase)(const ol_cfg *c, REAL *tab, int parity, int mu, const ol_prn *src, int kind)
{
    unsigned half = (unsigned)(sites_of(c) / 2);
    REAL beta = (REAL)(c->beta / c->group);
    if (kind == 0 && src && src->mode == 2) {
        /* one stream consumed link after link: in thread order, serially */
        for (unsigned t = 0; t < half; t++) FN(phase_link)(c, tab, parity, mu, src, kind, beta, t);
        return;
    }
    /* the links of one (parity, direction) class are updated independently
     * of one another, so the loop runs in parallel with the same result */
#pragma omp parallel for schedule(static)
    for (unsigned t = 0; t < half; t++) FN(phase_link)(c, tab, parity, mu, src, kind, beta, t);
}

/* --------------------------------------------------------- initialisation */
static void FN(init_cold)(const ol_cfg *c, REAL *tab)
{
    int V = sites_of(c);
    for (int g = 0; g < V; g++)
        for (int mu = 0; mu < 4; mu++) {
            if (c->group == 3) {
                G3 m; R4 z = { 0, 0, 0, 0 };
                m.uv1 = z; m.uv2 = z; m.uv3 = z; m.uv1.x = 1; m.uv3.y = 1;
                FN(store3)(c, tab, g, mu, m);
            } else {
                G2 m; m.uv1.x = 1; m.uv1.y = 0; m.uv1.z = 0; m.uv1.w = 0;
                FN(store2)(c, tab, g, mu, m);
            }
        }
}

/* lattice_init_gid, suncl.cl:190-347 (sin/cos in double, GS in REAL) */
static void FN(init_gid)(const ol_cfg *c, REAL *tab)
{
    int V = sites_of(c);
    double s = (double)V;
    for (int g = 0; g < V; g++) {
        double gd = (double)g;
        for (int mu = 0; mu < 4; mu++) {
            static const double off[4] = { 0.001, 0.002, 0.003, 0.004 };
            double o = off[mu];
            if (c->group == 3) {
                double f1  = sin((o + 10.0 / s) * gd) / 2.0;
                double f2  = cos((o - 10.0 / s) * gd) / 3.0;
                double f3  = sin((o - 18.0 / s) * gd) / 4.0;
                double f4  = cos((o + 12.0 / s) * gd) / 4.0;
                double f5  = sin((o - 12.0 / s) * gd) / 3.0;
                double f6  = cos((o - 15.0 / s) * gd) / 2.0;
                double f7  = sin((o + 15.0 / s) * gd) / 3.0;
                double f8  = cos((o - 11.0 / s) * gd) / 4.0;
                double f9  = sin((o - 11.0 / s) * gd) / 3.0;
                double f10 = cos((o + 16.0 / s) * gd) / 2.0;
                double f11 = sin((o - 16.0 / s) * gd) / 3.0;
                double f12 = cos((o - 18.0 / s) * gd) / 2.0;
                G3 m;
                m.uv1.x = (REAL)f1; m.uv1.y = (REAL)f3; m.uv1.z = (REAL)f5; m.uv1.w = (REAL)f11;
                m.uv2.x = (REAL)f2; m.uv2.y = (REAL)f4; m.uv2.z = (REAL)f6; m.uv2.w = (REAL)f12;
                m.uv3.x = (REAL)f7; m.uv3.y = (REAL)f9; m.uv3.z = (REAL)f8; m.uv3.w = (REAL)f10;
                FN(store3)(c, tab, g, mu, FN(gs3)(m));
            } else {
                double f1 = sin((o + 10.0 / s) * gd) / 2.0;
                double f2 = cos((o - 10.0 / s) * gd) / 3.0;
                double f3 = sin((o - 18.0 / s) * gd) / 4.0;
                double f4 = sqrt(1.0 - f1 * f1 - f2 * f2 - f3 * f3);
                G2 m;
                m.uv1.x = (REAL)f1; m.uv1.y = (REAL)f3; m.uv1.z = (REAL)f4; m.uv1.w = (REAL)f2;
                FN(store2)(c, tab, g, mu, m);
            }
        }
    }
}

/* lattice_random3 / lattice_random2 (su3_update_cl.cl:165-225,
 * su2_update_cl.cl:110-146): NOT Haar; alpha uniform in [0,pi]. */
static R4 FN(rnd_r4)(const float *prns, size_t idx)
{
    R4 r = { (REAL)prns[idx * 4], (REAL)prns[idx * 4 + 1], (REAL)prns[idx * 4 + 2], (REAL)prns[idx * 4 + 3] };
    return r;
}
static void FN(init_hot_dir)(const ol_cfg *c, REAL *tab, int mu, const float *prns)
{
    int V = sites_of(c);
#pragma omp parallel for schedule(static)
    for (int g = 0; g < V; g++) {
        if (c->group == 3) {
            R4 r1 = FN(rnd_r4)(prns, (size_t)g);
            R4 r2 = FN(rnd_r4)(prns, (size_t)g + c->rowsize);
            R4 r3 = FN(rnd_r4)(prns, (size_t)g + 2 * (size_t)c->rowsize);
            REAL a0[4], a1[4], a2[4], a3[4];
            REAL R1[4] = { r1.x, r1.y, r1.z, r1.w }, R2[4] = { r2.x, r2.y, r2.z, r2.w }, R3[4] = { r3.x, r3.y, r3.z, r3.w };
            for (int k = 0; k < 4; k++) {
                REAL alpha = RPI * R1[k], phi = RPI2 * R2[k];
#if IS_F
                REAL costh = 2.0f * R3[k] - 1.0f;
                REAL sinth = sqrtf(1.0f - costh * costh);
#else
                REAL costh = 2.0 * R3[k] - 1.0;
                REAL sinth = sqrt(1.0 - costh * costh);
#endif
                REAL sinal = RSIN(alpha);
                a0[k] = RCOS(alpha);
                REAL sinph = RSIN(phi), cosph = RCOS(phi);
                REAL t1 = sinal * sinth;
                a1[k] = t1 * cosph;
                a2[k] = t1 * sinph;
                a3[k] = sinal * costh;
            }
            /* product of three embedded SU(2) rotations, written out as in
             * su3_update_cl.cl:209-220 (components .x,.y,.z of a0..a3) */
            G3 m;
#define X 0
#define Y 1
#define Z 2
            m.uv1.x = a0[X] * a0[Y] - a3[X] * a3[Y];
            m.uv2.x = a0[Y] * a3[X] + a0[X] * a3[Y];
            m.uv1.y = -a0[X] * a1[Y] * a1[Z] + a0[Z] * a2[X] - a0[X] * a2[Y] * a2[Z] - a1[Z] * a2[Y] * a3[X] + a1[Y] * a2[Z] * a3[X] - a1[X] * a3[Z];
            m.uv2.y = a0[Z] * a1[X] + a0[X] * a1[Z] * a2[Y] - a0[X] * a1[Y] * a2[Z] - a1[Y] * a1[Z] * a3[X] - a2[Y] * a2[Z] * a3[X] + a2[X] * a3[Z];
            m.uv1.z = -a1[X] * a1[Z] + a0[X] * a0[Z] * a2[Y] + a2[X] * a2[Z] - a0[Z] * a1[Y] * a3[X] + a0[X] * a1[Y] * a3[Z] + a2[Y] * a3[X] * a3[Z];
            m.uv2.z = a0[X] * a0[Z] * a1[Y] + a1[Z] * a2[X] + a1[X] * a2[Z] + a0[Z] * a2[Y] * a3[X] - a0[X] * a2[Y] * a3[Z] + a1[Y] * a3[X] * a3[Z];
            m.uv1.w = -a0[Z] * a1[X] * a1[Y] - a0[Z] * a2[X] * a2[Y] + a0[X] * a2[Z] + a1[Z] * a3[X] - a1[Y] * a2[X] * a3[Z] + a1[X] * a2[Y] * a3[Z];
            m.uv2.w = a0[X] * a1[Z] - a0[Z] * a1[Y] * a2[X] + a0[Z] * a1[X] * a2[Y] - a2[Z] * a3[X] + a1[X] * a1[Y] * a3[Z] + a2[X] * a2[Y] * a3[Z];
            m.uv3.x = -a0[Y] * a2[X] - a1[X] * a3[Y];
            m.uv3.z = a0[Y] * a1[X] - a2[X] * a3[Y];
            m.uv3.y = a0[X] * a0[Z] + a1[Y] * a1[Z] * a2[X] - a1[X] * a1[Z] * a2[Y] + a1[X] * a1[Y] * a2[Z] + a2[X] * a2[Y] * a2[Z] + a3[X] * a3[Z];
            m.uv3.w = -a1[X] * a1[Y] * a1[Z] - a1[Z] * a2[X] * a2[Y] + a1[Y] * a2[X] * a2[Z] - a1[X] * a2[Y] * a2[Z] - a0[Z] * a3[X] + a0[X] * a3[Z];
#undef X
#undef Y
#undef Z
            FN(store3)(c, tab, g, mu, m);
        } else {
            R4 r = FN(rnd_r4)(prns, (size_t)g);
            REAL alpha = RPI * r.x, phi = RPI2 * r.y;
#if IS_F
            REAL costh = 2.0f * r.z - 1.0f;
            REAL sinth = sqrtf(1.0f - costh * costh);
#else
            REAL costh = 2.0 * r.z - 1.0;
            REAL sinth = sqrt(1.0 - costh * costh);
#endif
            REAL sinal = RSIN(alpha), a0 = RCOS(alpha);
            REAL sinph = RSIN(phi), cosph = RCOS(phi);
            REAL t1 = sinal * sinth;
            G2 m;
            m.uv1.x = a0; m.uv1.y = t1 * sinph; m.uv1.z = sinal * costh; m.uv1.w = t1 * cosph;
            FN(store2)(c, tab, g, mu, m);
        }
    }
}

/* lattice_GramSchmidt kernel, suncl.cl:350-396 (REAL precision) */
static void FN(gramschmidt)(const ol_cfg *c, REAL *tab)
{
    int V = sites_of(c);
#pragma omp parallel for schedule(static)
    for (int g = 0; g < V; g++)
        for (int mu = 0; mu < 4; mu++) {
            if (c->group == 3) {
                FN(store3)(c, tab, g, mu, FN(gs3)(FN(load3_notwist)(c, tab, g, mu)));
            } else {
                R4 m = FN(ld4)(tab, c->rowsize, g, mu);
                REAL det = RSQRT(m.x * m.x + m.y * m.y + m.z * m.z + m.w * m.w);
                m.x /= det; m.y /= det; m.z /= det; m.w /= det;
                FN(st4)(tab, c->rowsize, g, mu, m);
            }
        }
}

/* ------------------------------------------------------------ measurement */
/* lattice_reconstruct3_double + FP64 products (su3_measurements_cl.cl:292-548) */
static void FN(to_d3)(G3 a, cd3 *b)
{
    g3_d ad;
    ad.uv1.x = (double)a.uv1.x; ad.uv1.y = (double)a.uv1.y; ad.uv1.z = (double)a.uv1.z; ad.uv1.w = (double)a.uv1.w;
    ad.uv2.x = (double)a.uv2.x; ad.uv2.y = (double)a.uv2.y; ad.uv2.z = (double)a.uv2.z; ad.uv2.w = (double)a.uv2.w;
    ad.uv3.x = (double)a.uv3.x; ad.uv3.y = (double)a.uv3.y; ad.uv3.z = (double)a.uv3.z; ad.uv3.w = (double)a.uv3.w;
    m3_d s = expand_d(ad);
    memcpy(b, &s, sizeof(s));
}
static void FN(to_d2)(R4 a, cd3 *b)
{
    /* SU(2) embedded in the 2x2 block of a 3x3 with zero third row/column */
    memset(b, 0, sizeof(*b));
    b->m[0][0].re = (double)a.x;  b->m[0][0].im = (double)a.z;
    b->m[0][1].re = (double)a.y;  b->m[0][1].im = (double)a.w;
    b->m[1][0].re = -(double)a.y; b->m[1][0].im = (double)a.w;
    b->m[1][1].re = (double)a.x;  b->m[1][1].im = -(double)a.z;
}
static void FN(load_d)(const ol_cfg *c, const REAL *tab, const crd *co, int mu, cd3 *out)
{
    unsigned g = c2gid(c, *co);
    if (c->group == 3) FN(to_d3)(FN(load3)(c, tab, co, g, mu), out);
    else FN(to_d2)(FN(load2)(c, tab, co, g, mu).uv1, out);
}

/* the plaquette matrix U_m(x) U_n(x+m) U_m(x+n)^+ U_n(x)^+ in FP64
 * (lattice_retrace_plaquette3 / _F, su3_measurements_cl.cl:527-586) */
static void FN(plaq_mat)(const ol_cfg *c, const REAL *tab, crd co, int m, int n, cd3 *w1)
{
    crd cm = nb_plus(c, co, m), cn = nb_plus(c, co, n);
    cd3 a, b, d, e, w2, w3;
    FN(load_d)(c, tab, &co, m, &a);
    FN(load_d)(c, tab, &cm, n, &b);
    FN(load_d)(c, tab, &cn, m, &d);
    FN(load_d)(c, tab, &co, n, &e);
    int N = c->group;
    cd_mul(&a, &b, w1, N);
    cd_herm(&d, &w2, N);
    cd_mul(w1, &w2, &w3, N);
    cd_herm(&e, &w2, N);
    cd_mul(&w3, &w2, w1, N);
}
/* Re Tr of the spatial (xy, xz, yz) and temporal (xt, yt, zt) plaquettes
 * of one site, summed in the reference order xy, xz, xt, yz, yt, zt
 * (sun_measurements_cl.cl:1240-1305) */
static void FN(plaq_site)(const ol_cfg *c, const REAL *tab, crd co, double *rs_out, double *rt_out)
{
    static const int pl[6][2] = { {0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3} };
    double rs = 0, rt = 0;
    for (int q = 0; q < 6; q++) {
        cd3 w;
        FN(plaq_mat)(c, tab, co, pl[q][0], pl[q][1], &w);
        double tr = cd_retr(&w, c->group);
        if (pl[q][1] == 3) rt += tr; else rs += tr;
    }
    *rs_out = rs; *rt_out = rt;
}

static void FN(plaquette)(const ol_cfg *c, const REAL *tab, double out[2], double *act_out)
{
    int V = sites_of(c);
    double sp = 0, tp = 0, as = 0, at = 0;
    REAL bet = (REAL)(c->beta / c->group);
    for (int g = 0; g < V; g++) {
        crd co; gid2c(c, g, &co);
        double rs, rt;
        FN(plaq_site)(c, tab, co, &rs, &rt);
        sp += rs; tp += rt;
        as += (double)bet * (3.0 * c->group - rs);
        at += (double)bet * (3.0 * c->group - rt);
    }
    out[0] = sp; out[1] = tp;
    if (act_out) { act_out[0] = as; act_out[1] = at; }
}

/* The plaquette with the products of each plaquette and its trace in the
 * link precision (the FP32-product plaquette of FP32-link lattices; the
 * reference promotes to FP64, su3_measurements_cl.cl:292-319, which
 * FN(plaquette) follows): Re Tr(a b c^+ d^+) as a b (full product), then
 * (a b) c^+, then the trace against d, with the same dot products. */
static REAL FN(retr4_lp)(const M3 *a, const M3 *b, const M3 *c, const M3 *d)
{
    M3 ab = FN(mul3)(a, b), abc;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) abc.m[i][j] = FN(dotc3)(&ab.m[i][0], 1, &c->m[j][0], 1);
    REAL tr = 0;
    for (int i = 0; i < 3; i++) tr += FN(dotc3)(&abc.m[i][0], 1, &d->m[i][0], 1).re;
    return tr;
}
/* a stored link as a full 3x3 in the link precision; SU(2) in the upper
 * 2x2 block with a zero third row and column */
static M3 FN(load_lp)(const ol_cfg *c, const REAL *tab, const crd *co, int mu)
{
    unsigned g = c2gid(c, *co);
    if (c->group == 3) return FN(expand)(FN(load3)(c, tab, co, g, mu));
    R4 a = FN(load2)(c, tab, co, g, mu).uv1;
    M3 m;
    memset(&m, 0, sizeof(m));
    m.m[0][0].re = a.x;  m.m[0][0].im = a.z;
    m.m[0][1].re = a.y;  m.m[0][1].im = a.w;
    m.m[1][0].re = -a.y; m.m[1][0].im = a.w;
    m.m[1][1].re = a.x;  m.m[1][1].im = -a.z;
    return m;
}
/* spatial / temporal sums; per site the six traces in the order xy, xz,
 * xt, yz, yt, zt, each converted to FP64 and summed in FP64 */
static void FN(plaquette_lp)(const ol_cfg *c, const REAL *tab, double out[2])
{
    int V = sites_of(c);
    double sp = 0, tp = 0;
    for (int g = 0; g < V; g++) {
        crd co; gid2c(c, g, &co);
        crd cx = nb_plus(c, co, 0), cy = nb_plus(c, co, 1), cz = nb_plus(c, co, 2), ct = nb_plus(c, co, 3);
        M3 m1 = FN(load_lp)(c, tab, &co, 0), m4 = FN(load_lp)(c, tab, &co, 1);
        M3 m5 = FN(load_lp)(c, tab, &co, 2), m6 = FN(load_lp)(c, tab, &co, 3), b, d;
        double rs, rt;
        b = FN(load_lp)(c, tab, &cx, 1); d = FN(load_lp)(c, tab, &cy, 0); rs  = (double)FN(retr4_lp)(&m1, &b, &d, &m4);
        b = FN(load_lp)(c, tab, &cx, 2); d = FN(load_lp)(c, tab, &cz, 0); rs += (double)FN(retr4_lp)(&m1, &b, &d, &m5);
        b = FN(load_lp)(c, tab, &cx, 3); d = FN(load_lp)(c, tab, &ct, 0); rt  = (double)FN(retr4_lp)(&m1, &b, &d, &m6);
        b = FN(load_lp)(c, tab, &cy, 2); d = FN(load_lp)(c, tab, &cz, 1); rs += (double)FN(retr4_lp)(&m4, &b, &d, &m5);
        b = FN(load_lp)(c, tab, &cy, 3); d = FN(load_lp)(c, tab, &ct, 1); rt += (double)FN(retr4_lp)(&m4, &b, &d, &m6);
        b = FN(load_lp)(c, tab, &cz, 3); d = FN(load_lp)(c, tab, &ct, 2); rt += (double)FN(retr4_lp)(&m5, &b, &d, &m6);
        sp += rs; tp += rt;
    }
    out[0] = sp; out[1] = tp;
}

/* lattice_action_diff_{x,y,z} (sun_measurements_cl.cl:187-615): the
 * spatial and temporal action (beta/N)(3N - ReTr) summed over the sites of
 * each slice of coordinate `axis`; out[2 i], out[2 i + 1] for slice i */
static void FN(action_profile)(const ol_cfg *c, const REAL *tab, int axis, double *out)
{
    int V = sites_of(c);
    REAL bet = (REAL)(c->beta / c->group);
    memset(out, 0, sizeof(double) * 2 * c->n[axis]);
    for (int g = 0; g < V; g++) {
        crd co; gid2c(c, g, &co);
        double rs, rt;
        FN(plaq_site)(c, tab, co, &rs, &rt);
        int k = crd_get(co, axis);
        out[2 * k] += (double)bet * (3.0 * c->group - rs);
        out[2 * k + 1] += (double)bet * (3.0 * c->group - rt);
    }
}

/* F_munu (FMUNU / F0MU variants of lattice_measurement_plq,
 * sun_measurements_cl.cl:712-1175): for the planes xy, xz, yz (field 0,
 * chromomagnetic) or xt, yt, zt (field 1, chromoelectric) the projections
 * -i Tr(P T_a) of the plaquette matrix P on the generators T = lambda/2
 * (SU(3), index 1..8) or sigma/2 (SU(2), index 1..3), summed over sites:
 * out[2 p], out[2 p + 1] = Re, Im for generator i1 and plane p,
 * out[6 + 2 p], out[7 + 2 p] the same for i2 */
static void FN(fmunu)(const ol_cfg *c, const REAL *tab, int field, int i1, int i2, double out[12])
{
    static const int hp[3][2] = { {0, 1}, {0, 2}, {1, 2} }, ep[3][2] = { {0, 3}, {1, 3}, {2, 3} };
    int V = sites_of(c);
    memset(out, 0, sizeof(double) * 12);
    for (int g = 0; g < V; g++) {
        crd co; gid2c(c, g, &co);
        for (int p = 0; p < 3; p++) {
            const int *pl = field ? ep[p] : hp[p];
            cd3 w;
            double f[2];
            FN(plaq_mat)(c, tab, co, pl[0], pl[1], &w);
            gen_proj(&w, c->group, i1, f);
            out[2 * p] += f[0]; out[2 * p + 1] += f[1];
            gen_proj(&w, c->group, i2, f);
            out[6 + 2 * p] += f[0]; out[7 + 2 * p] += f[1];
        }
    }
}

/* lattice_polyakov, polyakov.cl:54-140: ordered product of N4 T-links in
 * REAL precision, Re/Im trace to double. */
static void FN(poly_site)(const ol_cfg *c, const REAL *tab, int x, int y, int z, double *pr_out, double *pi_out)
{
    crd co = { x, y, z, 0 };
    double pr, pi;
    if (c->group == 3) {
        M3 v0 = FN(expand)(FN(load3)(c, tab, &co, c2gid(c, co), 3));
        for (int i = 1; i < c->n[3]; i++) {
            co = nb_plus(c, co, 3);
            M3 v1 = FN(expand)(FN(load3)(c, tab, &co, c2gid(c, co), 3));
            v0 = FN(mul3)(&v0, &v1);
        }
        pr = (double)v0.m[0][0].re + (double)v0.m[1][1].re + (double)v0.m[2][2].re;
        pi = (double)v0.m[0][0].im + (double)v0.m[1][1].im + (double)v0.m[2][2].im;
    } else {
        S2 v0 = FN(rec2)(FN(load2)(c, tab, &co, c2gid(c, co), 3).uv1);
        for (int i = 1; i < c->n[3]; i++) {
            co = nb_plus(c, co, 3);
            S2 v1 = FN(rec2)(FN(load2)(c, tab, &co, c2gid(c, co), 3).uv1);
            v0 = FN(mul2)(&v0, &v1);
        }
        pr = (double)v0.u1.re + (double)v0.v2.re;
        pi = (double)v0.u1.im + (double)v0.v2.im;
    }
    *pr_out = pr; *pi_out = pi;
}
static void FN(polyakov)(const ol_cfg *c, const REAL *tab, double out[4])
{
    double re = 0, im = 0, p2 = 0, p4 = 0;
    for (int x = 0; x < c->n[0]; x++)
        for (int z = 0; z < c->n[2]; z++)
            for (int y = 0; y < c->n[1]; y++) {
                double pr, pi;
                FN(poly_site)(c, tab, x, y, z, &pr, &pi);
                re += pr; im += pi;
                double q2 = pr * pr + pi * pi;
                p2 += q2; p4 += q2 * q2;
            }
    out[0] = re; out[1] = im; out[2] = p2; out[3] = p4;
}
/* lattice_polyakov_diff_{x,y,z} (polyakov.cl:142-402): Re, Im Tr of the
 * Polyakov loop summed over the spatial sites of each slice of coordinate
 * `axis` (0 x, 1 y, 2 z); out[2 i], out[2 i + 1] for slice i */
static void FN(polyakov_profile)(const ol_cfg *c, const REAL *tab, int axis, double *out)
{
    memset(out, 0, sizeof(double) * 2 * c->n[axis]);
    for (int x = 0; x < c->n[0]; x++)
        for (int z = 0; z < c->n[2]; z++)
            for (int y = 0; y < c->n[1]; y++) {
                double pr, pi;
                FN(poly_site)(c, tab, x, y, z, &pr, &pi);
                int k = axis == 0 ? x : axis == 1 ? y : z;
                out[2 * k] += pr; out[2 * k + 1] += pi;
            }
}

/* lattice_measurement_wilson, wilson_loop.cl:55-454: for every site and
 * i in {x,y,z}, Re Tr of the R x T loop (R along i, T along t), FP64. */
static double FN(wilson)(const ol_cfg *c, const REAL *tab, int R, int T)
{
    int V = sites_of(c), N = c->group;
    double sum = 0;
    for (int g = 0; g < V; g++) {
        crd c1; gid2c(c, g, &c1);
        cd3 m1, m2, m3, m4, m5, w;
        crd co = c1;
        FN(load_d)(c, tab, &co, 3, &m1);
        for (int k = 1; k < T; k++) { co = nb_plus(c, co, 3); FN(load_d)(c, tab, &co, 3, &m5); cd_mul(&m1, &m5, &w, N); m1 = w; }
        crd c2 = nb_plus(c, co, 3);                 /* x + T t^ */
        for (int i = 0; i < 3; i++) {
            crd a = c1, b = c2;
            FN(load_d)(c, tab, &a, i, &m4);
            FN(load_d)(c, tab, &b, i, &m2);
            for (int k = 1; k < R; k++) {
                a = nb_plus(c, a, i); b = nb_plus(c, b, i);
                FN(load_d)(c, tab, &a, i, &m5); cd_mul(&m4, &m5, &w, N); m4 = w;
                FN(load_d)(c, tab, &b, i, &m5); cd_mul(&m2, &m5, &w, N); m2 = w;
            }
            crd c4 = nb_plus(c, a, i);             /* x + R i^ */
            FN(load_d)(c, tab, &c4, 3, &m3);
            for (int k = 1; k < T; k++) { c4 = nb_plus(c, c4, 3); FN(load_d)(c, tab, &c4, 3, &m5); cd_mul(&m3, &m5, &w, N); m3 = w; }
            cd3 h, w1, w3;
            cd_mul(&m1, &m2, &w1, N);
            cd_herm(&m3, &h, N);
            cd_mul(&w1, &h, &w3, N);
            cd_herm(&m4, &h, N);
            cd_mul(&w3, &h, &w1, N);
            sum += cd_retr(&w1, N);
        }
    }
    return sum;
}

/* local Wilson action of one link (used by property tests of OR) */
static double FN(local_action)(const ol_cfg *c, const REAL *tab, unsigned g, int mu)
{
    crd co; gid2c(c, g, &co);
    double s = 0;
    if (c->group == 3) {
        M3 st = FN(staple3)(c, tab, g, mu);
        M3 u = FN(expand)(FN(load3)(c, tab, &co, g, mu));
        M3 p = FN(mul3)(&u, &st);
        s = (double)p.m[0][0].re + (double)p.m[1][1].re + (double)p.m[2][2].re;
    } else {
        S2 st = FN(staple2)(c, tab, g, mu);
        S2 u = FN(rec2)(FN(load2)(c, tab, &co, g, mu).uv1);
        /* Re Tr(u * st) */
        s = (double)(u.u1.re * st.u1.re - u.u1.im * st.u1.im + u.u2.re * st.v1.re - u.u2.im * st.v1.im)
          + (double)(u.v1.re * st.u2.re - u.v1.im * st.u2.im + u.v2.re * st.v2.re - u.v2.im * st.v2.im);
    }
    return s;
}

#undef R4
#undef CX
#undef G3
#undef M3
#undef RFMA
#undef G2
#undef S2
#undef FN
#undef RPI
#undef RPI2
#undef RSIN
#undef RCOS
#undef RSQRT
