/*
 * qg_oracle_learned.h -- CPU restatement of the learned-proposal
 * Metropolis update and of its training gradient (SU(3), float links).
 *
 * TEST INFRASTRUCTURE ONLY.  Included once at the end of qg_oracle.c, after
 * the float instantiation of qg_oracle_impl.h, whose staple terms, algebra
 * and Gram-Schmidt it reuses.  The reference has no such update; this file
 * restates this library's own definition (qcdgpu_b200/csrc/qg_learned.cu) in
 * the same operation order, so that the Metropolis chain is reproduced bit
 * for bit and the training gradient to FP32 accumulation error:
 *   features  -> staple_features,   network -> mlp_out,
 *   one phase -> k_mh_phase,        gradient -> k_mh_grad.
 */

#define NF 8
#define NH 32
#define P_W1 0
#define P_B1 (P_W1 + NH * NF)
#define P_W2 (P_B1 + NH)
#define P_B2 (P_W2 + NH * NH)
#define P_W3 (P_B2 + NH)
#define P_B3 (P_W3 + NH)
#define NPAR (P_B3 + 1)

static cx_f tr_fbh_f(const m3_f *F, const m3_f *B)
{
    cx_f r;
    r.re = F->m[0][0].re * B->m[0][0].re;
    r.re = fmaf(F->m[0][0].im, B->m[0][0].im, r.re);
    r.im = F->m[0][0].im * B->m[0][0].re;
    r.im = fmaf(-F->m[0][0].re, B->m[0][0].im, r.im);
    for (int q = 1; q < 9; q++) {
        cx_f f = F->m[q / 3][q % 3], b = B->m[q / 3][q % 3];
        r.re = fmaf(f.re, b.re, r.re);
        r.re = fmaf(f.im, b.im, r.re);
        r.im = fmaf(f.im, b.re, r.im);
        r.im = fmaf(-f.re, b.im, r.im);
    }
    return r;
}

static cx_f cmsub_f(cx_f a, cx_f b, cx_f c, cx_f d)
{
    cx_f r;
    r.re = a.re * b.re;
    r.re = fmaf(-a.im, b.im, r.re);
    r.re = fmaf(-c.re, d.re, r.re);
    r.re = fmaf(c.im, d.im, r.re);
    r.im = a.re * b.im;
    r.im = fmaf(a.im, b.re, r.im);
    r.im = fmaf(-c.re, d.im, r.im);
    r.im = fmaf(-c.im, d.re, r.im);
    return r;
}

/* staple of link (g, mu) in staple3's order, and the 8 features */
static void mh_features_f(const ol_cfg *c, const float *tab, unsigned g, int mu, m3_f *st, float x[NF])
{
    crd co, cp, cn, cm, cmp;
    gid2c(c, g, &co);
    cp = nb_plus(c, co, mu);
    m3_f s2;
    float rr[3], qq[3];
    for (int i = 0; i < 3; i++) {
        int nu = nu_order_f[mu][i];
        cn = nb_plus(c, co, nu);
        cm = nb_minus(c, co, nu);
        cmp = nb_plus(c, cm, mu);
        g3_f a = load3_f(c, tab, &cp, c2gid(c, cp), nu);
        g3_f b = load3_f(c, tab, &cn, c2gid(c, cn), mu);
        g3_f d = load3_f(c, tab, &co, g, nu);
        m3_f fw = staple_fwd3_f(a, b, d);
        a = load3_f(c, tab, &cmp, c2gid(c, cmp), nu);
        b = load3_f(c, tab, &cm, c2gid(c, cm), mu);
        d = load3_f(c, tab, &cm, c2gid(c, cm), nu);
        m3_f bw = staple_bwd3_f(a, b, d);
        cx_f tr = tr_fbh_f(&fw, &bw);
        rr[i] = tr.re / 3.0f;
        qq[i] = tr.im / 3.0f;
        if (i == 0) {
            *st = add3_f(&fw, &bw);
        } else {
            s2 = add3_f(st, &fw);
            *st = add3_f(&bw, &s2);
        }
    }
    const m3_f *A = st;
    float tn = A->m[0][0].re * A->m[0][0].re;
    tn = fmaf(A->m[0][0].im, A->m[0][0].im, tn);
    for (int q = 1; q < 9; q++) {
        tn = fmaf(A->m[q / 3][q % 3].re, A->m[q / 3][q % 3].re, tn);
        tn = fmaf(A->m[q / 3][q % 3].im, A->m[q / 3][q % 3].im, tn);
    }
    float t2 = 0.0f;
    for (int q = 0; q < 9; q++) {
        cx_f m = dotc3_f(&A->m[q / 3][0], 1, &A->m[q % 3][0], 1);
        t2 = (q == 0) ? m.re * m.re : fmaf(m.re, m.re, t2);
        t2 = fmaf(m.im, m.im, t2);
    }
    cx_f c0 = cmsub_f(A->m[1][1], A->m[2][2], A->m[1][2], A->m[2][1]);
    cx_f c1 = cmsub_f(A->m[1][0], A->m[2][2], A->m[1][2], A->m[2][0]);
    cx_f c2 = cmsub_f(A->m[1][0], A->m[2][1], A->m[1][1], A->m[2][0]);
    float dre = A->m[0][0].re * c0.re;
    dre = fmaf(-A->m[0][0].im, c0.im, dre);
    dre = fmaf(-A->m[0][1].re, c1.re, dre);
    dre = fmaf(A->m[0][1].im, c1.im, dre);
    dre = fmaf(A->m[0][2].re, c2.re, dre);
    dre = fmaf(-A->m[0][2].im, c2.im, dre);
    float dim = A->m[0][0].re * c0.im;
    dim = fmaf(A->m[0][0].im, c0.re, dim);
    dim = fmaf(-A->m[0][1].re, c1.im, dim);
    dim = fmaf(-A->m[0][1].im, c1.re, dim);
    dim = fmaf(A->m[0][2].re, c2.im, dim);
    dim = fmaf(A->m[0][2].im, c2.re, dim);
    float s = tn / 3.0f, n3 = s * sqrtf(s);
    x[0] = tn / 108.0f;
    x[1] = (tn > 0.0f) ? t2 / (tn * tn) : 1.0f;
    x[2] = (n3 > 0.0f) ? dre / n3 : 0.0f;
    x[3] = (n3 > 0.0f) ? dim / n3 : 0.0f;
    x[4] = ((rr[0] + rr[1]) + rr[2]) / 3.0f;
    x[5] = fmaf(rr[2], rr[2], fmaf(rr[1], rr[1], rr[0] * rr[0])) / 3.0f;
    x[6] = ((qq[0] + qq[1]) + qq[2]) / 3.0f;
    x[7] = fmaf(qq[2], qq[2], fmaf(qq[1], qq[1], qq[0] * qq[0])) / 3.0f;
}

/* BF16 rounding (nearest even) of a finite float, as a float */
static float bf16r(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    u &= 0xFFFF0000u;
    float r;
    memcpy(&r, &u, 4);
    return r;
}

/* forward pass as the tensor-core kernels define it (net_forward of
 * qg_learned.cu): the features and the first hidden layer enter the
 * products rounded to BF16, products and sums in FP32 (here summed in
 * order; the tensor core sums in its own order), the bias added after the
 * product, the output layer an FP32 dot product from b3 in order */
static float mlp_fwd_tc_f(const float *w, const float x[NF], float z1[NH], float z2[NH])
{
    float xb[NF], h[NH];
    for (int k = 0; k < NF; k++) xb[k] = bf16r(x[k]);
    for (int j = 0; j < NH; j++) {
        float z = 0.0f;
        for (int k = 0; k < NF; k++) z = fmaf(xb[k], w[P_W1 + j * NF + k], z);
        z1[j] = z + w[P_B1 + j];
    }
    for (int k = 0; k < NH; k++) h[k] = bf16r(z1[k] > 0.0f ? z1[k] : 0.0f);
    float o = w[P_B3];
    for (int j = 0; j < NH; j++) {
        float z = 0.0f;
        for (int k = 0; k < NH; k++) z = fmaf(h[k], w[P_W2 + j * NH + k], z);
        z2[j] = z + w[P_B2 + j];
        o = fmaf(w[P_W3 + j], z2[j] > 0.0f ? z2[j] : 0.0f, o);
    }
    return o;
}

/* the same network without the BF16 operand rounding (FP32 throughout),
 * whose analytic gradient the finite-difference check compares with the
 * FP64 loss */
static float mlp_fwd_f(const float *w, const float x[NF], float z1[NH], float z2[NH])
{
    for (int j = 0; j < NH; j++) {
        float z = w[P_B1 + j];
        for (int k = 0; k < NF; k++) z = fmaf(w[P_W1 + j * NF + k], x[k], z);
        z1[j] = z;
    }
    float o = w[P_B3];
    for (int j = 0; j < NH; j++) {
        float z = w[P_B2 + j];
        for (int k = 0; k < NH; k++) z = fmaf(w[P_W2 + j * NH + k], z1[k] > 0.0f ? z1[k] : 0.0f, z);
        z2[j] = z;
        o = fmaf(w[P_W3 + j], z > 0.0f ? z : 0.0f, o);
    }
    return o;
}

static double sigmoid_dd(float o) { return 1.0 / (1.0 + ol_exp(-(double)o)); }

static void normals3_f(const float q[4], double *a0, double *a1, double *a2)
{
    double l1 = sqrt(-2.0 * ol_log((double)q[0])), l3 = sqrt(-2.0 * ol_log((double)q[2]));
    double s1, c1, s3, c3;
    ol_sincos(6.283185307179586 * (double)q[1], &s1, &c1);
    ol_sincos(6.283185307179586 * (double)q[3], &s3, &c3);
    *a0 = l1 * c1;
    *a1 = l1 * s1;
    *a2 = l3 * c3;
}

static void block_coeffs_f(const m3_f *U, const m3_f *A, int i, int j, double c[4])
{
    s2_f w;
    w.u1 = dot3_f(&U->m[i][0], 1, &A->m[0][i], 3);
    w.u2 = dot3_f(&U->m[i][0], 1, &A->m[0][j], 3);
    w.v1 = dot3_f(&U->m[j][0], 1, &A->m[0][i], 3);
    w.v2 = dot3_f(&U->m[j][0], 1, &A->m[0][j], 3);
    c[0] = (double)w.u1.re + (double)w.v2.re;
    c[1] = -((double)w.v1.im + (double)w.u2.im);
    c[2] = (double)w.v1.re - (double)w.u2.re;
    c[3] = -((double)w.u1.im - (double)w.v2.im);
}

/* ---------------------------------------------------------------- public */
void ol_mh_features(const ol_cfg *c, const void *tab, int gid, int mu, float x[NF])
{
    m3_f st;
    mh_features_f(c, (const float *)tab, (unsigned)gid, mu, &st, x);
}

float ol_mlp_out(const float *w, const float x[NF])
{
    float z1[NH], z2[NH];
    return mlp_fwd_tc_f(w, x, z1, z2);
}

/* the step of every link of a phase (the GPU's qg_net_eps) */
void ol_net_eps(const ol_cfg *c, const void *table, int parity, int mu, const float *w, double eps_max, float *eps)
{
    const float *tab = (const float *)table;
    unsigned half = (unsigned)(sites_of(c) / 2);
#pragma omp parallel for schedule(static)
    for (unsigned t = 0; t < half; t++) {
        unsigned g = parity ? odd_gid(c, t) : even_gid(c, t);
        m3_f st;
        float x[NF], z1[NH], z2[NH];
        mh_features_f(c, tab, g, mu, &st, x);
        eps[t] = (float)(eps_max * sigmoid_dd(mlp_fwd_tc_f(w, x, z1, z2)));
    }
}

/* the Metropolis hits of link t of a phase with step eps (k_mh_phase after
 * the network) */
static void mh_link_f(const ol_cfg *c, float *tab, int parity, int mu, unsigned t, float eps, int nhit,
                      const ol_prn *src, double bn, uint64_t *acc, double *jump)
{
    unsigned g = parity ? odd_gid(c, t) : even_gid(c, t);
    crd co;
    gid2c(c, g, &co);
    m3_f st;
    float x[NF];
    mh_features_f(c, tab, g, mu, &st, x);
    m3_f U = expand_f(load3_f(c, tab, &co, g, mu));
    uint32_t k = 0;
    for (int h = 0; h < nhit; h++)
        for (int sg = 0; sg < 3; sg++) {
            int i = (sg == 2) ? 1 : 0, j = (sg == 0) ? 1 : 2;
            float q1[4], q2[4];
            ol_philox_prn(src, t, k++, q1);
            ol_philox_prn(src, t, k++, q2);
            double a0, a1, a2;
            normals3_f(q1, &a0, &a1, &a2);
            double r = sqrt(fma(a2, a2, fma(a1, a1, a0 * a0)));
            double th = (double)eps * r, sn, cs;
            ol_sincos(th, &sn, &cs);
            double sr = (r > 0.0) ? sn / r : 0.0;
            float x0 = (float)cs, x1 = (float)(sr * a0), x2 = (float)(sr * a1), x3 = (float)(sr * a2);
            double cc[4];
            block_coeffs_f(&U, &st, i, j, cc);
            double dS = -bn * fma((double)x0 - 1.0, cc[0], fma((double)x1, cc[1], fma((double)x2, cc[2], (double)x3 * cc[3])));
            if (ol_log((double)q2[0]) <= -dS) {
                s2_f V;
                V.u1.re = x0; V.u1.im = x3; V.u2.re = x2; V.u2.im = x1;
                V.v1.re = -x2; V.v1.im = x1; V.v2.re = x0; V.v2.im = -x3;
                rotate_rows_f(&U, i, j, &V);
                (*acc)++;
                *jump += th * th;
            }
        }
    store3_f(c, tab, g, mu, gs3_f(compress_f(&U)));
}

/* one learned-proposal Metropolis phase (k_mh_phase); w holds the BF16
 * weights as floats, the network as the tensor-core kernels define it */
void ol_mh_phase(const ol_cfg *c, void *table, int parity, int mu, const float *w, double eps_max, int nhit,
                 uint32_t key0, uint32_t key1, uint64_t phase, uint64_t *acc_out, double *jump_out)
{
    unsigned half = (unsigned)(sites_of(c) / 2);
    float *eps = (float *)malloc((size_t)half * sizeof(float));
    ol_net_eps(c, table, parity, mu, w, eps_max, eps);
    ol_mh_phase_eps(c, table, parity, mu, eps, nhit, key0, key1, phase, acc_out, jump_out);
    free(eps);
}

/* the same phase with the step of link t given as eps[t] */
void ol_mh_phase_eps(const ol_cfg *c, void *table, int parity, int mu, const float *eps, int nhit, uint32_t key0,
                     uint32_t key1, uint64_t phase, uint64_t *acc_out, double *jump_out)
{
    float *tab = (float *)table;
    unsigned half = (unsigned)(sites_of(c) / 2);
    const double bn = (double)(float)(c->beta / c->group);
    ol_prn src;
    memset(&src, 0, sizeof(src));
    src.mode = 1; src.key0 = key0; src.key1 = key1; src.phase = phase;
    uint64_t acc = 0;
    double jump = 0.0;
    /* links updated independently; the jump sum's order differs with the
     * thread count (it is a statistic, compared within a tolerance) */
#pragma omp parallel for schedule(static) reduction(+ : acc, jump)
    for (unsigned t = 0; t < half; t++) mh_link_f(c, tab, parity, mu, t, eps[t], nhit, &src, bn, &acc, &jump);
    if (acc_out) *acc_out = acc;
    if (jump_out) *jump_out = jump;
}

/* the training loss gradient of one phase (k_mh_grad + k_mh_grad_reduce):
 * per-link arithmetic as on the GPU (FP32 network, FP64 acceptance), the
 * sums over links in FP64; grad[NPAR] = mean over links, stats = {loss,
 * ESJD, acceptance} per link and the link count.  tc = 1: the network and
 * the back-propagated values rounded to BF16 where the tensor-core kernels
 * round them (the features, h1, h2, dz2, dz1 and dL/do as MMA operands);
 * tc = 0: FP32 throughout (the analytic gradient of the FP32 network) */
void ol_mh_grad(const ol_cfg *c, const void *table, int parity, int mu, const float *w, double eps_max,
                uint32_t key0, uint32_t key1, uint64_t phase, int tc, double *grad, double stats[4])
{
    const float *tab = (const float *)table;
    unsigned half = (unsigned)(sites_of(c) / 2);
    const double bn = (double)(float)(c->beta / c->group);
    ol_prn src;
    memset(&src, 0, sizeof(src));
    src.mode = 1; src.key0 = key0; src.key1 = key1; src.phase = phase;
    for (int q = 0; q < NPAR; q++) grad[q] = 0.0;
    double sl = 0, se = 0, sa = 0;
    for (unsigned t = 0; t < half; t++) {
        unsigned g = parity ? odd_gid(c, t) : even_gid(c, t);
        crd co;
        gid2c(c, g, &co);
        m3_f st;
        float x[NF], z1[NH], z2[NH];
        mh_features_f(c, tab, g, mu, &st, x);
        float o = tc ? mlp_fwd_tc_f(w, x, z1, z2) : mlp_fwd_f(w, x, z1, z2);
        double sg = sigmoid_dd(o), eps = eps_max * sg;
        m3_f U = expand_f(load3_f(c, tab, &co, g, mu));
        double geps = 0, es = 0, ac = 0;
        for (int s = 0; s < 3; s++) {
            int i = (s == 2) ? 1 : 0, j = (s == 0) ? 1 : 2;
            float q1[4];
            ol_philox_prn(&src, t, (uint32_t)s, q1);
            double a0, a1, a2;
            normals3_f(q1, &a0, &a1, &a2);
            double r = sqrt(fma(a2, a2, fma(a1, a1, a0 * a0)));
            double th = eps * r, sn, cs;
            ol_sincos(th, &sn, &cs);
            double cc[4];
            block_coeffs_f(&U, &st, i, j, cc);
            double ahc = (r > 0.0) ? (a0 * cc[1] + a1 * cc[2] + a2 * cc[3]) / r : 0.0;
            double dS = -bn * ((cs - 1.0) * cc[0] + sn * ahc);
            double dSde = -bn * r * (-sn * cc[0] + cs * ahc);
            double a = (dS <= 0.0) ? 1.0 : ol_exp(-dS);
            double dade = (dS <= 0.0) ? 0.0 : -a * dSde;
            es += a * th * th;
            ac += a;
            geps -= dade * th * th + a * 2.0 * eps * r * r;
        }
        sl -= es;
        se += es;
        sa += ac / 3.0;
        float go = (float)(geps * eps_max * sg * (1.0 - sg));
        float dz2[NH], h1[NH], h2[NH], xo[NF];
        for (int jj = 0; jj < NH; jj++) {
            h1[jj] = z1[jj] > 0.0f ? z1[jj] : 0.0f;
            h2[jj] = z2[jj] > 0.0f ? z2[jj] : 0.0f;
            dz2[jj] = z2[jj] > 0.0f ? go * w[P_W3 + jj] : 0.0f;
            if (tc) { h1[jj] = bf16r(h1[jj]); h2[jj] = bf16r(h2[jj]); dz2[jj] = bf16r(dz2[jj]); }
        }
        for (int m = 0; m < NF; m++) xo[m] = tc ? bf16r(x[m]) : x[m];
        const float gq = tc ? bf16r(go) : go;
        for (int jj = 0; jj < NH; jj++) {
            grad[P_W3 + jj] += (double)gq * (double)h2[jj];
            grad[P_B2 + jj] += (double)dz2[jj];
            for (int k = 0; k < NH; k++) grad[P_W2 + jj * NH + k] += (double)dz2[jj] * (double)h1[k];
        }
        grad[P_B3] += (double)gq;
        for (int k = 0; k < NH; k++) {
            float d = 0.0f;
            for (int jj = 0; jj < NH; jj++) d = fmaf(w[P_W2 + jj * NH + k], dz2[jj], d);
            float dz1 = z1[k] > 0.0f ? d : 0.0f;
            if (tc) dz1 = bf16r(dz1);
            grad[P_B1 + k] += (double)dz1;
            for (int m = 0; m < NF; m++) grad[P_W1 + k * NF + m] += (double)dz1 * (double)xo[m];
        }
    }
    for (int q = 0; q < NPAR; q++) grad[q] /= (double)half;
    stats[0] = sl / half;
    stats[1] = se / half;
    stats[2] = sa / half;
    stats[3] = (double)half;
}

/* the training loss alone, in FP64 throughout (weights and features as
 * floats), for a finite-difference check of the analytic gradient */
double ol_mh_loss(const ol_cfg *c, const void *table, int parity, int mu, const double *w, double eps_max,
                  uint32_t key0, uint32_t key1, uint64_t phase)
{
    const float *tab = (const float *)table;
    unsigned half = (unsigned)(sites_of(c) / 2);
    const double bn = (double)(float)(c->beta / c->group);
    ol_prn src;
    memset(&src, 0, sizeof(src));
    src.mode = 1; src.key0 = key0; src.key1 = key1; src.phase = phase;
    double loss = 0.0;
    for (unsigned t = 0; t < half; t++) {
        unsigned g = parity ? odd_gid(c, t) : even_gid(c, t);
        crd co;
        gid2c(c, g, &co);
        m3_f st;
        float x[NF];
        mh_features_f(c, tab, g, mu, &st, x);
        double h1[NH], o = w[P_B3];
        for (int j = 0; j < NH; j++) {
            double z = w[P_B1 + j];
            for (int k = 0; k < NF; k++) z += w[P_W1 + j * NF + k] * x[k];
            h1[j] = z > 0 ? z : 0;
        }
        for (int j = 0; j < NH; j++) {
            double z = w[P_B2 + j];
            for (int k = 0; k < NH; k++) z += w[P_W2 + j * NH + k] * h1[k];
            o += w[P_W3 + j] * (z > 0 ? z : 0);
        }
        double eps = eps_max / (1.0 + exp(-o));
        m3_f U = expand_f(load3_f(c, tab, &co, g, mu));
        for (int s = 0; s < 3; s++) {
            int i = (s == 2) ? 1 : 0, j = (s == 0) ? 1 : 2;
            float q1[4];
            ol_philox_prn(&src, t, (uint32_t)s, q1);
            double a0, a1, a2;
            normals3_f(q1, &a0, &a1, &a2);
            double r = sqrt(a0 * a0 + a1 * a1 + a2 * a2);
            double th = eps * r;
            double cc[4];
            block_coeffs_f(&U, &st, i, j, cc);
            double ahc = (r > 0.0) ? (a0 * cc[1] + a1 * cc[2] + a2 * cc[3]) / r : 0.0;
            double dS = -bn * ((cos(th) - 1.0) * cc[0] + sin(th) * ahc);
            double a = (dS <= 0.0) ? 1.0 : exp(-dS);
            loss -= a * th * th;
        }
    }
    return loss / half;
}
