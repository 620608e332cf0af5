// qg_host.cpp -- the host side of a run: init.dat parsing, the run loop
// with its measurement cadence, the statistics, the CPU re-measurement of
// the last configuration and the results file.  Restates the reference's
// model class behaviour (SU(N)/suncl/suncl.cpp) on top of the C-ABI.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <chrono>
#include <string>
#include <vector>

#include "../../include/qcdgpu_b200.h"

void qg_set_global_error(const std::string &m);   // qg_capi.cu: qg_last_error(NULL)

namespace {

int host_fail(int code, const std::string &m)
{
    qg_set_global_error(m);
    return code;
}

std::string trim(const std::string &s)
{
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// ------------------------------------------------------------------ FP64
// host re-measurement of the last configuration from the reference-layout
// table, as LatticeCheckCPU does (SU(N)/suncl/su3cpu.cpp:1155-1433)
struct C { double re, im; };
struct M { C m[3][3]; };

struct Table {
    int group, n[4], prec;
    uint32_t rowsize;
    const void *p;
    double at(uint32_t site, int plane, int c) const
    {
        size_t i = ((size_t)site + (size_t)plane * rowsize) * 4 + c;
        return prec ? ((const double *)p)[i] : (double)((const float *)p)[i];
    }
    uint32_t site(const int x[4]) const
    {
        return (uint32_t)(x[1] + x[2] * n[1] + x[3] * n[1] * n[2] + x[0] * n[1] * n[2] * n[3]);
    }
    M link(const int x[4], int mu, double phi, double omega) const
    {
        uint32_t s = site(x);
        M a;
        memset(&a, 0, sizeof(a));
        if (group == 3) {
            double r1[4], i1[4], v[4];
            for (int c = 0; c < 4; c++) { r1[c] = at(s, mu, c); i1[c] = at(s, mu + 4, c); v[c] = at(s, mu + 8, c); }
            a.m[0][0] = { r1[0], i1[0] }; a.m[0][1] = { r1[1], i1[1] }; a.m[0][2] = { r1[2], i1[2] };
            a.m[1][0] = { v[0], v[2] };   a.m[1][1] = { v[1], v[3] };   a.m[1][2] = { r1[3], i1[3] };
            if (mu == 1 && x[0] == n[0] - 1 && !(phi == 0.0 && omega == 0.0)) {
                double p = (phi + omega) / 2, q = (omega - phi) / 2;
                C e1 = { cos(p), sin(p) }, e2 = { cos(q), sin(q) };
                for (int j = 0; j < 3; j++) {
                    C u = a.m[0][j], w = a.m[1][j];
                    a.m[0][j] = { u.re * e1.re - u.im * e1.im, u.re * e1.im + u.im * e1.re };
                    a.m[1][j] = { w.re * e2.re - w.im * e2.im, w.re * e2.im + w.im * e2.re };
                }
            }
            for (int j = 0; j < 3; j++) {     // row 3 = conj(row1 x row2)
                int p = (j + 1) % 3, q = (j + 2) % 3;
                C u1 = a.m[0][p], u2 = a.m[0][q], v1 = a.m[1][p], v2 = a.m[1][q];
                a.m[2][j] = { u1.re * v2.re - u1.im * v2.im - u2.re * v1.re + u2.im * v1.im,
                              -(u1.re * v2.im + u1.im * v2.re - u2.re * v1.im - u2.im * v1.re) };
            }
        } else {
            double q[4];
            for (int c = 0; c < 4; c++) q[c] = at(s, mu, c);
            if (mu == 1 && x[0] == n[0] - 1 && phi != 0.0) {
                double o[4] = { cos(phi / 2), 0.0, sin(phi / 2), 0.0 }, r[4];
                r[0] = o[0] * q[0] - o[1] * q[1] - o[2] * q[2] - o[3] * q[3];
                r[2] = o[0] * q[2] + o[2] * q[0] + o[1] * q[3] - o[3] * q[1];
                r[1] = o[0] * q[1] + o[1] * q[0] + o[3] * q[2] - o[2] * q[3];
                r[3] = o[0] * q[3] + o[3] * q[0] + o[2] * q[1] - o[1] * q[2];
                memcpy(q, r, sizeof(q));
            }
            a.m[0][0] = { q[0], q[2] };  a.m[0][1] = { q[1], q[3] };
            a.m[1][0] = { -q[1], q[3] }; a.m[1][1] = { q[0], -q[2] };
        }
        return a;
    }
};

M mul(const M &a, const M &b, int N)
{
    M r;
    memset(&r, 0, sizeof(r));
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            double re = 0, im = 0;
            for (int k = 0; k < N; k++) {
                re += a.m[i][k].re * b.m[k][j].re - a.m[i][k].im * b.m[k][j].im;
                im += a.m[i][k].re * b.m[k][j].im + a.m[i][k].im * b.m[k][j].re;
            }
            r.m[i][j] = { re, im };
        }
    return r;
}
M dag(const M &a, int N)
{
    M r;
    memset(&r, 0, sizeof(r));
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) r.m[i][j] = { a.m[j][i].re, -a.m[j][i].im };
    return r;
}
double retr(const M &a, int N)
{
    double s = 0;
    for (int i = 0; i < N; i++) s += a.m[i][i].re;
    return s;
}
void shift(int x[4], int d, int s, const int n[4]) { x[d] = (x[d] + s + n[d]) % n[d]; }

struct HostObs { double plq_s, plq_t, s_s, s_t, pre, pim, p2, p4, wilson, f[12], f2[12]; };

// -i Tr(P T_a) with T_a = lambda_a / 2 (SU(3)) or sigma_a / 2 (SU(2))
// (trace_lambda1..8_double, su3_measurements_cl.cl:355-460;
// trace_sigma1..3_double, su2_measurements_cl.cl:89-124)
void gen_proj(const M &P, int N, int a, double &re, double &im)
{
    const C u1 = P.m[0][0], u2 = P.m[0][1], u3 = P.m[0][2], v1 = P.m[1][0], v2 = P.m[1][1], v3 = P.m[1][2];
    const C w1 = P.m[2][0], w2 = P.m[2][1], w3 = P.m[2][2];
    re = 0; im = 0;
    if (N == 2) { re = a == 1 ? u2.im : a == 2 ? u2.re : u1.im; return; }
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
    }
    re /= 2; im /= 2;
}

// model_lattice_init (suncl.cpp:2212-2230): the F_munu generators
void fmunu_indices(int N, const qg_run_options &o, int &i1, int &i2)
{
    i1 = o.fmunu_index1; i2 = o.fmunu_index2;
    if (N == 3) {
        if (i1 != 1 && i1 != 2 && i1 != 4) i1 = 3;
        if (i2 < 5 || i2 > 7) i2 = 8;
    } else {
        if (i1 != 1) i1 = 3;
        i2 = 2;
    }
}

HostObs host_measure(const Table &T, const qg_config &f, const qg_run_options &o)
{
    HostObs h;
    memset(&h, 0, sizeof(h));
    const int N = T.group;
    const int *n = T.n;
    const double bet = f.precision ? f.beta / N : (double)(float)(f.beta / N);
    const double phi = f.precision ? f.phi : (double)(float)f.phi, om = f.precision ? f.omega : (double)(float)f.omega;
    int x[4];
    const long V = (long)n[0] * n[1] * n[2] * n[3];
    for (x[0] = 0; x[0] < n[0]; x[0]++)
        for (x[3] = 0; x[3] < n[3]; x[3]++)
            for (x[2] = 0; x[2] < n[2]; x[2]++)
                for (x[1] = 0; x[1] < n[1]; x[1]++) {
                    double rs = 0, rt = 0;
                    for (int mu = 0; mu < 3; mu++)
                        for (int nu = mu + 1; nu < 4; nu++) {
                            int a[4], b[4];
                            memcpy(a, x, sizeof(a)); shift(a, mu, 1, n);
                            memcpy(b, x, sizeof(b)); shift(b, nu, 1, n);
                            M p = mul(mul(mul(T.link(x, mu, phi, om), T.link(a, nu, phi, om), N),
                                          dag(T.link(b, mu, phi, om), N), N), dag(T.link(x, nu, phi, om), N), N);
                            (nu == 3 ? rt : rs) += retr(p, N);
                            if ((o.fmunu == 1 && nu != 3) || (o.fmunu == 2 && nu == 3)) {
                                int i1, i2;
                                fmunu_indices(N, o, i1, i2);
                                const int pl = o.fmunu == 2 ? mu : (mu == 0 ? nu - 1 : 2);
                                double re, im;
                                gen_proj(p, N, i1, re, im);
                                h.f[2 * pl] += re; h.f[2 * pl + 1] += im;
                                h.f2[2 * pl] += re * re; h.f2[2 * pl + 1] += im * im;
                                gen_proj(p, N, i2, re, im);
                                h.f[6 + 2 * pl] += re; h.f[7 + 2 * pl] += im;
                                h.f2[6 + 2 * pl] += re * re; h.f2[7 + 2 * pl] += im * im;
                            }
                        }
                    h.plq_s += rs; h.plq_t += rt;
                    h.s_s += bet * (3.0 * N - rs);
                    h.s_t += bet * (3.0 * N - rt);
                    if (o.get_wilson) {
                        const int R = f.wilson_r, TT = f.wilson_t;
                        for (int i = 0; i < 3; i++) {
                            int c[4];
                            memcpy(c, x, sizeof(c));
                            M w = T.link(c, i, phi, om);
                            for (int k = 1; k < R; k++) { shift(c, i, 1, n); w = mul(w, T.link(c, i, phi, om), N); }
                            shift(c, i, 1, n);
                            for (int k = 0; k < TT; k++) { w = mul(w, T.link(c, 3, phi, om), N); shift(c, 3, 1, n); }
                            for (int k = 0; k < R; k++) { shift(c, i, -1, n); w = mul(w, dag(T.link(c, i, phi, om), N), N); }
                            for (int k = 0; k < TT; k++) { shift(c, 3, -1, n); w = mul(w, dag(T.link(c, 3, phi, om), N), N); }
                            h.wilson += retr(w, N);
                        }
                    }
                }
    if (o.pl_level > 0) {
        for (x[0] = 0; x[0] < n[0]; x[0]++)
            for (x[2] = 0; x[2] < n[2]; x[2]++)
                for (x[1] = 0; x[1] < n[1]; x[1]++) {
                    x[3] = 0;
                    M p = T.link(x, 3, phi, om);
                    for (int k = 1; k < n[3]; k++) { x[3] = k; p = mul(p, T.link(x, 3, phi, om), N); }
                    double re = 0, im = 0;
                    for (int i = 0; i < N; i++) { re += p.m[i][i].re; im += p.m[i][i].im; }
                    double q2 = re * re + im * im;
                    h.pre += re; h.pim += im; h.p2 += q2; h.p4 += q2 * q2;
                }
    }
    (void)V;
    return h;
}

// data_analysis::lattice_data_analysis (SU(N)/data_analysis/data_analysis.cpp:107-134):
// mean and population variance over samples 1..n-1
void mean_var(const std::vector<double> &d, double &mean, double &var)
{
    mean = 0; var = 0;
    int last = (int)d.size() - 1;
    for (int i = 1; i <= last; i++) mean += d[i];
    if (last > 0) mean /= last;
    for (int i = 1; i <= last; i++) var += (d[i] - mean) * (d[i] - mean);
    if (last > 0) var /= last;
}

// CPU_GPU_verification_single / _double (data_analysis.cpp:40-43,76-100)
bool verify(double gpu, double cpu, bool single)
{
    const double floor_ = single ? 1e-6 : 1e-12, tol = single ? 0.00005 : 0.00000000001;
    if (fabs(gpu) > floor_ && fabs(cpu) > floor_) return fabs(1.0 - cpu / gpu) <= tol;
    return true;
}

}  // namespace

extern "C" int qg_default_run_options(qg_run_options *o)
{
    if (!o) return QG_ERR_ARG;
    memset(o, 0, sizeof(*o));
    o->iter = 2;
    o->niter = 1;
    o->nav = 0;
    o->pl_level = 3;
    o->get_wilson = 0;
    o->get_plaquettes = 1;
    o->get_actions = 1;
    o->verify = 1;
    o->write_results = 1;
    o->tune_shapes = 1;
    o->profile = 0;
    o->init = 1;
    snprintf(o->prefix, sizeof(o->prefix), "su3-");
    return QG_OK;
}

// GPU::get_init_file + model::lattice_get_init_file
// (SU(N)/clinterface/clinterface.cpp:2060-2154, SU(N)/suncl/suncl.cpp:289-464)
extern "C" int qg_parse_init_file(const char *path, qg_config *cfg, qg_run_options *o)
{
    if (!path || !cfg || !o) return host_fail(QG_ERR_ARG, "null argument");
    FILE *fp = fopen(path, "r");
    if (!fp) return host_fail(QG_ERR_IO, std::string("cannot open ") + path);
    char line[1024];
    int lineno = 0;
    while (fgets(line, sizeof(line), fp)) {
        lineno++;
        std::string s(line);
        size_t hash = s.find('#');
        if (hash != std::string::npos) s = s.substr(0, hash);
        size_t eq = s.find('=');
        if (eq == std::string::npos) continue;
        std::string key = trim(s.substr(0, eq)), val = trim(s.substr(eq + 1));
        if (key.empty()) continue;
        long iv = strtol(val.c_str(), nullptr, 10);
        double dv = strtod(val.c_str(), nullptr);
        if (key == "GROUP") { cfg->group = (int)iv; snprintf(o->prefix, sizeof(o->prefix), "su%ld-", iv); }
        else if (key == "ND") { if (iv != 4) { fclose(fp); return host_fail(QG_ERR_UNSUPPORTED, "only ND = 4 is supported"); } }
        else if (key == "L1") cfg->size[0] = (int)iv;
        else if (key == "L2") cfg->size[1] = (int)iv;
        else if (key == "L3") cfg->size[2] = (int)iv;
        else if (key == "L4") cfg->size[3] = (int)iv;
        else if (key == "LS") { cfg->size[0] = cfg->size[1] = cfg->size[2] = (int)iv; }
        else if (key == "LT") cfg->size[3] = (int)iv;
        else if (key == "ITER") o->iter = (int)iv;
        else if (key == "NITER") o->niter = (int)iv;
        else if (key == "NAV") o->nav = (int)iv;
        else if (key == "NHIT") cfg->nhit = (int)iv;
        else if (key == "BETA") cfg->beta = dv;
        else if (key == "PHI") cfg->phi = dv;
        else if (key == "OMEGA") cfg->omega = dv;
        else if (key == "INTS") cfg->start = (iv == 1) ? QG_START_COLD : (iv == 2) ? QG_START_GID : (iv == 3) ? QG_START_HAAR : QG_START_HOT;
        else if (key == "RANDSERIES") cfg->randseries = (uint32_t)iv;
        else if (key == "PRNG") {
            static const char *lux[] = { "RANLUX0", "RANLUX1", "RANLUX2", "RANLUX3", "RANLUX4" };
            static const int skips[] = { 24, 48, 97, 223, 389 };
            bool ok = false;
            for (int k = 0; k < 5; k++)
                if (val == lux[k]) { cfg->prng = QG_PRNG_RANLUX; cfg->ranlux_nskip = skips[k]; ok = true; }
            if (val == "RANLUX") { cfg->prng = QG_PRNG_RANLUX; ok = true; }
            if (val == "PHILOX") { cfg->prng = QG_PRNG_PHILOX; ok = true; }
            if (!ok) {
                fclose(fp);
                return host_fail(QG_ERR_UNSUPPORTED, "PRNG " + val + " is not available (RANLUX0..4, RANLUX, PHILOX)");
            }
        }
        else if (key == "OUTPUTPATH") snprintf(o->output_path, sizeof(o->output_path), "%s", val.c_str());
        else if (key == "GETWILSON") o->get_wilson = 1;
        else if (key == "GETRETRACE") o->get_plaquettes = 1;
        else if (key == "PL_LEVEL") o->pl_level = (int)iv;
        else if (key == "WILSONR") cfg->wilson_r = (int)iv;
        else if (key == "WILSONT") cfg->wilson_t = (int)iv;
        else if (key == "PRECISION") cfg->precision = (int)iv;
        else if (key == "NHITPAR") cfg->nhitpar = (int)iv;
        else if (key == "NOR") cfg->n_or = (int)iv;
        else if (key == "REUNIT_EVERY") cfg->reunit_every = (int)iv;
        else if (key == "REUNIT_FP64") cfg->reunit_fp64 = (int)iv;
        else if (key == "PRNG_INSTANCES") cfg->prng_instances = (int)iv;
        else if (key == "ROW_ALIGN") cfg->row_align = (int)iv;
        else if (key == "INIT") o->init = (int)iv;
        else if (key == "STATEFILE") snprintf(o->state_file, sizeof(o->state_file), "%s", val.c_str());
        else if (key == "SAVESTATE") o->save_state = (int)iv;
        else if (key == "SAVEEVERY") o->save_every_iter = (int)iv;
        else if (key == "STATEOUT") snprintf(o->state_out, sizeof(o->state_out), "%s", val.c_str());
        else if (key == "FMUNU") o->fmunu = 1;
        else if (key == "F0MU") o->fmunu = 2;
        else if (key == "TURNOFFFMUNU") o->fmunu = 0;
        else if (key == "FMUNU1") o->fmunu_index1 = 1;
        else if (key == "FMUNU2") o->fmunu_index1 = 2;
        else if (key == "FMUNU4") o->fmunu_index1 = 4;
        else if (key == "FMUNU5") o->fmunu_index2 = 5;
        else if (key == "FMUNU6") o->fmunu_index2 = 6;
        else if (key == "FMUNU7") o->fmunu_index2 = 7;
        else if (key == "ACTIONS_DIFF") o->get_actions_diff = (int)iv;
        else if (key == "TUNE") o->tune_shapes = (int)iv;
        else if (key == "PROFILE") o->profile = (int)iv;
        else if (key == "PLATFORM" || key == "DEVICE" || key == "FINISHPATH" || key == "TURNOFFWAITING" ||
                 key == "REBUILDBINARY" || key.rfind("FMUNU", 0) == 0 || key == "N1") {
            /* device selection, dispatcher handshake and OpenCL binaries have
               no role in this library; FMUNU3, FMUNU8, ... select nothing in the
               reference either */
        }
        else {
            fclose(fp);
            return host_fail(QG_ERR_ARG, "unknown key " + key + " at line " + std::to_string(lineno));
        }
    }
    fclose(fp);
    return QG_OK;
}

extern "C" int qg_run(const qg_config *cfg_in, const qg_run_options *o_in, qg_run_result *res)
{
    if (!cfg_in || !o_in || !res) return host_fail(QG_ERR_ARG, "null argument");
    memset(res, 0, sizeof(*res));
    res->verification_passed = -1;
    qg_config cfg = *cfg_in;
    qg_run_options opts = *o_in;
    const qg_run_options *o = &opts;
    const bool resume = (opts.init == 0);
    qg_run_state rs;
    memset(&rs, 0, sizeof(rs));
    int rc;
    if (resume) {
        // lattice_load_bin_header: the file's settings replace init.dat's
        if (!opts.state_file[0]) return host_fail(QG_ERR_ARG, "INIT = 0 needs STATEFILE");
        if ((rc = qg_read_state_file(opts.state_file, &cfg, &rs, nullptr, 0))) return rc;
        opts.nav = rs.nav;
        opts.niter = rs.niter;
        opts.iter = rs.iter;
        opts.pl_level = rs.pl_level;
        opts.get_actions = rs.get_actions;
        opts.get_plaquettes = rs.get_plaquettes;
        opts.get_wilson = rs.get_wilson;
        opts.fmunu = rs.fmunu;
        opts.fmunu_index1 = rs.fmunu_index1;
        opts.fmunu_index2 = rs.fmunu_index2;
        opts.get_actions_diff = rs.get_actions_diff;
    }
    if (o->iter < 1 || o->niter < 0 || o->nav < 0) return host_fail(QG_ERR_ARG, "ITER >= 1, NITER >= 0, NAV >= 0");
    // raw lattice sums per measured iteration, the reference's buffers
    std::vector<double> s_act(2 * (size_t)o->iter, 0.0), s_plq(2 * (size_t)o->iter, 0.0),
        s_wil((size_t)o->iter, 0.0), s_pol(4 * (size_t)o->iter, 0.0);
    rs.actions = s_act.data();
    rs.plaquettes = s_plq.data();
    rs.wilson = s_wil.data();
    rs.polyakov = s_pol.data();
    // F_munu sums (12 per iteration) and the profiles along x, y, z
    const size_t plen = 2 * (size_t)(cfg.size[0] + cfg.size[1] + cfg.size[2]);
    const size_t poff = o->pl_level > 2 ? plen : 0;                 // action profiles after Polyakov's
    const size_t prow = poff + (o->get_actions_diff ? plen : 0);
    std::vector<double> s_f(12 * (size_t)o->iter, 0.0), s_prof(prow * (size_t)o->iter + 1, 0.0);
    rs.fmunu_series = s_f.data();
    rs.profiles = s_prof.data();
    if (o->fmunu < 0 || o->fmunu > 2) return host_fail(QG_ERR_ARG, "fmunu must be 0 (off), 1 (FMUNU) or 2 (F0MU)");
    int fi1, fi2;
    fmunu_indices(cfg.group, *o, fi1, fi2);
    qg_ctx *ctx = nullptr;
    rc = qg_create(&cfg, &ctx);
    if (rc) return host_fail(rc, std::string("qg_create: ") + qg_last_error(nullptr));
    auto bail = [&](int code) {
        std::string m = qg_last_error(ctx);
        if (m.empty()) m = qg_last_error(nullptr);
        qg_destroy(ctx);
        return host_fail(code, m);
    };
    qg_info info;
    qg_get_info(ctx, &info);
    const size_t real = cfg.precision ? 8 : 4;
    const int N = cfg.group;
    const double V = info.sites;
    const double nsp = (double)cfg.size[0] * cfg.size[1] * cfg.size[2];
    // lattice_init: PRNG::initialize, then the start configuration -- or
    // the saved table, with the PRN stream brought to where it stopped
    if ((rc = qg_prng_seed(ctx, cfg.randseries))) return bail(rc);
    if (resume) {
        std::vector<char> table((size_t)info.ref_elems * real);
        if ((rc = qg_read_state_file(opts.state_file, &cfg, &rs, table.data(), (uint64_t)table.size()))) {
            qg_destroy(ctx);
            return rc;
        }
        if ((rc = qg_links_upload(ctx, table.data(), QG_LAYOUT_REFERENCE))) return bail(rc);
        if (cfg.prng == QG_PRNG_RANLUX) {
            for (;;) {                                  // suncl.cpp:5349-5351
                qg_get_info(ctx, &info);
                if (info.prng_counter >= rs.prng_counter) break;
                if ((rc = qg_prng_produce(ctx))) return bail(rc);
            }
        } else if ((rc = qg_set_phase_counter(ctx, rs.phase_counter))) {
            return bail(rc);
        }
        if ((rc = qg_set_sweeps_done(ctx, rs.sweeps_done))) return bail(rc);
    } else {
        if ((rc = qg_init_links(ctx, cfg.start))) return bail(rc);
        rs.init = 1;
        rs.nav = o->nav;
        rs.niter = o->niter;
        rs.iter = o->iter;
        rs.pl_level = o->pl_level;
        rs.get_actions = o->get_actions;
        rs.get_plaquettes = o->get_plaquettes;
        rs.get_wilson = o->get_wilson;
        rs.fmunu = o->fmunu;
        rs.fmunu_index1 = fi1;
        rs.fmunu_index2 = fi2;
        rs.get_actions_diff = o->get_actions_diff;
    }
    // launch shapes for this lattice (field restored, PRN counters untouched)
    if (o->tune_shapes && (rc = qg_tune(ctx, 4, nullptr))) return bail(rc);
    time_t t_start = time(nullptr);
    // one measurement per kind of site work: plaquette, action and the
    // action profiles from one pass (qg_measure_plaquette_all), the Polyakov
    // loop and its profiles from another -- the same numbers as the separate
    // qg_measure / qg_measure_*_profile calls
    std::vector<double> all(4 + plen);
    auto measure = [&](int i) -> int {
        double a[4];
        int r;
        const size_t prof_row = prow * (size_t)i;
        if (o->get_plaquettes || o->get_actions || o->get_actions_diff) {
            if (o->get_actions || o->get_actions_diff) {
                if ((r = qg_measure_plaquette_all(ctx, all.data()))) return r;
                memcpy(a, all.data(), sizeof(a));
                if (o->get_actions_diff) memcpy(&s_prof[prof_row + poff], all.data() + 4, plen * sizeof(double));
            } else if ((r = qg_measure(ctx, QG_MEAS_PLAQUETTE, a))) {
                return r;
            }
            if (o->get_plaquettes) { s_plq[2 * i] = a[0]; s_plq[2 * i + 1] = a[1]; }
            if (o->get_actions) { s_act[2 * i] = a[2]; s_act[2 * i + 1] = a[3]; }
        }
        if (o->get_wilson) {
            if ((r = qg_measure(ctx, QG_MEAS_WILSON, a))) return r;
            s_wil[i] = a[0];
        }
        if (o->pl_level > 2) {
            if ((r = qg_measure_polyakov_all(ctx, all.data()))) return r;
            for (int k = 0; k < 4; k++) s_pol[4 * i + k] = all[k];
            memcpy(&s_prof[prof_row], all.data() + 4, plen * sizeof(double));
        } else if (o->pl_level > 0) {
            if ((r = qg_measure(ctx, QG_MEAS_POLYAKOV, a))) return r;
            for (int k = 0; k < 4; k++) s_pol[4 * i + k] = a[k];
        }
        if (o->fmunu && (r = qg_measure_fmunu(ctx, o->fmunu - 1, fi1, fi2, &s_f[12 * (size_t)i]))) return r;
        return QG_OK;
    };
    // lattice_save_state: the name the reference gives it, or STATEOUT
    auto save = [&]() -> int {
        char name[640];
        if (o->state_out[0]) {
            snprintf(name, sizeof(name), "%s", o->state_out);
        } else {
            time_t now = time(nullptr);
            char tb[64];
            snprintf(tb, sizeof(tb), "%s", ctime(&now));
            snprintf(name, sizeof(name), "%s%s%.2s-%.3s-%.2s-%.2s-%.2s-%.2s.qcg", o->output_path, o->prefix, tb + 22,
                     tb + 4, tb + 8, tb + 11, tb + 14, tb + 17);
        }
        int r = qg_save_state(ctx, name, &rs);
        if (r == QG_OK) snprintf(res->state_file, sizeof(res->state_file), "%s", name);
        return r;
    };
    auto t0 = std::chrono::steady_clock::now();
    if (!resume) {
        if ((rc = measure(0))) return bail(rc);                  // iteration 0: start configuration
        rs.iter_counter = 1;
        if (o->save_state && (rc = save())) return bail(rc);
    }
    const int nav_start = rs.nav_counter;
    if (rs.nav_counter < o->nav) {                                // thermalisation
        if ((rc = qg_sweep(ctx, o->nav - rs.nav_counter))) return bail(rc);
        rs.nav_counter = o->nav;
    }
    const int first = rs.iter_counter;
    for (int i = first; i < o->iter; i++) {
        if ((rc = qg_sweep(ctx, o->niter))) return bail(rc);
        if ((rc = measure(i))) return bail(rc);
        rs.iter_counter = i + 1;
        if (o->save_every_iter > 0 && rs.iter_counter % o->save_every_iter == 0 && rs.iter_counter < o->iter &&
            (rc = save()))
            return bail(rc);
        if (!o->quiet && i % 10 == 0) { printf("\rGPU working iteration [%d]", i); fflush(stdout); }
    }
    if ((rc = qg_sync(ctx))) return bail(rc);
    if (o->save_state && (rc = save())) return bail(rc);
    auto t1 = std::chrono::steady_clock::now();
    time_t t_end = time(nullptr);
    res->seconds = std::chrono::duration<double>(t1 - t0).count();
    const double sweeps = (double)(o->nav - nav_start) + (double)(o->iter - first) * o->niter;
    res->link_updates_per_second = res->seconds > 0 ? 4.0 * V * sweeps * (1 + cfg.n_or) / res->seconds : 0.0;
    res->samples = o->iter;
    // lattice_analysis: normalised series (suncl.cpp:1328-1612)
    std::vector<double> d[QG_OBS_COUNT];
    for (int i = 0; i < o->iter; i++) {
        if (o->get_plaquettes) {
            d[QG_OBS_PLQ_SPAT].push_back(s_plq[2 * i] / (3 * V));
            d[QG_OBS_PLQ_TEMP].push_back(s_plq[2 * i + 1] / (3 * V));
            d[QG_OBS_PLQ_TOTAL].push_back(0.5 * (s_plq[2 * i] + s_plq[2 * i + 1]) / (3 * V));
        }
        if (o->get_wilson) d[QG_OBS_WILSON].push_back(s_wil[i] / (3 * V));
        if (o->get_actions) {
            d[QG_OBS_S_SPAT].push_back(s_act[2 * i] / (3 * V));
            d[QG_OBS_S_TEMP].push_back(s_act[2 * i + 1] / (3 * V));
            d[QG_OBS_S_TOTAL].push_back(0.5 * (s_act[2 * i] + s_act[2 * i + 1]) / (3 * V));
        }
        if (o->pl_level > 0) {
            d[QG_OBS_POLYAKOV].push_back(s_pol[4 * i] / (nsp * N));
            d[QG_OBS_POLYAKOV_IM].push_back(s_pol[4 * i + 1] / (nsp * N));
            if (o->pl_level > 1) {
                d[QG_OBS_POLYAKOV_P2].push_back(s_pol[4 * i + 2] / (nsp * N * N));
                d[QG_OBS_POLYAKOV_P4].push_back(s_pol[4 * i + 3] / (nsp * N * N * N * N));
            }
        }
    }
    for (int k = 0; k < QG_OBS_COUNT; k++) {
        if (d[k].empty()) continue;
        mean_var(d[k], res->mean[k], res->variance[k]);
        res->gpu_last[k] = d[k].back();
        // tau_int and the error of the mean over samples 1..ITER-1
        const int n = (int)d[k].size() - 1;
        int w = 0;
        res->tau_int[k] = 0.5;
        if (n > 1) qg_tau_int(d[k].data() + 1, n, 6.0, &res->tau_int[k], &w);
        res->error[k] = n > 0 ? sqrt(2.0 * res->tau_int[k] * res->variance[k] / n) : 0.0;
    }
    // the 16 F_munu columns (lattice_make_header2, suncl.cpp:1613-1670):
    // planes of index1, planes of index2 (Re, Im), then |F| per generator
    // (data_analysis_joint3: sqrt of the sum of squares over the planes)
    auto fmunu_row = [&](const double *f, double *row) {
        for (int k = 0; k < 12; k++) row[k] = f[k] / V;
        for (int g = 0; g < 2; g++)
            for (int ri = 0; ri < 2; ri++) {
                double q = 0;
                for (int p = 0; p < 3; p++) q += row[6 * g + 2 * p + ri] * row[6 * g + 2 * p + ri];
                row[12 + 2 * g + ri] = sqrt(q);
            }
    };
    std::vector<double> fd[QG_FMUNU_COLS];
    if (o->fmunu) {
        for (int i = 0; i < o->iter; i++) {
            double row[QG_FMUNU_COLS];
            fmunu_row(&s_f[12 * (size_t)i], row);
            for (int k = 0; k < QG_FMUNU_COLS; k++) fd[k].push_back(row[k]);
        }
        for (int k = 0; k < QG_FMUNU_COLS; k++) {
            mean_var(fd[k], res->fmunu_mean[k], res->fmunu_variance[k]);
            res->fmunu_gpu_last[k] = fd[k].back();
        }
    }
    // profiles (lattice_analysis_PL_diff / _Action_diff and their
    // normalisations, suncl.cpp:1116-1260,1376-1612): per slice the mean and
    // variance over samples 1..ITER-1 of the Polyakov loop (Re, Im, per
    // spatial site / N) and of the total action (per plaquette)
    struct Slice { double pl, pl_im, pl_var, pl_im_var, s, s_var; };
    std::vector<Slice> prof[3];
    for (int axis = 0; axis < 3; axis++) {
        const int na = cfg.size[axis];
        prof[axis].assign(na, Slice{ 0, 0, 0, 0, 0, 0 });
        size_t aoff = 0;
        for (int b = 0; b < axis; b++) aoff += 2 * (size_t)cfg.size[b];
        for (int k = 0; k < na; k++) {
            std::vector<double> re, im, st;
            for (int i = 0; i < o->iter; i++) {
                const double *row = &s_prof[prow * (size_t)i];
                if (o->pl_level > 2) {
                    re.push_back(row[aoff + 2 * k] / (N * nsp / na));
                    im.push_back(row[aoff + 2 * k + 1] / (N * nsp / na));
                }
                if (o->get_actions_diff)
                    st.push_back(0.5 * (row[poff + aoff + 2 * k] + row[poff + aoff + 2 * k + 1]) / (3.0 * V / na));
            }
            Slice &sl = prof[axis][k];
            if (!re.empty()) { mean_var(re, sl.pl, sl.pl_var); mean_var(im, sl.pl_im, sl.pl_im_var); }
            if (!st.empty()) mean_var(st, sl.s, sl.s_var);
        }
    }
    if (o->profile) {   // the per-kernel table (GPU_debug.profiling, print_time_detailed)
        if ((rc = qg_profile_kernels(ctx, 20, res->kernel_ms, res->kernel_ms_sigma))) return bail(rc);
        if (!o->quiet) {
            static const char *names[QG_KERNEL_CLASSES] = { "heatbath phase", "overrelaxation phase",
                                                            "Gram-Schmidt", "plaquette + action",
                                                            "Polyakov loop", "Wilson loop" };
            printf("\n kernel                   ms per launch (20 launches)\n");
            for (int k = 0; k < QG_KERNEL_CLASSES; k++)
                printf(" %-22s %10.5f +- %.5f\n", names[k], res->kernel_ms[k], res->kernel_ms_sigma[k]);
        }
    }
    {   // the final configuration is finite and in SU(N) (a NaN or a broken
        // link would otherwise only show as odd averages)
        uint64_t bad = 0;
        if ((rc = qg_field_check(ctx, cfg.precision ? 1e-9 : 1e-3, &bad))) return bail(rc);
        if (bad) {
            qg_destroy(ctx);
            return host_fail(QG_ERR_NUMERIC, std::to_string(bad) + " links of the final configuration are not "
                                             "finite or not in SU(N)");
        }
    }
    // LatticeCheckCPU: FP64 re-measurement of the final configuration
    double f_varnc[12] = { 0 };
    char platform[64] = "", device[128] = "";
    if ((rc = qg_device_info(platform, sizeof(platform), device, sizeof(device)))) return bail(rc);
    if (o->verify) {
        std::vector<char> buf(info.ref_elems * (cfg.precision ? 8 : 4));
        if ((rc = qg_links_download(ctx, buf.data(), QG_LAYOUT_REFERENCE))) return bail(rc);
        Table T;
        T.group = N; memcpy(T.n, cfg.size, sizeof(T.n)); T.prec = cfg.precision; T.rowsize = info.rowsize;
        T.p = buf.data();
        HostObs h = host_measure(T, cfg, *o);
        res->cpu_last[QG_OBS_PLQ_SPAT] = h.plq_s / (3 * V);
        res->cpu_last[QG_OBS_PLQ_TEMP] = h.plq_t / (3 * V);
        res->cpu_last[QG_OBS_PLQ_TOTAL] = 0.5 * (h.plq_s + h.plq_t) / (3 * V);
        res->cpu_last[QG_OBS_S_SPAT] = h.s_s / (3 * V);
        res->cpu_last[QG_OBS_S_TEMP] = h.s_t / (3 * V);
        res->cpu_last[QG_OBS_S_TOTAL] = 0.5 * (h.s_s + h.s_t) / (3 * V);
        res->cpu_last[QG_OBS_POLYAKOV] = h.pre / (nsp * N);
        res->cpu_last[QG_OBS_POLYAKOV_IM] = h.pim / (nsp * N);
        res->cpu_last[QG_OBS_POLYAKOV_P2] = h.p2 / (nsp * N * N);
        res->cpu_last[QG_OBS_POLYAKOV_P4] = h.p4 / (nsp * N * N * N * N);
        res->cpu_last[QG_OBS_WILSON] = h.wilson / (3 * V);
        bool ok = true;
        for (int k = 0; k < QG_OBS_COUNT; k++)
            if (!d[k].empty()) ok = verify(res->gpu_last[k], res->cpu_last[k], cfg.precision == 0) && ok;
        if (o->fmunu) {
            fmunu_row(h.f, res->fmunu_cpu_last);
            for (int k = 0; k < QG_FMUNU_COLS; k++)
                ok = verify(res->fmunu_gpu_last[k], res->fmunu_cpu_last[k], cfg.precision == 0) && ok;
            // the lattice variance of each projection on the final configuration
            // (the "CPU l.varnc" lines; su3cpu.cpp:1367-1378)
            for (int k = 0; k < 12; k++) f_varnc[k] = h.f2[k] / V - (h.f[k] / V) * (h.f[k] / V);
        }
        res->verification_passed = ok ? 1 : 0;
    }
    qg_destroy(ctx);
    // the results file (lattice_write_results, suncl.cpp:1679-1854) and the
    // companion statistics file (qg_results.cpp)
    if (o->write_results) {
        const size_t it = (size_t)o->iter;
        std::vector<double> ser(QG_OBS_COUNT * it, 0.0), fser(o->fmunu ? QG_FMUNU_COLS * it : 0, 0.0);
        for (int k = 0; k < QG_OBS_COUNT; k++)
            for (size_t i = 0; i < d[k].size() && i < it; i++) ser[k * it + i] = d[k][i];
        for (int k = 0; k < QG_FMUNU_COLS && o->fmunu; k++)
            for (size_t i = 0; i < fd[k].size() && i < it; i++) fser[k * it + i] = fd[k][i];
        std::vector<double> pr;
        for (int a = 0; a < 3; a++)
            for (const Slice &q : prof[a]) {
                const double v[6] = { q.pl, q.pl_im, q.pl_var, q.pl_im_var, q.s, q.s_var };
                pr.insert(pr.end(), v, v + 6);
            }
        if ((rc = qg_write_results(&cfg, o, res, resume ? 1 : 0, ser.data(), o->fmunu ? fser.data() : nullptr,
                                   pr.data(), o->fmunu && o->verify ? f_varnc : nullptr, (int64_t)t_start,
                                   (int64_t)t_end, platform, device, res->results_file, sizeof(res->results_file))))
            return rc;
    }
    if (!o->quiet) {
        printf("\n #        ");
        printf(" Plq_spat    Plq_temp    S_spat      S_temp\n");
        for (int i = 0; i < o->iter && o->get_plaquettes && o->get_actions; i++)
            printf("[%5d]:   %.8f  %.8f  %.8f  %.8f\n", i, d[QG_OBS_PLQ_SPAT][i], d[QG_OBS_PLQ_TEMP][i],
                   d[QG_OBS_S_SPAT][i], d[QG_OBS_S_TEMP][i]);
        if (res->verification_passed >= 0)
            printf("%s\n", res->verification_passed ? "Verification successfully passed!" : "Verification failed!");
    }
    return QG_OK;
}
