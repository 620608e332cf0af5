// qg_results.cpp -- the run's results file in the reference's layout
// (model::lattice_write_results with lattice_make_header, model_make_header
// and lattice_make_header2, SU(N)/suncl/suncl.cpp:534-615, 779-865,
// 1679-1854), and a companion file with what this library adds.
//
// Host code only (no CUDA).  Sections, labels, column widths and their
// order follow the reference's GPU build: the header with the run
// parameters and the device, start / finish / elapsed time, mean and
// variance of the 7 observables, the F_munu blocks (means, variances,
// GPU / CPU last values, the CPU lattice variances) -- always present, zero
// when F_munu is not measured, as the reference prints them -- the CPU /
// GPU last values of the observables and the verification line, the
// Polyakov-loop and action profile sections, and the data rows.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "qcdgpu_b200.h"

void qg_set_global_error(const std::string &m);

namespace {

const char *kVersion = "1.0";
const char *kStars = " ***************************************************\n";
const char *kObsNames[QG_OBS_COUNT] = { "S_total", "Plq_total", "Polyakov_loop", "Polyakov_loop_im",
                                        "Polyakov_loop_P2", "Polyakov_loop_P4", "Wilson_loop",
                                        "Plq_spat", "Plq_temp", "S_spat", "S_temp" };

int fail(int code, const std::string &m)
{
    qg_set_global_error(m);
    return code;
}

// the generator line(s) of PRNG::print_generator (random/random.cpp:156-172)
void print_generator(FILE *fp, const qg_config &c)
{
    fprintf(fp, " random series               : %u\n", c.randseries);
    if (c.prng == QG_PRNG_RANLUX) {
        const int lux = c.ranlux_nskip == 24 ? 0 : c.ranlux_nskip == 48 ? 1 : c.ranlux_nskip == 97 ? 2
                      : c.ranlux_nskip == 223 ? 3 : c.ranlux_nskip == 389 ? 4 : -1;
        if (lux >= 0) fprintf(fp, " PRN generator               : RANLUX%d\n", lux);
        else fprintf(fp, " PRN generator (%3u)         : RANLUX\n", (unsigned)c.ranlux_nskip);
    } else {
        fprintf(fp, " PRN generator               : PHILOX4x32-10\n");
    }
}

}  // namespace

extern "C" int qg_write_results(const qg_config *cfgp, const qg_run_options *op, const qg_run_result *res,
                                int resumed, const double *series, const double *fmunu, const double *profiles,
                                const double *fmunu_cpu_lattice_variance, int64_t t_start, int64_t t_end,
                                const char *platform, const char *device, char *path, size_t path_len)
{
    if (!cfgp || !op || !res || !series || !path || path_len < 2) return fail(QG_ERR_ARG, "qg_write_results: null argument");
    const qg_config &cfg = *cfgp;
    const qg_run_options &o = *op;
    const int N = cfg.group, iter = o.iter;
    if (iter < 1) return fail(QG_ERR_ARG, "qg_write_results: ITER >= 1");
    if (o.fmunu && !fmunu) return fail(QG_ERR_ARG, "qg_write_results: F_munu series missing");
    if ((o.pl_level > 2 || o.get_actions_diff) && !profiles)
        return fail(QG_ERR_ARG, "qg_write_results: profiles missing");
    // the file name of lattice_write_results: prefix + "YY-Mon-DD-hh-mm-ss.txt"
    // from ctime of the finish time
    const time_t ts = (time_t)t_start, te = (time_t)t_end;
    char cs[64] = "", ce[64] = "";
    if (!ctime_r(&ts, cs) || !ctime_r(&te, ce)) return fail(QG_ERR_ARG, "qg_write_results: bad start or end time");
    char stamp[96];
    snprintf(stamp, sizeof(stamp), "%.2s-%.3s-%.2s-%.2s-%.2s-%.2s", ce + 22, ce + 4, ce + 8, ce + 11, ce + 14, ce + 17);
    const std::string name = std::string(o.output_path) + o.prefix + stamp;
    if (name.size() + 5 > path_len) return fail(QG_ERR_ARG, "qg_write_results: path buffer too small");
    snprintf(path, path_len, "%s.txt", name.c_str());
    FILE *fp = fopen(path, "w");
    if (!fp) return fail(QG_ERR_IO, std::string("cannot write ") + path);

    // F_munu column names (suncl.h:235-252 order) for the generators in use
    int fi1 = o.fmunu_index1, fi2 = o.fmunu_index2;
    if (N == 3) {
        if (fi1 != 1 && fi1 != 2 && fi1 != 4) fi1 = 3;
        if (fi2 < 5 || fi2 > 7) fi2 = 8;
    } else {
        if (fi1 != 1) fi1 = 3;
        fi2 = 2;
    }
    char fnames[QG_FMUNU_COLS][24];
    {
        static const char *xyz = "xyz";
        static const int hp[3][2] = { { 0, 1 }, { 0, 2 }, { 1, 2 } };
        for (int k = 0; k < 12; k++) {
            const int p = (k % 6) / 2, idx = k < 6 ? fi1 : fi2;
            const char *ri = (k & 1) ? "im" : "re";
            if (o.fmunu == 2) snprintf(fnames[k], 24, "Fmunu_%ct_%u_%s", xyz[p], idx, ri);
            else snprintf(fnames[k], 24, "Fmunu_%c%c_%u_%s", xyz[hp[p][0]], xyz[hp[p][1]], idx, ri);
        }
        for (int k = 12; k < QG_FMUNU_COLS; k++)
            snprintf(fnames[k], 24, "Fmunu_abs_%1u_%s", k < 14 ? fi1 : fi2, (k & 1) ? "im" : "re");
    }

    // lattice_make_header (GPU build) and model_make_header
    fprintf(fp, " GPU SU(%u) simulator %s (qcdgpu_b200)\n\n", (unsigned)N, kVersion);
    fprintf(fp, " Monte Carlo simulation of 4D SU(%u) LGT\n\n", (unsigned)N);
    fprintf(fp, "%s", kStars);
    fprintf(fp, " Active CUDA platform     : %s\n", platform ? platform : "");
    fprintf(fp, " Active CUDA device       : %s\n", device ? device : "");
    fprintf(fp, "%s", kStars);
    fprintf(fp, " lattice size                : %3u x %3u x %3u x %3u\n", (unsigned)cfg.size[0], (unsigned)cfg.size[1],
            (unsigned)cfg.size[2], (unsigned)cfg.size[3]);
    fprintf(fp, " init                        : %i\n", resumed ? 0 : 1);
    fprintf(fp, " ints (0=hot, 1=cold, 2=gid) : %d\n",
            cfg.start == QG_START_COLD ? 1 : cfg.start == QG_START_GID ? 2 : 0);
    print_generator(fp, cfg);
    fprintf(fp, " nav                         : %i\n", o.nav);
    fprintf(fp, " niter                       : %i\n", o.niter);
    fprintf(fp, " iter (# of samples)         : %i\n", o.iter);
    fprintf(fp, " nhit                        : %i\n", cfg.nhit);
    fprintf(fp, " nhitPar                     : %i\n", cfg.nhitpar);
    fprintf(fp, " precision                   : %s\n", cfg.precision ? "double" : "single");
    fprintf(fp, "%s", kStars);
    fprintf(fp, " Wilson loop R               : %i\n", cfg.wilson_r);
    fprintf(fp, " Wilson loop T               : %i\n", cfg.wilson_t);
    if (o.fmunu == 1) fprintf(fp, " FMUNU(%u, %u)\n", (unsigned)fi1, (unsigned)fi2);
    if (o.fmunu == 2) fprintf(fp, " F0MU(%u, %u)\n", (unsigned)fi1, (unsigned)fi2);
    fprintf(fp, " BETA                        : %16.13e\n", cfg.beta);
    fprintf(fp, " PHI   (lambda_3)            : %16.13e\n", cfg.phi);
    fprintf(fp, " OMEGA (lambda_8)            : %16.13e\n", cfg.omega);
    fprintf(fp, "%s", kStars);

    // lattice_make_header2
    const int el = (int)difftime(te, ts);
    fprintf(fp, " Start time               : %s", cs);
    fprintf(fp, " Finish time              : %s", ce);
    // days:hours:minutes:seconds (hours modulo 24; the reference's formula,
    // suncl.cpp:805, keeps counting hours past the first day)
    fprintf(fp, " Elapsed time             : %i:%2.2i:%2.2i:%2.2i\n", el / 86400, (el / 3600) % 24, (el / 60) % 60,
            el % 60);
    fprintf(fp, "%s", kStars);
    for (int k = 0; k <= QG_OBS_WILSON; k++) {
        fprintf(fp, " Mean %-20s: % 16.13e\n", kObsNames[k], res->mean[k]);
        fprintf(fp, " Variance %-16s: % 16.13e\n", kObsNames[k], res->variance[k]);
    }
    fprintf(fp, "%s", kStars);
    for (int k = 0; k < QG_FMUNU_COLS; k++) fprintf(fp, " Mean %-20s: % 16.13e\n", fnames[k], res->fmunu_mean[k]);
    for (int k = 0; k < QG_FMUNU_COLS; k++) fprintf(fp, " Variance %-16s: % 16.13e\n", fnames[k], res->fmunu_variance[k]);
    fprintf(fp, "%s", kStars);
    for (int k = 0; k < QG_FMUNU_COLS; k++) {
        fprintf(fp, " GPU last %-16s: % 16.13e\n", fnames[k], res->fmunu_gpu_last[k]);
        fprintf(fp, " CPU last %-16s: % 16.13e\n", fnames[k], res->fmunu_cpu_last[k]);
    }
    fprintf(fp, "%s", kStars);
    for (int k = 0; k < 12; k++)
        fprintf(fp, " CPU l.varnc %-13s: % 16.13e\n", fnames[k],
                fmunu_cpu_lattice_variance ? fmunu_cpu_lattice_variance[k] : 0.0);
    fprintf(fp, "%s", kStars);
    for (int k = 0; k <= QG_OBS_WILSON; k++) {
        fprintf(fp, " CPU last %-16s: % 16.13e\n", kObsNames[k], res->cpu_last[k]);
        fprintf(fp, " GPU last %-16s: % 16.13e\n", kObsNames[k], res->gpu_last[k]);
    }
    if (res->verification_passed == 1) fprintf(fp, " *** Verification successfully passed! *************\n");
    else if (res->verification_passed == 0) fprintf(fp, " --- Verification failed! --------------------------\n");
    else fprintf(fp, " --- Verification not run --------------------------\n");

    // profile sections
    static const char *axis_name[3] = { "X", "Y", "Z" };
    auto prof = [&](int axis, int slice, int q) {
        size_t off = 0;
        for (int a = 0; a < axis; a++) off += (size_t)cfg.size[a];
        return profiles[6 * (off + (size_t)slice) + q];
    };
    if (o.pl_level > 2) {
        fprintf(fp, "%s", kStars);
        fprintf(fp, "Differentiated Polyakov loop data (#, PL, PL_im, PL_variance, PL_im_variance):\n");
        static const char *rows[4] = { "PL             ", "PL_im          ", "PL_variance    ", "PL_im_variance " };
        static const int qs[4] = { 0, 1, 2, 3 };
        for (int a = 0; a < 3; a++) {
            fprintf(fp, "\n%s              ", axis_name[a]);
            for (int k = 0; k < cfg.size[a]; k++) fprintf(fp, "%2u                   ", (unsigned)k);
            for (int r = 0; r < 4; r++) {
                fprintf(fp, "\n%s", rows[r]);
                for (int k = 0; k < cfg.size[a]; k++) fprintf(fp, "% 16.13e ", prof(a, k, qs[r]));
            }
            fprintf(fp, "\n");
        }
    }
    if (o.get_actions_diff) {
        fprintf(fp, "%s", kStars);
        fprintf(fp, "Differentiated S data (#, S_total, S_variance):\n");
        for (int a = 0; a < 3; a++) {
            fprintf(fp, "\n%s              ", axis_name[a]);
            for (int k = 0; k < cfg.size[a]; k++) fprintf(fp, "%2u                   ", (unsigned)k);
            fprintf(fp, "\nS             ");
            for (int k = 0; k < cfg.size[a]; k++) fprintf(fp, "% 16.13e ", prof(a, k, 4));
            fprintf(fp, "\nS_variance    ");
            for (int k = 0; k < cfg.size[a]; k++) fprintf(fp, "% 16.13e ", prof(a, k, 5));
            fprintf(fp, "\n");
        }
    }

    // data rows
    fprintf(fp, "%s", kStars);
    fprintf(fp, " Data fields:\n    #,  ");
    std::vector<int> cols;
    if (o.get_plaquettes) { cols.push_back(QG_OBS_PLQ_SPAT); cols.push_back(QG_OBS_PLQ_TEMP); cols.push_back(QG_OBS_PLQ_TOTAL); }
    if (o.get_wilson) cols.push_back(QG_OBS_WILSON);
    if (o.get_actions) { cols.push_back(QG_OBS_S_SPAT); cols.push_back(QG_OBS_S_TEMP); cols.push_back(QG_OBS_S_TOTAL); }
    if (o.pl_level > 0) { cols.push_back(QG_OBS_POLYAKOV); cols.push_back(QG_OBS_POLYAKOV_IM); }
    if (o.pl_level > 1) { cols.push_back(QG_OBS_POLYAKOV_P2); cols.push_back(QG_OBS_POLYAKOV_P4); }
    for (int k : cols) fprintf(fp, "%-21s ", kObsNames[k]);
    if (o.fmunu)
        for (int k = 0; k < QG_FMUNU_COLS; k++) fprintf(fp, "%-21s ", fnames[k]);
    fprintf(fp, "\n%s", kStars);
    for (int i = 0; i < iter; i++) {
        fprintf(fp, "%5i", i);
        for (int k : cols) fprintf(fp, " % 16.13e", series[(size_t)k * iter + i]);
        if (o.fmunu)
            for (int k = 0; k < QG_FMUNU_COLS; k++) fprintf(fp, " % 16.13e", fmunu[(size_t)k * iter + i]);
        fprintf(fp, "\n");
    }
    if (fclose(fp) != 0) return fail(QG_ERR_IO, std::string("cannot close ") + path);

    // what this library adds: tau_int and the error of each mean, and the
    // run settings the reference's header has no line for
    const std::string stats = name + "-stats.txt";
    fp = fopen(stats.c_str(), "w");
    if (!fp) return fail(QG_ERR_IO, "cannot write " + stats);
    fprintf(fp, " qcdgpu_b200 %s: statistics and settings beside %s\n", kVersion, path);
    fprintf(fp, "%s", kStars);
    fprintf(fp, " overrelaxation sweeps       : %d\n", cfg.n_or);
    fprintf(fp, " reunitarisation every       : %d%s\n", cfg.reunit_every, cfg.reunit_fp64 ? " (FP64)" : "");
    fprintf(fp, " PRN instances               : %d\n", cfg.prng == QG_PRNG_RANLUX ? cfg.prng_instances : 0);
    fprintf(fp, " link updates per second     : % 16.13e\n", res->link_updates_per_second);
    fprintf(fp, "%s", kStars);
    for (int k = 0; k <= QG_OBS_WILSON; k++) {
        fprintf(fp, " Tau_int %-17s: % 16.13e\n", kObsNames[k], res->tau_int[k]);
        fprintf(fp, " Error %-19s: % 16.13e\n", kObsNames[k], res->error[k]);
    }
    if (fclose(fp) != 0) return fail(QG_ERR_IO, "cannot close " + stats);
    return QG_OK;
}
