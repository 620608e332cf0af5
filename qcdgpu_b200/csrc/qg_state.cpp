// qg_state.cpp -- lattice state files (.qcg) and the integrated
// autocorrelation time of a measured series.
//
// The state file restates the reference's binary format
// (model::lattice_save_state / lattice_make_bin_header /
// lattice_load_bin_header / lattice_load_state, SU(N)/suncl/suncl.cpp:
// 1857-2079): 64 little-endian uint32 header words, the measurement
// buffers, then the link table in the reference layout.  The word order,
// the code tables (start, generator, precision) and the buffer order follow
// the reference so that files interchange; header words 48-59 and a tagged
// block after the link table carry what this library adds (Philox counter,
// overrelaxation and reunitarisation settings, |P|^2 and |P|^4 series).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/qcdgpu_b200.h"

void qg_set_global_error(const std::string &m);   // qg_capi.cu: qg_last_error(NULL)

namespace {

int st_fail(int code, const std::string &m)
{
    qg_set_global_error(m);
    return code;
}

// model::convert_str_uint: four characters of s from `off`, little-endian
uint32_t str_word(const char *s, size_t off)
{
    uint32_t r = 0;
    const size_t n = strlen(s);
    for (unsigned i = 0; i < 4; i++)
        if (off + i < n) r |= (uint32_t)(unsigned char)s[off + i] << (8 * i);
    return r;
}

const char *kPrefix = "QCDGPU";
const char *kVersion = "1.5";                // QCDGPU.cpp:42, the version the reference writes
const char *kExtTag = "B200";                // marks this library's header words 48-59
const char *kTailTag = "QGP4";               // tagged |P|^2, |P|^4 block after the table
const char *kProfTag = "QGPF";               // tagged block of the per-iteration profiles after it

// header word indices (lattice_make_bin_header order)
enum {
    W_INIT = 4, W_INTS, W_SERIES, W_GEN, W_NSKIP, W_PRNG_COUNTER, W_NAV, W_NAV_COUNTER, W_NITER, W_ITER,
    W_ITER_COUNTER, W_NHIT, W_WILSON_R, W_WILSON_T, W_PRECISION, W_BETA_LO, W_BETA_HI, W_PHI_LO, W_PHI_HI,
    W_OMEGA_LO, W_OMEGA_HI, W_PL_LEVEL, W_FMUNU1, W_FMUNU2, W_GET_FMUNU, W_GET_ACTIONS, W_GET_PLAQUETTES,
    W_GET_WILSON, W_MEAS_SIZE_F, W_ENERGIES_SIZE, W_ENERGIES_SIZE_F, W_POLYAKOV_SIZE, W_GROUP, W_ND,
    W_FULL_SIZE, W_DOMAIN_SIZE = W_FULL_SIZE + 4,
    // this library
    W_EXT_TAG = 48, W_PRNG_KIND, W_PHASE_LO, W_PHASE_HI, W_SWEEPS_LO, W_SWEEPS_HI, W_NOR, W_REUNIT_EVERY,
    W_REUNIT_FP64, W_NHITPAR, W_INSTANCES, W_ROW_ALIGN, W_FMUNU_KIND, W_ACTIONS_DIFF
};

// PRNG::convert_generator_to_uint (random.cpp:110-123): RANLUX0..4 = 2..6;
// the counter-based stream of this library gets 12, a code the reference
// does not use
uint32_t generator_code(const qg_config &c)
{
    if (c.prng == QG_PRNG_PHILOX) return 12;
    switch (c.ranlux_nskip) {
    case 24: return 2;
    case 48: return 3;
    case 97: return 4;
    case 223: return 5;
    case 389: return 6;
    default: return 7;                        // RANLUX with a custom skip
    }
}

uint32_t lo_word(double v) { uint64_t u; memcpy(&u, &v, 8); return (uint32_t)u; }
uint32_t hi_word(double v) { uint64_t u; memcpy(&u, &v, 8); return (uint32_t)(u >> 32); }
double from_words(uint32_t lo, uint32_t hi) { uint64_t u = ((uint64_t)hi << 32) | lo; double v; memcpy(&v, &u, 8); return v; }

uint32_t align_up(uint64_t n, uint32_t a) { return (uint32_t)(((n + a - 1) / a) * a); }

struct Sizes {
    uint32_t meas_F, energies, energies_F, polyakov;
};

// buffer sizes as lattice_create_buffers computes them (suncl.cpp:2266-2291),
// with the alignment of this library's ROWSIZE in place of the device's
// work-group size
Sizes sizes_for(const qg_config &c, int iter)
{
    const uint32_t a = c.row_align > 0 ? (uint32_t)c.row_align : 64;
    const uint64_t V = (uint64_t)c.size[0] * c.size[1] * c.size[2] * c.size[3];
    Sizes s;
    s.energies = align_up((uint64_t)(iter > 0 ? iter : 1), a);
    s.energies_F = s.energies * 7;             // MODEL_energies_size: plaquettes + 6 F_munu series
    s.meas_F = align_up((V + 255) / 256, a);
    s.polyakov = s.energies;
    return s;
}

uint64_t table_float4s(const qg_config &c)
{
    const uint32_t a = c.row_align > 0 ? (uint32_t)c.row_align : 64;
    const uint64_t V = (uint64_t)c.size[0] * c.size[1] * c.size[2] * c.size[3];
    const uint64_t rowsize = ((V + a - 1) / a) * a;
    return rowsize * 4 * (c.group == 3 ? 12 : 4) / 4;
}

}  // namespace

extern "C" int qg_write_state_file(const char *path, const qg_config *cfg, const qg_run_state *st,
                                   const void *links, uint64_t links_bytes)
{
    if (!path || !cfg || !st || !links) return st_fail(QG_ERR_ARG, "qg_write_state_file: null argument");
    const qg_config &c = *cfg;
    const size_t real = c.precision ? 8 : 4;
    const uint64_t nq = table_float4s(c);
    if (links_bytes != nq * 4 * real)
        return st_fail(QG_ERR_ARG, "qg_write_state_file: link table of " + std::to_string(links_bytes) +
                                       " bytes, expected " + std::to_string(nq * 4 * real));
    const Sizes z = sizes_for(c, st->iter);
    uint32_t h[QCDGPU_STATE_HEADER_WORDS] = {};
    h[0] = str_word(kPrefix, 0);
    h[1] = str_word(kPrefix, 4);
    h[2] = str_word(kVersion, 0);
    h[W_INIT] = (uint32_t)st->init;
    h[W_INTS] = (uint32_t)c.start;            // hot 0, cold 1, gid 2 (Haar 3 is this library's)
    h[W_SERIES] = c.randseries;
    h[W_GEN] = generator_code(c);
    h[W_NSKIP] = (uint32_t)c.ranlux_nskip;
    h[W_PRNG_COUNTER] = st->prng_counter;
    h[W_NAV] = (uint32_t)st->nav;
    h[W_NAV_COUNTER] = (uint32_t)st->nav_counter;
    h[W_NITER] = (uint32_t)st->niter;
    h[W_ITER] = (uint32_t)st->iter;
    h[W_ITER_COUNTER] = (uint32_t)st->iter_counter;
    h[W_NHIT] = (uint32_t)c.nhit;
    h[W_WILSON_R] = (uint32_t)c.wilson_r;
    h[W_WILSON_T] = (uint32_t)c.wilson_t;
    h[W_PRECISION] = c.precision ? 2 : 1;     // convert_precision_to_uint
    h[W_BETA_LO] = lo_word(c.beta);
    h[W_BETA_HI] = hi_word(c.beta);
    h[W_PHI_LO] = lo_word(c.phi);
    h[W_PHI_HI] = hi_word(c.phi);
    h[W_OMEGA_LO] = lo_word(c.omega);
    h[W_OMEGA_HI] = hi_word(c.omega);
    h[W_PL_LEVEL] = (uint32_t)st->pl_level;
    h[W_FMUNU1] = (uint32_t)st->fmunu_index1;
    h[W_FMUNU2] = (uint32_t)st->fmunu_index2;
    h[W_GET_FMUNU] = st->fmunu == 1 ? 1 : 0;
    h[W_GET_ACTIONS] = st->get_actions ? 1 : 0;
    h[W_GET_PLAQUETTES] = st->get_plaquettes ? 1 : 0;
    h[W_GET_WILSON] = st->get_wilson ? 1 : 0;
    h[W_MEAS_SIZE_F] = z.meas_F;
    h[W_ENERGIES_SIZE] = z.energies;
    h[W_ENERGIES_SIZE_F] = z.energies_F;
    h[W_POLYAKOV_SIZE] = z.polyakov;
    h[W_GROUP] = (uint32_t)c.group;
    h[W_ND] = 4;
    for (int i = 0; i < 4; i++) h[W_FULL_SIZE + i] = h[W_DOMAIN_SIZE + i] = (uint32_t)c.size[i];
    h[W_EXT_TAG] = str_word(kExtTag, 0);
    h[W_PRNG_KIND] = (uint32_t)c.prng;
    h[W_PHASE_LO] = (uint32_t)st->phase_counter;
    h[W_PHASE_HI] = (uint32_t)(st->phase_counter >> 32);
    h[W_SWEEPS_LO] = (uint32_t)st->sweeps_done;
    h[W_SWEEPS_HI] = (uint32_t)(st->sweeps_done >> 32);
    h[W_NOR] = (uint32_t)c.n_or;
    h[W_REUNIT_EVERY] = (uint32_t)c.reunit_every;
    h[W_REUNIT_FP64] = (uint32_t)c.reunit_fp64;
    h[W_NHITPAR] = (uint32_t)c.nhitpar;
    h[W_INSTANCES] = (uint32_t)c.prng_instances;
    h[W_ROW_ALIGN] = (uint32_t)c.row_align;
    h[W_FMUNU_KIND] = (uint32_t)st->fmunu;
    h[W_ACTIONS_DIFF] = (uint32_t)st->get_actions_diff;

    // series buffers, in the reference's element order (double2 .x/.y as
    // lattice_analysis reads them: S_spat/S_temp, Plq_spat/Plq_temp, Re/Im)
    const int n = st->iter_counter < st->iter ? st->iter_counter : st->iter;
    std::vector<double> meas(2 * (size_t)z.meas_F, 0.0), en(2 * (size_t)z.energies, 0.0),
        plq(2 * (size_t)z.energies_F, 0.0), wil((size_t)z.energies, 0.0), pol(2 * (size_t)z.polyakov, 0.0),
        p24(2 * (size_t)z.polyakov, 0.0);
    // the per-iteration profile rows (this library's tail block)
    const size_t plen = 2 * (size_t)(c.size[0] + c.size[1] + c.size[2]);
    const size_t prow = (st->pl_level > 2 ? plen : 0) + (st->get_actions_diff ? plen : 0);
    std::vector<double> prof(prow * (size_t)z.energies, 0.0);   // rows: the series' aligned length
    for (int i = 0; i < n; i++) {
        if (st->actions) { en[2 * i] = st->actions[2 * i]; en[2 * i + 1] = st->actions[2 * i + 1]; }
        if (st->plaquettes) { plq[2 * i] = st->plaquettes[2 * i]; plq[2 * i + 1] = st->plaquettes[2 * i + 1]; }
        // F_munu in energies_plq blocks 1..6 (reduce_measurement_plq_double2,
        // sun_measurements_cl.cl:1313-1357): index1 planes, then index2
        if (st->fmunu && st->fmunu_series)
            for (int k = 0; k < 6; k++) {
                plq[2 * ((size_t)(k + 1) * z.energies + i)] = st->fmunu_series[12 * i + 2 * k];
                plq[2 * ((size_t)(k + 1) * z.energies + i) + 1] = st->fmunu_series[12 * i + 2 * k + 1];
            }
        if (prow && st->profiles)
            for (size_t k = 0; k < prow; k++) prof[prow * i + k] = st->profiles[prow * i + k];
        if (st->wilson) wil[i] = st->wilson[i];
        if (st->polyakov) {
            pol[2 * i] = st->polyakov[4 * i];
            pol[2 * i + 1] = st->polyakov[4 * i + 1];
            p24[2 * i] = st->polyakov[4 * i + 2];
            p24[2 * i + 1] = st->polyakov[4 * i + 3];
        }
    }
    FILE *fp = fopen(path, "wb");
    if (!fp) return st_fail(QG_ERR_IO, std::string("cannot write ") + path);
    bool ok = fwrite(h, sizeof(uint32_t), QCDGPU_STATE_HEADER_WORDS, fp) == QCDGPU_STATE_HEADER_WORDS;
    ok = ok && fwrite(meas.data(), sizeof(double), meas.size(), fp) == meas.size();
    ok = ok && fwrite(en.data(), sizeof(double), en.size(), fp) == en.size();
    if (st->get_plaquettes || st->fmunu) ok = ok && fwrite(plq.data(), sizeof(double), plq.size(), fp) == plq.size();
    if (st->get_wilson) ok = ok && fwrite(wil.data(), sizeof(double), wil.size(), fp) == wil.size();
    if (st->pl_level > 0) ok = ok && fwrite(pol.data(), sizeof(double), pol.size(), fp) == pol.size();
    ok = ok && fwrite(links, 1, (size_t)links_bytes, fp) == (size_t)links_bytes;
    if (st->pl_level > 0) {
        const uint32_t tag = str_word(kTailTag, 0);
        ok = ok && fwrite(&tag, sizeof(tag), 1, fp) == 1;
        ok = ok && fwrite(p24.data(), sizeof(double), p24.size(), fp) == p24.size();
    }
    if (prow) {
        const uint32_t tag = str_word(kProfTag, 0);
        ok = ok && fwrite(&tag, sizeof(tag), 1, fp) == 1;
        ok = ok && fwrite(prof.data(), sizeof(double), prof.size(), fp) == prof.size();
    }
    if (fclose(fp) != 0) ok = false;
    if (!ok) return st_fail(QG_ERR_IO, std::string("short write to ") + path);
    return QG_OK;
}

extern "C" int qg_read_state_file(const char *path, qg_config *cfg, qg_run_state *st, void *links,
                                  uint64_t links_bytes)
{
    if (!path || !cfg || !st) return st_fail(QG_ERR_ARG, "qg_read_state_file: null argument");
    FILE *fp = fopen(path, "rb");
    if (!fp) return st_fail(QG_ERR_IO, std::string("cannot open ") + path);
    uint32_t h[QCDGPU_STATE_HEADER_WORDS];
    if (fread(h, sizeof(uint32_t), QCDGPU_STATE_HEADER_WORDS, fp) != QCDGPU_STATE_HEADER_WORDS) {
        fclose(fp);
        return st_fail(QG_ERR_IO, std::string("truncated state header in ") + path);
    }
    // lattice_load_bin_header: prefix and version must match
    if (h[0] != str_word(kPrefix, 0) || h[1] != str_word(kPrefix, 4) || h[2] != str_word(kVersion, 0)) {
        fclose(fp);
        return st_fail(QG_ERR_IO, std::string(path) + " is not a QCDGPU state file (prefix/version mismatch)");
    }
    if (h[W_ND] != 4 || (h[W_GROUP] != 2 && h[W_GROUP] != 3)) {
        fclose(fp);
        return st_fail(QG_ERR_UNSUPPORTED, "state file: only SU(2)/SU(3) in 4 dimensions");
    }
    qg_config &c = *cfg;
    c.group = (int)h[W_GROUP];
    for (int i = 0; i < 4; i++) c.size[i] = (int)h[W_FULL_SIZE + i];
    c.start = h[W_INTS] <= 3 ? (int)h[W_INTS] : QG_START_HOT;   // convert_uint_to_start
    c.randseries = h[W_SERIES];
    c.ranlux_nskip = (int)h[W_NSKIP];
    c.prng = QG_PRNG_RANLUX;
    c.nhit = (int)h[W_NHIT];
    c.wilson_r = (int)h[W_WILSON_R];
    c.wilson_t = (int)h[W_WILSON_T];
    c.precision = (h[W_PRECISION] == 2) ? 1 : 0;
    c.beta = from_words(h[W_BETA_LO], h[W_BETA_HI]);
    c.phi = from_words(h[W_PHI_LO], h[W_PHI_HI]);
    c.omega = from_words(h[W_OMEGA_LO], h[W_OMEGA_HI]);
    st->init = (int)h[W_INIT];
    st->prng_counter = h[W_PRNG_COUNTER];
    st->nav = (int)h[W_NAV];
    st->nav_counter = (int)h[W_NAV_COUNTER];
    st->niter = (int)h[W_NITER];
    st->iter = (int)h[W_ITER];
    st->iter_counter = (int)h[W_ITER_COUNTER];
    st->pl_level = (int)h[W_PL_LEVEL];
    st->get_actions = (int)h[W_GET_ACTIONS];
    st->get_plaquettes = (int)h[W_GET_PLAQUETTES];
    st->get_wilson = (int)h[W_GET_WILSON];
    st->fmunu = h[W_GET_FMUNU] ? 1 : 0;
    st->fmunu_index1 = (int)h[W_FMUNU1];
    st->fmunu_index2 = (int)h[W_FMUNU2];
    st->get_actions_diff = 0;
    st->phase_counter = 0;
    st->sweeps_done = 0;
    const bool ext = h[W_EXT_TAG] == str_word(kExtTag, 0);
    if (ext) {
        c.prng = (int)h[W_PRNG_KIND];
        st->phase_counter = ((uint64_t)h[W_PHASE_HI] << 32) | h[W_PHASE_LO];
        st->sweeps_done = ((uint64_t)h[W_SWEEPS_HI] << 32) | h[W_SWEEPS_LO];
        c.n_or = (int)h[W_NOR];
        c.reunit_every = (int)h[W_REUNIT_EVERY];
        c.reunit_fp64 = (int)h[W_REUNIT_FP64];
        c.nhitpar = (int)h[W_NHITPAR];
        c.prng_instances = (int)h[W_INSTANCES];
        c.row_align = (int)h[W_ROW_ALIGN];
        st->fmunu = (int)h[W_FMUNU_KIND];
        st->get_actions_diff = (int)h[W_ACTIONS_DIFF];
    } else {
        // a file of the reference: every sweep ends with a Gram-Schmidt pass
        c.n_or = 0;
        c.reunit_every = 1;
        c.reunit_fp64 = 0;
        c.nhitpar = 1;
    }
    const uint32_t meas_F = h[W_MEAS_SIZE_F], en_n = h[W_ENERGIES_SIZE], en_F = h[W_ENERGIES_SIZE_F],
                   pol_n = h[W_POLYAKOV_SIZE];
    const bool want = links || st->actions || st->plaquettes || st->wilson || st->polyakov || st->fmunu_series ||
                      st->profiles;
    if (!want) { fclose(fp); return QG_OK; }
    const int n = st->iter_counter < st->iter ? st->iter_counter : st->iter;
    if ((uint32_t)n > en_n || (uint32_t)n > pol_n || (uint32_t)n > en_F) {
        fclose(fp);
        return st_fail(QG_ERR_IO, "state file: ITER_counter beyond the stored series");
    }
    auto rd = [&](std::vector<double> &v, size_t count) {
        v.assign(count, 0.0);
        return fread(v.data(), sizeof(double), count, fp) == count;
    };
    std::vector<double> meas, en, plq, wil, pol;
    bool ok = rd(meas, 2 * (size_t)meas_F) && rd(en, 2 * (size_t)en_n);
    if (ok && (st->get_plaquettes || st->fmunu)) ok = rd(plq, 2 * (size_t)en_F);
    if (ok && st->get_wilson) ok = rd(wil, (size_t)en_n);
    if (ok && st->pl_level > 0) ok = rd(pol, 2 * (size_t)pol_n);
    const size_t real = c.precision ? 8 : 4;
    const uint64_t table_bytes = table_float4s(c) * 4 * real;
    std::vector<char> skip;
    if (ok && links) {
        if (links_bytes != table_bytes) {
            fclose(fp);
            return st_fail(QG_ERR_ARG, "qg_read_state_file: link buffer of " + std::to_string(links_bytes) +
                                           " bytes, the file holds " + std::to_string(table_bytes));
        }
        ok = fread(links, 1, (size_t)table_bytes, fp) == (size_t)table_bytes;
    } else if (ok) {
        ok = fseek(fp, (long)table_bytes, SEEK_CUR) == 0;
    }
    std::vector<double> p24, prof;
    const size_t plen = 2 * (size_t)(c.size[0] + c.size[1] + c.size[2]);
    const size_t prow = (st->pl_level > 2 ? plen : 0) + (st->get_actions_diff ? plen : 0);
    uint32_t tag = 0;
    bool have_tag = ok && fread(&tag, sizeof(tag), 1, fp) == 1;
    if (have_tag && tag == str_word(kTailTag, 0)) {
        ok = rd(p24, 2 * (size_t)pol_n);
        have_tag = ok && fread(&tag, sizeof(tag), 1, fp) == 1;
    }
    if (have_tag && tag == str_word(kProfTag, 0) && prow) ok = rd(prof, prow * (size_t)en_n);
    fclose(fp);
    if (!ok) return st_fail(QG_ERR_IO, std::string("truncated state file ") + path);
    for (int i = 0; i < n; i++) {
        if (st->actions) { st->actions[2 * i] = en[2 * i]; st->actions[2 * i + 1] = en[2 * i + 1]; }
        if (st->plaquettes && !plq.empty()) { st->plaquettes[2 * i] = plq[2 * i]; st->plaquettes[2 * i + 1] = plq[2 * i + 1]; }
        if (st->wilson && !wil.empty()) st->wilson[i] = wil[i];
        if (st->polyakov && !pol.empty()) {
            st->polyakov[4 * i] = pol[2 * i];
            st->polyakov[4 * i + 1] = pol[2 * i + 1];
            st->polyakov[4 * i + 2] = p24.empty() ? 0.0 : p24[2 * i];
            st->polyakov[4 * i + 3] = p24.empty() ? 0.0 : p24[2 * i + 1];
        }
        if (st->fmunu_series && st->fmunu && (size_t)en_F >= 7 * (size_t)en_n)
            for (int k = 0; k < 6; k++) {
                st->fmunu_series[12 * i + 2 * k] = plq[2 * ((size_t)(k + 1) * en_n + i)];
                st->fmunu_series[12 * i + 2 * k + 1] = plq[2 * ((size_t)(k + 1) * en_n + i) + 1];
            }
        if (st->profiles && !prof.empty())
            for (size_t k = 0; k < prow; k++) st->profiles[prow * i + k] = prof[prow * i + k];
    }
    return QG_OK;
}

extern "C" int qg_save_state(qg_ctx *ctx, const char *path, const qg_run_state *st)
{
    if (!ctx || !path || !st) return st_fail(QG_ERR_ARG, "qg_save_state: null argument");
    qg_info info;
    int rc = qg_get_info(ctx, &info);
    if (rc) return rc;
    qg_config cfg;
    if ((rc = qg_get_config(ctx, &cfg))) return rc;
    const size_t real = cfg.precision ? 8 : 4;
    std::vector<char> buf((size_t)info.ref_elems * real);
    if ((rc = qg_links_download(ctx, buf.data(), QG_LAYOUT_REFERENCE))) return rc;
    qg_run_state s = *st;
    s.prng_counter = info.prng_counter;
    s.phase_counter = info.phase_counter;
    s.sweeps_done = info.sweeps_done;
    return qg_write_state_file(path, &cfg, &s, buf.data(), (uint64_t)buf.size());
}

extern "C" int qg_tau_int(const double *x, int n, double c, double *tau, int *window)
{
    if (!x || !tau || !window || n < 0) return st_fail(QG_ERR_ARG, "qg_tau_int: bad argument");
    *tau = 0.5;
    *window = 0;
    if (n < 2) return QG_OK;
    double mean = 0;
    for (int i = 0; i < n; i++) mean += x[i];
    mean /= n;
    double c0 = 0;
    for (int i = 0; i < n; i++) c0 += (x[i] - mean) * (x[i] - mean);
    c0 /= n;
    if (!(c0 > 0)) return QG_OK;
    double t = 0.5;
    for (int w = 1; w < n; w++) {
        double ct = 0;
        for (int i = 0; i + w < n; i++) ct += (x[i] - mean) * (x[i + w] - mean);
        ct /= n;
        t += ct / c0;
        if (w >= c * t) {
            *tau = t;
            *window = w;
            return QG_OK;
        }
    }
    *tau = t;
    *window = n - 1;
    return QG_OK;
}
