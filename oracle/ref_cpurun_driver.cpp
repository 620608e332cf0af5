// Test and baseline infrastructure only.  Drives the reference's own
// sequential CPU path (SU(N)/suncpp, the -D CPU_RUN build of vadimdi/QCDGPU)
// through its templates: modelCPU<su_n> (suncpp/sunh.h), lattice_update_odd /
// lattice_update_even (suncpp/Update/sun_update.h:80-119) and plqConf
// (suncpp/Measurements/Plq.h:47-95), in the sweep order of
// suncpp/suncpp.h:143-167.  Compiled from the reference sources where they
// lie; nothing of it is copied into this repository.
//
// Usage:
//   ref_cpurun plaq  <group> <L1> <L2> <L3> <L4> <beta> <ints> <randseries> <sweeps>
//       prints "sweep spat temp total" per sweep with %.17g (sweep 0 = start)
//   ref_cpurun bench <group> <L1> <L2> <L3> <L4> <beta> <randseries> <warm> <timed>
//       cold start, <warm> untimed sweeps, then times <timed> sweeps and
//       prints "link_updates_per_s <value> seconds <t>"
//   ref_cpurun phases <group> <L1> <L2> <L3> <L4> <beta> <randseries> <warm> <timed>
//       cold start, <warm> untimed phases, then <timed> phases (the sweep's
//       odd X..T, even X..T order, V/2 link updates each); prints
//       "phase_seconds t1 t2 ..."
//   ref_cpurun phases_from <group> <L1> <L2> <L3> <L4> <beta> <randseries> <in> <warm> <timed>
//       as "phases", from the start field read from <in> (the "links" format)
//   ref_cpurun links <group> <L1> <L2> <L3> <L4> <beta> <randseries> <phases> <in|-> <out>
//       cold start, or the stored rows read from <in> (per site, dir fastest:
//       SU(3) u1 u2 u3 v1 v2 v3, SU(2) u1 u2, each re im, as doubles; the
//       other rows rebuilt by the reference's matrix_reconstruct), then
//       <phases> heatbath phases in the sweep order; the rows written to
//       <out> in the same format
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "QCDGPU.h"

template <typename su_n>
static void sweep(modelCPU<su_n> *lat, PRNG_CL::PRNG *prng)
{
    lattice_update_odd(lat, X, prng);
    lattice_update_odd(lat, Y, prng);
    lattice_update_odd(lat, Z, prng);
    lattice_update_odd(lat, T, prng);
    lattice_update_even(lat, X, prng);
    lattice_update_even(lat, Y, prng);
    lattice_update_even(lat, Z, prng);
    lattice_update_even(lat, T, prng);
}

template <typename su_n>
static void phase(modelCPU<su_n> *lat, PRNG_CL::PRNG *prng, int k)
{
    int dir = k % 4;
    if ((k / 4) % 2 == 0) lattice_update_odd(lat, dir, prng);
    else lattice_update_even(lat, dir, prng);
}

static void put_rows(const su_3 &m, double *r)
{
    const hgpu_complex c[6] = { m.u1, m.u2, m.u3, m.v1, m.v2, m.v3 };
    for (int k = 0; k < 6; k++) { r[2 * k] = c[k].re; r[2 * k + 1] = c[k].im; }
}
static void get_rows(su_3 &m, const double *r)
{
    hgpu_complex *c[6] = { &m.u1, &m.u2, &m.u3, &m.v1, &m.v2, &m.v3 };
    for (int k = 0; k < 6; k++) { c[k]->re = r[2 * k]; c[k]->im = r[2 * k + 1]; }
    matrix_reconstruct(&m);
}
static void put_rows(const su_2 &m, double *r)
{
    r[0] = m.u1.re; r[1] = m.u1.im; r[2] = m.u2.re; r[3] = m.u2.im;
}
static void get_rows(su_2 &m, const double *r)
{
    m.u1.re = r[0]; m.u1.im = r[1]; m.u2.re = r[2]; m.u2.im = r[3];
    matrix_reconstruct(&m);
}

template <typename su_n>
static int links(int group, int *L, double beta, int series, int phases, const char *in, const char *out,
                 int timed = 0)
{
    modelCPU<su_n> *lat = new modelCPU<su_n>;
    lat->lattice_ndCPU = 4;
    lat->lattice_size = (int *)calloc(4, sizeof(int));
    for (int i = 0; i < 4; i++) lat->lattice_size[i] = L[i];
    lat->ints = 1;
    lat->nhit = 10;
    lat->beta = beta;
    lat->lattice_group = group;
    lat->lattice_sitesCPU = L[0] * L[1] * L[2] * L[3];
    PRNG_CL::PRNG *prng = new PRNG_CL::PRNG;
    prng->PRNG_generator = PRNG_CL::PRNG::PRNG_generator_RANLUX3;
    prng->PRNG_randseries = series;
    prng->PRNG_precision = PRNG_CL::PRNG::PRNG_precision_single;
    prng->initialize_CPU();
    lat->create_latticeCPU();
    lat->lattice_initializeCPU();
    const int nrow = group == 3 ? 12 : 4;
    const size_t nlinks = (size_t)lat->lattice_sitesCPU * 4;
    double *rows = (double *)malloc(nlinks * nrow * sizeof(double));
    if (strcmp(in, "-") != 0) {
        FILE *f = fopen(in, "rb");
        if (!f || fread(rows, sizeof(double), nlinks * nrow, f) != nlinks * nrow) {
            fprintf(stderr, "cannot read %s\n", in);
            return 1;
        }
        fclose(f);
        for (size_t i = 0; i < nlinks; i++) get_rows(lat->lattice_tableCPU[i], rows + i * nrow);
    }
    for (int k = 0; k < phases; k++) phase(lat, prng, k);
    if (timed > 0) {                          // phases_from: time the next phases, write nothing
        printf("phase_seconds");
        for (int k = phases; k < phases + timed; k++) {
            auto t0 = std::chrono::steady_clock::now();
            phase(lat, prng, k);
            auto t1 = std::chrono::steady_clock::now();
            printf(" %.6f", std::chrono::duration<double>(t1 - t0).count());
        }
        printf("\n");
        free(rows);
        lat->delete_latticeCPU();
        free(lat->lattice_size);
        delete lat;
        delete prng;
        return 0;
    }
    for (size_t i = 0; i < nlinks; i++) put_rows(lat->lattice_tableCPU[i], rows + i * nrow);
    FILE *f = fopen(out, "wb");
    if (!f || fwrite(rows, sizeof(double), nlinks * nrow, f) != nlinks * nrow) {
        fprintf(stderr, "cannot write %s\n", out);
        return 1;
    }
    fclose(f);
    free(rows);
    lat->delete_latticeCPU();
    free(lat->lattice_size);
    delete lat;
    delete prng;
    return 0;
}

template <typename su_n>
static int run(int mode, int group, int *L, double beta, int ints, int series, int a, int b)
{
    modelCPU<su_n> *lat = new modelCPU<su_n>;
    lat->lattice_ndCPU = 4;
    lat->lattice_size = (int *)calloc(4, sizeof(int));
    for (int i = 0; i < 4; i++) lat->lattice_size[i] = L[i];
    lat->ints = ints;
    lat->nhit = 10;
    lat->beta = beta;
    lat->lattice_group = group;
    lat->lattice_sitesCPU = L[0] * L[1] * L[2] * L[3];
    PRNG_CL::PRNG *prng = new PRNG_CL::PRNG;
    prng->PRNG_generator = PRNG_CL::PRNG::PRNG_generator_RANLUX3;
    prng->PRNG_randseries = series;
    prng->PRNG_precision = PRNG_CL::PRNG::PRNG_precision_single;
    prng->initialize_CPU();
    lat->create_latticeCPU();
    lat->lattice_initializeCPU();
    if (mode == 0) {
        for (int s = 0; s <= a; s++) {
            if (s > 0) sweep(lat, prng);
            hgpu_double tot;
            hgpu_complex p = plqConf(lat, &tot);
            printf("%d %.17g %.17g %.17g\n", s, (double)p.re, (double)p.im, (double)tot);
        }
    } else if (mode == 2) {
        for (int k = 0; k < a; k++) phase(lat, prng, k);
        printf("phase_seconds");
        for (int k = a; k < a + b; k++) {
            auto t0 = std::chrono::steady_clock::now();
            phase(lat, prng, k);
            auto t1 = std::chrono::steady_clock::now();
            printf(" %.6f", std::chrono::duration<double>(t1 - t0).count());
        }
        printf("\n");
    } else {
        for (int s = 0; s < a; s++) sweep(lat, prng);
        auto t0 = std::chrono::steady_clock::now();
        for (int s = 0; s < b; s++) sweep(lat, prng);
        auto t1 = std::chrono::steady_clock::now();
        double sec = std::chrono::duration<double>(t1 - t0).count();
        double lu = 4.0 * lat->lattice_sitesCPU * b / sec;
        hgpu_double tot;
        plqConf(lat, &tot);
        printf("link_updates_per_s %.6e seconds %.6f plaquette %.10f\n", lu, sec, (double)tot);
    }
    lat->delete_latticeCPU();
    free(lat->lattice_size);
    delete lat;
    delete prng;
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 11) { fprintf(stderr, "see source for usage\n"); return 2; }
    if (strcmp(argv[1], "phases_from") == 0) {
        if (argc < 12) { fprintf(stderr, "see source for usage\n"); return 2; }
        int L[4] = { atoi(argv[3]), atoi(argv[4]), atoi(argv[5]), atoi(argv[6]) };
        return atoi(argv[2]) == 3
                   ? links<su_3>(3, L, atof(argv[7]), atoi(argv[8]), atoi(argv[10]), argv[9], nullptr, atoi(argv[11]))
                   : links<su_2>(2, L, atof(argv[7]), atoi(argv[8]), atoi(argv[10]), argv[9], nullptr, atoi(argv[11]));
    }
    if (strcmp(argv[1], "links") == 0) {
        if (argc < 12) { fprintf(stderr, "see source for usage\n"); return 2; }
        int L[4] = { atoi(argv[3]), atoi(argv[4]), atoi(argv[5]), atoi(argv[6]) };
        return atoi(argv[2]) == 3 ? links<su_3>(3, L, atof(argv[7]), atoi(argv[8]), atoi(argv[9]), argv[10], argv[11])
                                  : links<su_2>(2, L, atof(argv[7]), atoi(argv[8]), atoi(argv[9]), argv[10], argv[11]);
    }
    int mode = strcmp(argv[1], "plaq") == 0 ? 0 : strcmp(argv[1], "phases") == 0 ? 2 : 1;
    int group = atoi(argv[2]);
    int L[4] = { atoi(argv[3]), atoi(argv[4]), atoi(argv[5]), atoi(argv[6]) };
    double beta = atof(argv[7]);
    if (mode == 0)
        return group == 3 ? run<su_3>(0, 3, L, beta, atoi(argv[8]), atoi(argv[9]), atoi(argv[10]), 0)
                          : run<su_2>(0, 2, L, beta, atoi(argv[8]), atoi(argv[9]), atoi(argv[10]), 0);
    return group == 3 ? run<su_3>(mode, 3, L, beta, 1, atoi(argv[8]), atoi(argv[9]), atoi(argv[10]))
                      : run<su_2>(mode, 2, L, beta, 1, atoi(argv[8]), atoi(argv[9]), atoi(argv[10]));
}
