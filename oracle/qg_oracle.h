/*
 * qg_oracle.h -- CPU oracle for the SU(2)/SU(3) checkerboard link sweep.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the QCDGPU
 * reference algorithm (vadimdi/QCDGPU, OpenCL kernels under SU(N)/suncl and
 * SU(N)/random).  It exists to check the CUDA product path; nothing in the
 * product may link, load or call it.  Only tests/, __graft_entry__.smoke()
 * and the cpu_baseline leg of bench.py use it.
 *
 * Link tables handed to this oracle use the reference's storage layout
 * (SU(N)/suncl/su3_matrix_memory.cl:43-176, su2_matrix_memory.cl:56-143):
 * SoA planes of 4-vectors, element (site, plane) at (site + plane*rowsize)*4,
 * SU(3) planes dir, dir+4, dir+8 = (Re u11,Re u12,Re u13,Re u23),
 * (Im u11,Im u12,Im u13,Im u23), (Re u21,Re u22,Im u21,Im u22);
 * SU(2) plane dir = (Re u11, Re u12, Im u11, Im u12).
 * Site index gid = y + N2*z + N2N3*t + N2N3N4*x (SU(N)/suncl/sun_common.cl:41-66).
 */
#ifndef QG_ORACLE_H
#define QG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ol_cfg {
    int group;          /* 2 or 3                                        */
    int n[4];           /* N1..N4 = x, y, z, t extents                   */
    int precision;      /* 0: float links/arithmetic, 1: double          */
    int rowsize;        /* ROWSIZE  (V aligned)                          */
    int prngstep;       /* PRNGSTEP (V/2 aligned)                        */
    int nhit;           /* NHIT                                          */
    int nhitpar;        /* NHITPar                                       */
    double beta;        /* BETA; kernels see (Real)(BETA/N)              */
    double phi, omega;  /* twisted boundary parameters (0,0 = periodic)  */
    int gid_mode;       /* INTS=2 deterministic update formulas          */
} ol_cfg;

/* ---- PRNG: glibc seeding + RANLUX (random/random.cpp, prngcl_ranlux.cl) */
typedef struct ol_ranlux {
    float seeds[24];
    int i24, j24, in24, nskip;
    float carry;
} ol_ranlux;

/* PRN source for the heatbath: 0 = reference-layout float4 buffer read at
 * GID + k*PRNGSTEP; 1 = Philox4x32-10 counter stream (fast mode);
 * 2 = one RANLUX stream consumed in order, as the reference's sequential
 * CPU path draws it (SU(N)/suncpp/su2/update_su2.cpp:81,101: 4 numbers per
 * Kennedy-Pendleton try, 2 for the direction, no skip after a rejection);
 * the links of a phase are then visited one after the other.               */
typedef struct ol_prn {
    int mode;
    const float *prns;        /* mode 0: float4 buffer                      */
    uint32_t key0, key1;      /* mode 1: Philox key                         */
    uint64_t phase;           /* mode 1: phase counter                      */
    ol_ranlux *stream;        /* mode 2: the stream (advanced in place)     */
} ol_prn;

void  ol_glibc_seeds(uint32_t randseries, int instances, uint32_t *seeds);
void  ol_ranlux_init(ol_ranlux *st, int32_t jseed, int nskip);
float ol_ranlux_next(ol_ranlux *st);
void  ol_ranlux_states(const uint32_t *seeds, int instances, int nskip, ol_ranlux *states);
void  ol_ranlux_batch(ol_ranlux *states, int instances, int samples, float *prns);
int   ol_sizeof_ranlux(void);

/* ---- Philox4x32-10 (Salmon et al., SC'11) */
void  ol_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void  ol_philox_prn(const ol_prn *src, uint32_t thread, uint32_t k, float out[4]);

/* ---- test-only: the heatbath's delta as the reference writes it (unfused,
 *      the C library's cos / sin / log); 0 restores this build's arithmetic */
void  ol_set_reference_arith(int on);
extern int ol_ref_arith;

/* ---- the float sin / cos of the FP32 update path */
float ol_sinf_own(float x);
float ol_cosf_own(float x);

/* ---- lattice kernels (table in reference layout, Real = float|double) */
void ol_init_cold(const ol_cfg *c, void *table);
void ol_init_gid(const ol_cfg *c, void *table);
void ol_init_hot_dir(const ol_cfg *c, void *table, int dir, const float *prns);
void ol_phase_hb(const ol_cfg *c, void *table, int parity, int dir, const ol_prn *src);
void ol_phase_or(const ol_cfg *c, void *table, int parity, int dir);
void ol_gramschmidt(const ol_cfg *c, void *table);        /* Real precision  */
void ol_gramschmidt_fp64(const ol_cfg *c, void *table);   /* FP64 arithmetic */
void ol_plaquette(const ol_cfg *c, const void *table, double out[2]);
/* the plaquette sums with FP32 products and traces (FP32 links; FP64 links: ol_plaquette) */
void ol_plaquette_f32(const ol_cfg *c, const void *table, double out[2]);
void ol_action(const ol_cfg *c, const void *table, double out[2]);
void ol_polyakov(const ol_cfg *c, const void *table, double out[4]);
/* F_munu projections of the plaquettes (field 0: xy, xz, yz; 1: xt, yt, zt)
 * on generators i1, i2: out[2p], out[2p+1] = Re, Im sum over sites for i1
 * and plane p, out[6+2p], out[7+2p] for i2 */
void ol_fmunu(const ol_cfg *c, const void *table, int field, int i1, int i2, double out[12]);
/* per slice of coordinate axis (0..2): spatial, temporal action sums */
void ol_action_profile(const ol_cfg *c, const void *table, int axis, double *out);
/* per slice of spatial coordinate axis (0..2): Re, Im Polyakov trace sums */
void ol_polyakov_profile(const ol_cfg *c, const void *table, int axis, double *out);
double ol_wilson(const ol_cfg *c, const void *table, int R, int T);
double ol_local_action_link(const ol_cfg *c, const void *table, int gid, int dir);

/* ---- learned-proposal Metropolis (SU(3), float links; qg_oracle_learned.h) */
double ol_expd(double x);
void   ol_mh_features(const ol_cfg *c, const void *table, int gid, int mu, float x[8]);
float  ol_mlp_out(const float *w, const float x[8]);
void   ol_mh_phase(const ol_cfg *c, void *table, int parity, int mu, const float *w, double eps_max, int nhit,
                   uint32_t key0, uint32_t key1, uint64_t phase, uint64_t *acc, double *jump);
void   ol_mh_phase_eps(const ol_cfg *c, void *table, int parity, int mu, const float *eps, int nhit,
                       uint32_t key0, uint32_t key1, uint64_t phase, uint64_t *acc, double *jump);
void   ol_net_eps(const ol_cfg *c, const void *table, int parity, int mu, const float *w, double eps_max, float *eps);
void   ol_mh_grad(const ol_cfg *c, const void *table, int parity, int mu, const float *w, double eps_max,
                  uint32_t key0, uint32_t key1, uint64_t phase, int tc, double *grad, double stats[4]);
double ol_mh_loss(const ol_cfg *c, const void *table, int parity, int mu, const double *w, double eps_max,
                  uint32_t key0, uint32_t key1, uint64_t phase);

#ifdef __cplusplus
}
#endif
#endif
