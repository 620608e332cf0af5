// qg_ranlux.cu -- RANLUX (Luescher 1994; James 1994) in the reference's
// batch layout: one generator per instance, generator i writes its n-th
// four consecutive outputs to prns[n*instances + i]
// (SU(N)/random/prngcl_ranlux.cl:97-563).  Bit-exact: the subtract-with-
// borrow arithmetic on multiples of 2^-24 is exact in FP32, and the small-
// value refinement is one correctly rounded add of an exact product.
//
// The 24-word state lives in registers (as exact integers, rl_step).
// Within a block of 24 outputs the
// word indices are compile-time constants (switch on the float4 number
// 0..5); the luxury skip of NSKIP words is whole 24-step rounds plus
// NSKIP%24 single steps followed by a register rotation that restores the
// block-start indexing (i24 = 23, j24 = 9).
#include "qg_internal.h"
#include "qg_rlx576.h"

namespace qg {

#define RL_TWOM24 5.9604644775390625e-8f
#define RL_TWOM12 2.44140625e-4f

// The words are kept as exact integers x = (word * 2^24) << 8 (the 24
// significant bits at the top of a 32-bit register) and the borrow as 0/1:
// a subtract-with-borrow step is x_i = x_j - x_i - 256 c (mod 2^32), with
// c = the borrow of that subtraction -- the float recurrence of the
// reference (u = s[j] - s[i] - carry; u < 0: u += 1, carry = 2^-24) on the
// same exact values.  Outputs and the table are floats (x * 2^-32, exact).
__device__ __forceinline__ uint32_t rl_step(uint32_t (&x)[24], int i, int j, uint32_t &c)
{
    const uint32_t a = x[j], b = x[i];
    const uint32_t u = a - b - (c << 8);
    c = (a < b || (a == b && c)) ? 1u : 0u;
    x[i] = u;
    return u;
}
__device__ __forceinline__ float rl_float(uint32_t x) { return __uint2float_rn(x) * 2.3283064365386963e-10f; }

// One round of 24 steps (i24 = 23 .. 0 with j24 = 9 .. 0, 23 .. 10) on
// words held as x = w << 8 in one asm block: each step one subtraction
// with borrow-in and borrow-out (the carry flag is the subtract-with-
// borrow borrow; the 2^24 wrap of a word is the 2^32 wrap of x) and a mask
// of the low byte, which a borrow-in fills with ones.  and.b32 leaves the
// flag alone, so the borrow chain is one instruction per step.
__device__ __forceinline__ void rl_round24(uint32_t (&x)[24], uint32_t &c)
{
    asm volatile(
        "{\n\t"
        ".reg .u32 z, t;\n\t"
        "mov.u32 z, 0;\n\t"
        "sub.cc.u32 t, z, %24;\n\t"
        "subc.cc.u32 %23, %9, %23;\n\t"
        "and.b32 %23, %23, 0xffffff00;\n\t"
        "subc.cc.u32 %22, %8, %22;\n\t"
        "and.b32 %22, %22, 0xffffff00;\n\t"
        "subc.cc.u32 %21, %7, %21;\n\t"
        "and.b32 %21, %21, 0xffffff00;\n\t"
        "subc.cc.u32 %20, %6, %20;\n\t"
        "and.b32 %20, %20, 0xffffff00;\n\t"
        "subc.cc.u32 %19, %5, %19;\n\t"
        "and.b32 %19, %19, 0xffffff00;\n\t"
        "subc.cc.u32 %18, %4, %18;\n\t"
        "and.b32 %18, %18, 0xffffff00;\n\t"
        "subc.cc.u32 %17, %3, %17;\n\t"
        "and.b32 %17, %17, 0xffffff00;\n\t"
        "subc.cc.u32 %16, %2, %16;\n\t"
        "and.b32 %16, %16, 0xffffff00;\n\t"
        "subc.cc.u32 %15, %1, %15;\n\t"
        "and.b32 %15, %15, 0xffffff00;\n\t"
        "subc.cc.u32 %14, %0, %14;\n\t"
        "and.b32 %14, %14, 0xffffff00;\n\t"
        "subc.cc.u32 %13, %23, %13;\n\t"
        "and.b32 %13, %13, 0xffffff00;\n\t"
        "subc.cc.u32 %12, %22, %12;\n\t"
        "and.b32 %12, %12, 0xffffff00;\n\t"
        "subc.cc.u32 %11, %21, %11;\n\t"
        "and.b32 %11, %11, 0xffffff00;\n\t"
        "subc.cc.u32 %10, %20, %10;\n\t"
        "and.b32 %10, %10, 0xffffff00;\n\t"
        "subc.cc.u32 %9, %19, %9;\n\t"
        "and.b32 %9, %9, 0xffffff00;\n\t"
        "subc.cc.u32 %8, %18, %8;\n\t"
        "and.b32 %8, %8, 0xffffff00;\n\t"
        "subc.cc.u32 %7, %17, %7;\n\t"
        "and.b32 %7, %7, 0xffffff00;\n\t"
        "subc.cc.u32 %6, %16, %6;\n\t"
        "and.b32 %6, %6, 0xffffff00;\n\t"
        "subc.cc.u32 %5, %15, %5;\n\t"
        "and.b32 %5, %5, 0xffffff00;\n\t"
        "subc.cc.u32 %4, %14, %4;\n\t"
        "and.b32 %4, %4, 0xffffff00;\n\t"
        "subc.cc.u32 %3, %13, %3;\n\t"
        "and.b32 %3, %3, 0xffffff00;\n\t"
        "subc.cc.u32 %2, %12, %2;\n\t"
        "and.b32 %2, %2, 0xffffff00;\n\t"
        "subc.cc.u32 %1, %11, %1;\n\t"
        "and.b32 %1, %1, 0xffffff00;\n\t"
        "subc.cc.u32 %0, %10, %0;\n\t"
        "and.b32 %0, %0, 0xffffff00;\n\t"
        "subc.u32 t, z, z;\n\t"
        "neg.s32 %24, t;\n\t"
        "}"
        : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5]), "+r"(x[6]), "+r"(x[7]), "+r"(x[8]), "+r"(x[9]), "+r"(x[10]), "+r"(x[11]), "+r"(x[12]), "+r"(x[13]), "+r"(x[14]), "+r"(x[15]), "+r"(x[16]), "+r"(x[17]), "+r"(x[18]), "+r"(x[19]), "+r"(x[20]), "+r"(x[21]), "+r"(x[22]), "+r"(x[23]), "+r"(c));
}

// q-th output of a block: i24 = 23-q, j24 = (9-q) mod 24; the refinement
// reads the word at the decremented j24
template <int Q>
__device__ __forceinline__ float rl_out(uint32_t (&x)[24], uint32_t &c)
{
    constexpr int I = 23 - Q;
    constexpr int J = (33 - Q) % 24;
    constexpr int JN = (32 - Q) % 24;
    float u = rl_float(rl_step(x, I, J, c));
    if (u < RL_TWOM12) {
        u = u + RL_TWOM24 * rl_float(x[JN]);
        if (u == 0.0f) u = RL_TWOM24 * RL_TWOM24;
    }
    return u;
}

template <int M>
__device__ __forceinline__ float4 rl_quad(uint32_t (&x)[24], uint32_t &c)
{
    float4 r;
    r.x = rl_out<4 * M + 0>(x, c);
    r.y = rl_out<4 * M + 1>(x, c);
    r.z = rl_out<4 * M + 2>(x, c);
    r.w = rl_out<4 * M + 3>(x, c);
    return r;
}

template <int NSKIP>
__device__ __forceinline__ void rl_skip(uint32_t (&x)[24], uint32_t &c)
{
#pragma unroll 1
    for (int r = 0; r < NSKIP / 24; r++) rl_round24(x, c);
    constexpr int R = NSKIP % 24;
#pragma unroll
    for (int q = 0; q < R; q++) rl_step(x, 23 - q, (33 - q) % 24, c);
    if (R) {
        uint32_t t[24];
#pragma unroll
        for (int k = 0; k < 24; k++) t[(k + R) % 24] = x[k];
#pragma unroll
        for (int k = 0; k < 24; k++) x[k] = t[k];
    }
}

template <int NSKIP>
__global__ void __launch_bounds__(128) k_ranlux(float4 *table, float4 *prns, int instances, int samples)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= instances) return;
    uint32_t x[24];
#pragma unroll
    for (int k = 0; k < 6; k++) {
        float4 v = table[(size_t)k * instances + i];
        x[4 * k] = (uint32_t)(v.x * 16777216.0f) << 8; x[4 * k + 1] = (uint32_t)(v.y * 16777216.0f) << 8;
        x[4 * k + 2] = (uint32_t)(v.z * 16777216.0f) << 8; x[4 * k + 3] = (uint32_t)(v.w * 16777216.0f) << 8;
    }
    float4 ci = table[(size_t)6 * instances + i];
    int in24 = (int)ci.z;
    uint32_t c = ci.w != 0.0f ? 1u : 0u;
    for (int n = 0; n < samples; n++) {
        if (in24 >= 6) { rl_skip<NSKIP>(x, c); in24 = 0; }
        float4 out;
        switch (in24) {
        case 0: out = rl_quad<0>(x, c); break;
        case 1: out = rl_quad<1>(x, c); break;
        case 2: out = rl_quad<2>(x, c); break;
        case 3: out = rl_quad<3>(x, c); break;
        case 4: out = rl_quad<4>(x, c); break;
        default: out = rl_quad<5>(x, c); break;
        }
        in24++;
        prns[(size_t)n * instances + i] = out;
    }
#pragma unroll
    for (int k = 0; k < 6; k++)
        table[(size_t)k * instances + i] =
            make_float4(rl_float(x[4 * k]), rl_float(x[4 * k + 1]), rl_float(x[4 * k + 2]), rl_float(x[4 * k + 3]));
    table[(size_t)6 * instances + i] = make_float4(0.0f, 0.0f, (float)in24, c ? RL_TWOM24 : 0.0f);
}

// ---------------------------------------------- one generator, several threads
// A batch of whole luxury blocks (samples % 6 == 0; every batch then starts
// at a block boundary, in24 = 6) split over `parts` threads per generator:
// segment j produces luxury blocks [j B / parts, (j+1) B / parts) of the
// B = samples / 6.  k_ranlux_jump gives each segment its start state --
// the batch-start state moved S_j = b0_j (NSKIP + 24) steps ahead by one
// multiplication by a^S_j modulo 2^576 - 2^240 + 1 (qg_rlx576.h; mult holds
// a^S_j for every segment, host-computed) -- into seg[j]; k_ranlux_seg
// runs the serial kernel's steps from there, and the last segment writes
// the batch-end state back to the table.  The outputs are those of the
// serial kernel bit for bit.

// the table rows of a state at a block start: x[23 - k] is the k-th oldest word
__device__ __forceinline__ void rl_load(const float4 *t, int instances, int i, uint32_t (&x)[24], uint32_t &c)
{
#pragma unroll
    for (int k = 0; k < 6; k++) {
        float4 v = t[(size_t)k * instances + i];
        x[4 * k] = (uint32_t)(v.x * 16777216.0f) << 8; x[4 * k + 1] = (uint32_t)(v.y * 16777216.0f) << 8;
        x[4 * k + 2] = (uint32_t)(v.z * 16777216.0f) << 8; x[4 * k + 3] = (uint32_t)(v.w * 16777216.0f) << 8;
    }
    c = t[(size_t)6 * instances + i].w != 0.0f ? 1u : 0u;
}
__device__ __forceinline__ void rl_store(float4 *t, int instances, int i, const uint32_t (&x)[24], uint32_t c)
{
#pragma unroll
    for (int k = 0; k < 6; k++)
        t[(size_t)k * instances + i] =
            make_float4(rl_float(x[4 * k]), rl_float(x[4 * k + 1]), rl_float(x[4 * k + 2]), rl_float(x[4 * k + 3]));
    t[(size_t)6 * instances + i] = make_float4(0.0f, 0.0f, 6.0f, c ? RL_TWOM24 : 0.0f);
}

__global__ void __launch_bounds__(128) k_ranlux_jump(const float4 *table, float4 *seg, int instances, int parts,
                                                      const uint32_t *mult)
{
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= instances * parts) return;
    const int i = id % instances, j = id / instances;
    uint32_t x[24], c;
    rl_load(table, instances, i, x, c);
    if (j > 0) {
        uint32_t L[24], E[rlx::kLimbs], M[rlx::kLimbs], J[rlx::kLimbs];
        for (int k = 0; k < 24; k++) L[k] = x[23 - k] >> 8;
        rlx::encode(L, c, E);
        for (int k = 0; k < rlx::kLimbs; k++) M[k] = __ldg(mult + (size_t)j * rlx::kLimbs + k);
        rlx::mulmod(E, M, J);
        rlx::decode(J, L, c);
        for (int k = 0; k < 24; k++) x[23 - k] = L[k] << 8;
    }
    rl_store(seg + (size_t)j * 7 * instances, instances, i, x, c);
}

template <int NSKIP>
__global__ void __launch_bounds__(128) k_ranlux_seg(float4 *table, const float4 *seg, float4 *prns, int instances,
                                                    int samples, int parts)
{
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= instances * parts) return;
    const int i = id % instances, j = id / instances;
    const int B = samples / 6;
    const int b0 = (int)((long long)j * B / parts), b1 = (int)((long long)(j + 1) * B / parts);
    uint32_t x[24], c;
    rl_load(seg + (size_t)j * 7 * instances, instances, i, x, c);
#pragma unroll 1
    for (int bl = b0; bl < b1; bl++) {
        rl_skip<NSKIP>(x, c);
        float4 *o = prns + (size_t)6 * bl * instances + i;
        o[0] = rl_quad<0>(x, c);
        o[(size_t)instances] = rl_quad<1>(x, c);
        o[(size_t)2 * instances] = rl_quad<2>(x, c);
        o[(size_t)3 * instances] = rl_quad<3>(x, c);
        o[(size_t)4 * instances] = rl_quad<4>(x, c);
        o[(size_t)5 * instances] = rl_quad<5>(x, c);
    }
    if (j == parts - 1) rl_store(table, instances, i, x, c);
}

int ranlux_split_parts(int instances, int samples)
{
    if (samples % 6 != 0 || instances < 1) return 1;
    const int B = samples / 6;
    int parts = (1 << 17) / instances;          // about 2^17 threads per batch
    if (parts > B / 8) parts = B / 8;           // at least 8 blocks per segment
    if (parts > 16) parts = 16;
    return parts < 2 ? 1 : parts;
}

void ranlux_split_multipliers(int samples, int nskip, int parts, uint32_t *out)
{
    const int B = samples / 6;
    for (int j = 0; j < parts; j++) {
        const uint64_t steps = (uint64_t)((long long)j * B / parts) * (uint64_t)(nskip + 24);
        uint32_t r[rlx::kLimbs];
        rlx::binv_pow(steps, r);
        for (int k = 0; k < rlx::kLimbs; k++) out[(size_t)j * rlx::kLimbs + k] = r[k];
    }
}

// ranlux_init (prngcl_ranlux.cl:137-157): 24 seed words from the
// 40014/53668 LCG started at the instance's glibc seed; in24 = 6 forces the
// luxury skip before the first output.
__global__ void k_ranlux_init(const uint32_t *seeds, float4 *table, int instances)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= instances) return;
    int32_t j = (int32_t)seeds[i];
    float w[24];
    for (int k = 0; k < 24; k++) {
        int32_t q = j / 53668;
        j = 40014 * (j - q * 53668) - q * 12211;
        if (j < 0) j += 2147483563;
        w[k] = (float)(j % 16777216) * RL_TWOM24;
    }
    for (int k = 0; k < 6; k++)
        table[(size_t)k * instances + i] = make_float4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
    table[(size_t)6 * instances + i] = make_float4(0.0f, 0.0f, 6.0f, (w[23] == 0.0f) ? RL_TWOM24 : 0.0f);
}

cudaError_t launch_ranlux_init(const uint32_t *seeds, float4 *table, int instances, cudaStream_t s)
{
    k_ranlux_init<<<(instances + 127) / 128, 128, 0, s>>>(seeds, table, instances);
    return cudaGetLastError();
}

cudaError_t launch_ranlux_produce(float4 *table, float4 *prns, int instances, int samples, int nskip, cudaStream_t s,
                                  const RanluxSplit *split)
{
    if (split && split->parts > 1) {
        const int P = split->parts;
        const unsigned nbp = (unsigned)(((size_t)instances * P + 127) / 128);
        k_ranlux_jump<<<nbp, 128, 0, s>>>(table, split->seg, instances, P, split->mult);
        switch (nskip) {
        case 24: k_ranlux_seg<24><<<nbp, 128, 0, s>>>(table, split->seg, prns, instances, samples, P); break;
        case 48: k_ranlux_seg<48><<<nbp, 128, 0, s>>>(table, split->seg, prns, instances, samples, P); break;
        case 97: k_ranlux_seg<97><<<nbp, 128, 0, s>>>(table, split->seg, prns, instances, samples, P); break;
        case 223: k_ranlux_seg<223><<<nbp, 128, 0, s>>>(table, split->seg, prns, instances, samples, P); break;
        case 389: k_ranlux_seg<389><<<nbp, 128, 0, s>>>(table, split->seg, prns, instances, samples, P); break;
        default: return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }
    unsigned nb = (instances + 127) / 128;
    switch (nskip) {
    case 24: k_ranlux<24><<<nb, 128, 0, s>>>(table, prns, instances, samples); break;
    case 48: k_ranlux<48><<<nb, 128, 0, s>>>(table, prns, instances, samples); break;
    case 97: k_ranlux<97><<<nb, 128, 0, s>>>(table, prns, instances, samples); break;
    case 223: k_ranlux<223><<<nb, 128, 0, s>>>(table, prns, instances, samples); break;
    case 389: k_ranlux<389><<<nb, 128, 0, s>>>(table, prns, instances, samples); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace qg
