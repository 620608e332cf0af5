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

namespace qg {

#define RL_TWOM24 5.9604644775390625e-8f
#define RL_TWOM12 2.44140625e-4f

// The words are kept as exact 24-bit integers W = word * 2^24 and the
// borrow as 0/1: one subtract-with-borrow step is W_i = W_j - W_i - c,
// c = (W_i < 0), W_i += c * 2^24 -- the float recurrence of the reference
// (u = s[j] - s[i] - carry; u < 0: u += 1, carry = 2^-24) on the same exact
// values, with an integer add and a shift on the borrow chain in place of
// float subtract, compare and select.  Outputs and the table are floats.
__device__ __forceinline__ int32_t rl_step(int32_t (&w)[24], int i, int j, int32_t &c)
{
    int32_t u = w[j] - w[i] - c;
    c = (int32_t)((uint32_t)u >> 31);
    u += c << 24;
    w[i] = u;
    return u;
}

// q-th output of a block: i24 = 23-q, j24 = (9-q) mod 24; the refinement
// reads the word at the decremented j24
template <int Q>
__device__ __forceinline__ float rl_out(int32_t (&w)[24], int32_t &c)
{
    constexpr int I = 23 - Q;
    constexpr int J = (33 - Q) % 24;
    constexpr int JN = (32 - Q) % 24;
    float u = (float)rl_step(w, I, J, c) * RL_TWOM24;
    if (u < RL_TWOM12) {
        u = u + RL_TWOM24 * ((float)w[JN] * RL_TWOM24);
        if (u == 0.0f) u = RL_TWOM24 * RL_TWOM24;
    }
    return u;
}

template <int M>
__device__ __forceinline__ float4 rl_quad(int32_t (&w)[24], int32_t &c)
{
    float4 r;
    r.x = rl_out<4 * M + 0>(w, c);
    r.y = rl_out<4 * M + 1>(w, c);
    r.z = rl_out<4 * M + 2>(w, c);
    r.w = rl_out<4 * M + 3>(w, c);
    return r;
}

template <int NSKIP>
__device__ __forceinline__ void rl_skip(int32_t (&w)[24], int32_t &c)
{
#pragma unroll 1
    for (int r = 0; r < NSKIP / 24; r++) {
#pragma unroll
        for (int q = 0; q < 24; q++) rl_step(w, 23 - q, (33 - q) % 24, c);
    }
    constexpr int R = NSKIP % 24;
#pragma unroll
    for (int q = 0; q < R; q++) rl_step(w, 23 - q, (33 - q) % 24, c);
    if (R) {
        int32_t t[24];
#pragma unroll
        for (int k = 0; k < 24; k++) t[(k + R) % 24] = w[k];
#pragma unroll
        for (int k = 0; k < 24; k++) w[k] = t[k];
    }
}

template <int NSKIP>
__global__ void __launch_bounds__(128) k_ranlux(float4 *table, float4 *prns, int instances, int samples)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= instances) return;
    int32_t w[24];
#pragma unroll
    for (int k = 0; k < 6; k++) {
        float4 v = table[(size_t)k * instances + i];
        w[4 * k] = (int32_t)(v.x * 16777216.0f); w[4 * k + 1] = (int32_t)(v.y * 16777216.0f);
        w[4 * k + 2] = (int32_t)(v.z * 16777216.0f); w[4 * k + 3] = (int32_t)(v.w * 16777216.0f);
    }
    float4 ci = table[(size_t)6 * instances + i];
    int in24 = (int)ci.z;
    int32_t c = ci.w != 0.0f ? 1 : 0;
    for (int n = 0; n < samples; n++) {
        if (in24 >= 6) { rl_skip<NSKIP>(w, c); in24 = 0; }
        float4 out;
        switch (in24) {
        case 0: out = rl_quad<0>(w, c); break;
        case 1: out = rl_quad<1>(w, c); break;
        case 2: out = rl_quad<2>(w, c); break;
        case 3: out = rl_quad<3>(w, c); break;
        case 4: out = rl_quad<4>(w, c); break;
        default: out = rl_quad<5>(w, c); break;
        }
        in24++;
        prns[(size_t)n * instances + i] = out;
    }
#pragma unroll
    for (int k = 0; k < 6; k++)
        table[(size_t)k * instances + i] =
            make_float4((float)w[4 * k] * RL_TWOM24, (float)w[4 * k + 1] * RL_TWOM24, (float)w[4 * k + 2] * RL_TWOM24,
                        (float)w[4 * k + 3] * RL_TWOM24);
    table[(size_t)6 * instances + i] = make_float4(0.0f, 0.0f, (float)in24, c ? RL_TWOM24 : 0.0f);
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

cudaError_t launch_ranlux_produce(float4 *table, float4 *prns, int instances, int samples, int nskip, cudaStream_t s)
{
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
