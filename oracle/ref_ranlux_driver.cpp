// Test infrastructure only: drives the reference's own host-side RANLUX
// (random/random.cpp, PRNG::initialize_CPU + PRNG::produce_CPU, built from the
// reference sources with -D CPU_RUN) and prints the first N outputs of the
// stream that the reference assigns to generator instance 0, as hex floats.
// Usage: ref_ranlux <randseries> <luxury 0..4> <count>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#define private public
#include "random/random.h"
#undef private

int main(int argc, char **argv)
{
    if (argc < 4) { fprintf(stderr, "usage: %s randseries luxury count\n", argv[0]); return 2; }
    PRNG_CL::PRNG prng;
    prng.PRNG_randseries = atoi(argv[1]);
    int lux = atoi(argv[2]);
    const PRNG_CL::PRNG::PRNG_generators gens[5] = {
        PRNG_CL::PRNG::PRNG_generator_RANLUX0, PRNG_CL::PRNG::PRNG_generator_RANLUX1,
        PRNG_CL::PRNG::PRNG_generator_RANLUX2, PRNG_CL::PRNG::PRNG_generator_RANLUX3,
        PRNG_CL::PRNG::PRNG_generator_RANLUX4 };
    if (lux < 0 || lux > 4) return 2;
    prng.PRNG_generator = gens[lux];
    prng.initialize_CPU();
    int n = atoi(argv[3]);
    float *buf = (float *)calloc(n, sizeof(float));
    prng.produce_CPU(buf, n);
    printf("jseed %d nskip %d\n", prng.RL_jseed, prng.RL_nskip);
    for (int i = 0; i < n; i++) printf("%a\n", (double)buf[i]);
    free(buf);
    return 0;
}
