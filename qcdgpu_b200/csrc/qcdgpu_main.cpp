// qcdgpu -- command-line run driver, the counterpart of the reference's
// QCDGPU executable (SU(N)/QCDGPU.cpp:61-269): defaults, then the keys of
// the init file given as the first argument, then one run on the current
// CUDA device with its results file.
#include <stdio.h>
#include <string.h>

#include "../../include/qcdgpu_b200.h"

int main(int argc, char **argv)
{
    qg_config cfg;
    qg_run_options opts;
    qg_default_config(&cfg);
    qg_default_run_options(&opts);
    if (argc > 1 && qg_parse_init_file(argv[1], &cfg, &opts) != QG_OK) {
        fprintf(stderr, "qcdgpu: %s\n", qg_last_error(NULL));
        return 1;
    }
    qg_run_result res;
    if (qg_run(&cfg, &opts, &res) != QG_OK) {
        fprintf(stderr, "qcdgpu: %s\n", qg_last_error(NULL));
        return 1;
    }
    printf("\n Mean Plq_total %.13e  Mean S_total %.13e  Mean Polyakov_loop %.13e\n", res.mean[QG_OBS_PLQ_TOTAL],
           res.mean[QG_OBS_S_TOTAL], res.mean[QG_OBS_POLYAKOV]);
    printf(" %.3f s, %.4e link updates/s%s%s\n", res.seconds, res.link_updates_per_second,
           res.results_file[0] ? ", results in " : "", res.results_file);
    return res.verification_passed == 0 ? 2 : 0;
}
