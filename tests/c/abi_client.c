/*
 * A plain C99 caller of the library, as a host written in another language
 * would bind it: both headers compile as C, the libraries link by name, and
 * one task runs through create / init / sweep / measure / destroy.
 *
 *   abi_client L T seed sweeps   prints "version", then "energy E m2 M accepted A"
 *
 * Exit status: 0 on success; 3 when the library reports that no CUDA device
 * is available (its message goes to stderr); 1 on any other error.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "slsf_gpu.h"
#include "slsf_host.h"

static int fail(const char* what) {
    char msg[512];
    slsf_last_error(msg, sizeof msg);
    fprintf(stderr, "%s: %s\n", what, msg);
    return strstr(msg, "no CUDA device") ? 3 : 1;
}

int main(int argc, char** argv) {
    if (argc != 5) {
        fprintf(stderr, "usage: %s L T seed sweeps\n", argv[0]);
        return 1;
    }
    const uint32_t L = (uint32_t)atoi(argv[1]);
    const double T = atof(argv[2]);
    const uint64_t seed = (uint64_t)strtoull(argv[3], NULL, 10);
    const uint32_t sweeps = (uint32_t)atoi(argv[4]);
    printf("version %s\n", slsf_version());
    /* the reference's run seed formula is exported by the host library */
    printf("run seed of task 1 at L=%u: %llu\n", L,
           (unsigned long long)slsf_task_seed(seed, L, 1, T, 0.0, 0.0));

    slsf_ctx* ctx = NULL;
    if (slsf_ctx_create(0, 0, 0, &ctx) != SLSF_OK) return fail("slsf_ctx_create");
    double* jxy = malloc(sizeof(double) * L);
    double* jz = malloc(sizeof(double) * L);
    for (uint32_t z = 0; z < L; ++z) {
        jxy[z] = 1.2;
        jz[z] = 0.5 + (double)z / (double)L;
    }
    slsf_task_desc d;
    memset(&d, 0, sizeof d);
    d.lx = d.ly = d.lz = L;
    d.temperature = T;
    d.proposal_width = 3.141592653589793;
    d.wolff_steps = 1;
    d.seed = seed;
    d.j_xy = jxy;
    d.n_j_xy = L;
    d.j_z = jz;
    d.n_j_z = L;
    slsf_task* task = NULL;
    int rc = 0;
    if (slsf_task_create(ctx, &d, &task) != SLSF_OK) {
        rc = fail("slsf_task_create");
    } else {
        slsf_sweep_stats st;
        slsf_observables o;
        if (slsf_task_init_random(task) != SLSF_OK) rc = fail("slsf_task_init_random");
        else if (slsf_task_sweep(task, sweeps, &st) != SLSF_OK) rc = fail("slsf_task_sweep");
        else if (slsf_task_measure(task, &o) != SLSF_OK) rc = fail("slsf_task_measure");
        else
            printf("energy %.17g m2 %.17g accepted %llu\n", o.energy, o.magnetization_squared,
                   (unsigned long long)st.accepted);
        slsf_task_destroy(task);
    }
    slsf_ctx_destroy(ctx);
    free(jxy);
    free(jz);
    return rc;
}
