/*
 * Prints the size and field offsets of every struct the C ABI passes, as the
 * C compiler lays them out, one line per struct:
 *   name sizeof field:offset field:offset ...
 * tests/test_c_client.py compares them with the Python ctypes structs and
 * with the #[repr(C)] structs of the Rust binding in INTEGRATION.md.
 */
#include <stddef.h>
#include <stdio.h>

#include "slsf_gpu.h"

#define F(T, f) printf(" %s:%zu", #f, offsetof(T, f))

int main(void) {
    printf("slsf_task_desc %zu", sizeof(slsf_task_desc));
    F(slsf_task_desc, lx); F(slsf_task_desc, ly); F(slsf_task_desc, lz);
    F(slsf_task_desc, temperature); F(slsf_task_desc, proposal_width); F(slsf_task_desc, wolff_steps);
    F(slsf_task_desc, seed); F(slsf_task_desc, j_xy); F(slsf_task_desc, n_j_xy); F(slsf_task_desc, j_z);
    F(slsf_task_desc, n_j_z); F(slsf_task_desc, thermalization); F(slsf_task_desc, binsize);
    F(slsf_task_desc, n_bins);
    printf("\nslsf_observables %zu", sizeof(slsf_observables));
    F(slsf_observables, energy); F(slsf_observables, magnetization_squared); F(slsf_observables, cos_x);
    F(slsf_observables, cos_y); F(slsf_observables, cos_z); F(slsf_observables, sin_x);
    F(slsf_observables, sin_y); F(slsf_observables, sin_z);
    printf("\nslsf_sweep_stats %zu", sizeof(slsf_sweep_stats));
    F(slsf_sweep_stats, sweeps); F(slsf_sweep_stats, accepted); F(slsf_sweep_stats, wolff_clusters);
    F(slsf_sweep_stats, wolff_cluster_sites);
    printf("\nslsf_kernel_choice %zu", sizeof(slsf_kernel_choice));
    F(slsf_kernel_choice, kind); F(slsf_kernel_choice, cluster); F(slsf_kernel_choice, threads);
    printf("\n");
    return 0;
}
