/*
 * Per-task binning of the measurement stream on the device, shared by the
 * batched kernels.  ThetaModel::measure records, after every sweep past
 * thermalization, Energy, EnergySquared, MagnetizationSquared and the
 * helicity cos / sin / sin^2 sums (src/model.rs:406-409, :890-904); carlo-mc
 * averages them in bins of `binsize` measurements.  A task's bins hold the
 * column sums of each bin (kBinCols columns, engine.h).
 */
#ifndef SLSF_BINS_CUH
#define SLSF_BINS_CUH

#include "engine.h"

namespace slsf {

/* Adds the measurement of the state after `done` sweeps (sums a = mx, my,
 * cos xyz, sin xyz of a `volume`-site lattice) to the task's bins.  One
 * thread per task calls it; bin_acc collects the current bin in shared
 * memory and is flushed to the task's bins when the bin changes (and once
 * more by flush_bin at the end of the launch). */
__device__ __forceinline__ void bin_measurement(const TaskView& t, uint32_t volume, uint64_t done,
                                                const double (&a)[8], double* bin_acc, int64_t& bin_cur) {
    const int64_t b = (int64_t)((done - t.thermalization - 1) / t.binsize);
    if (b != bin_cur) {
        if (bin_cur >= 0 && bin_cur < (int64_t)t.n_bins)
            for (int q = 0; q < kBinCols; ++q) t.bins[bin_cur * kBinCols + q] += bin_acc[q];
        for (int q = 0; q < kBinCols; ++q) bin_acc[q] = 0.0;
        bin_cur = b;
    }
    const double v = (double)volume;
    const double e = -(a[2] + a[3] + a[4]) / v;
    const double vals[kBinCols] = {e,    e * e, (a[0] * a[0] + a[1] * a[1]) / (v * v),
                                   a[2], a[3],  a[4],
                                   a[5], a[6],  a[7],
                                   a[5] * a[5], a[6] * a[6], a[7] * a[7]};
    for (int q = 0; q < kBinCols; ++q) bin_acc[q] += vals[q];
}

__device__ __forceinline__ void flush_bin(const TaskView& t, const double* bin_acc, int64_t bin_cur) {
    if (bin_cur >= 0 && bin_cur < (int64_t)t.n_bins)
        for (int q = 0; q < kBinCols; ++q) t.bins[bin_cur * kBinCols + q] += bin_acc[q];
}

}  // namespace slsf

#endif /* SLSF_BINS_CUH */
