// Batched mixed-precision sweeps of many small systems in one persistent
// launch (fh_batchsolve.cu) and the autotuner that picks their tile shapes
// (fh_batchtune.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "fh_internal.h"

namespace fhb {

// One system on the device: R_m, L_m (column-major, leading dimension ld),
// m internal loops and p ports.
struct BatchSys {
    const double *R = nullptr, *L = nullptr;
    int64_t ld = 0, m = 0, p = 0;
};

// One (system, frequency) work item.
struct BatchItem {
    int32_t sys = 0;
    int32_t cfg = 0;       // tile configuration (kBatchConfigs)
    double omega = 0.0;
    int64_t z_offset = 0;  // complex entries into the batch's Z array
    int32_t index = 0;     // position in the caller's item order (status slot)
    int32_t pad = 0;
};

// Tile configurations: panel width NB x trailing tile TILE.
constexpr int kBatchConfigs = 4;
constexpr int kBatchNb[kBatchConfigs] = {16, 16, 32, 32};
constexpr int kBatchTile[kBatchConfigs] = {32, 64, 32, 64};

size_t batch_smem_bytes();
size_t batch_slot_bytes(int64_t mmax, int pmax);
// Persistent CTAs that fit the device at once.
int batch_resident_ctas();
// One launch over all items (sorted by cost, largest first).  status[index]
// receives the refinement iterations, or -1 for an item that must be redone
// in FP64 (zero pivot, or refinement without convergence).
fh_status batch_launch(const BatchSys *d_systems, const BatchItem *d_items, int nitems, unsigned *d_counter,
                       void *d_work, size_t slot_bytes, int64_t mmax, int pmax, double2 *d_z, int32_t *d_status,
                       int ctas, cudaStream_t s, fh_error_info *err);

// The autotuner's table: the best configuration per order bucket (orders
// 128 (b - 1) < m <= 128 b), measured on this device on first use and kept
// in a JSON file (FH_AUTOTUNE_CACHE, else $XDG_CACHE_HOME or
// $HOME/.cache/fasterhenry_b200/batch_tiles.json).
struct BatchTuner {
    static int bucket_of(int64_t m) { return (int)((m + 127) / 128); }
    // The configuration for order m; tunes the bucket on first use with the
    // given system (items of one frequency, timed with one CTA).
    fh_status config_for(const BatchSys &sys, const BatchSys *d_sys_one, cudaStream_t s, int *cfg,
                         fh_error_info *err);
    std::string cache_path() const;
    int tuned_now = 0;  // buckets measured by this process
};
BatchTuner &batch_tuner();

}  // namespace fhb
