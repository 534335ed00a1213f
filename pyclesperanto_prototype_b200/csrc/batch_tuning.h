// batch_tuning.h -- lane counts of the batched form per batch size class,
// written by pyclesperanto_prototype_b200/autotune.py from measurements
// (cle_vol_batch_plan with lanes = 0 reads it).  A class applies to batches
// whose mean tile voxel count is at least min_mean_voxels; the last class
// that applies wins.
#pragma once

namespace cle {

struct BatchTuning {
    double min_mean_voxels;
    int lanes;
};

static const BatchTuning kBatchTuning[] = {
    {0.0, 16},   // 64x64 x 256 tiles; Mvoxels/s by lanes {1: 35, 2: 47, 4: 102, 8: 155, 12: 158, 16: 182}
    {16384.0, 16},   // 256x256 x 256 tiles; Mvoxels/s by lanes {1: 389, 2: 646, 4: 1349, 8: 2255, 12: 2007, 16: 2401}
    {185363.8, 16},   // 32x128x128 x 256 tiles; Mvoxels/s by lanes {1: 1818, 2: 2714, 4: 4780, 8: 6337, 12: 5875, 16: 6640}
    {1482910.4, 8},   // 64x256x256 x 47 tiles; Mvoxels/s by lanes {1: 8717, 2: 13283, 4: 17601, 8: 20245, 12: 16860, 16: 18233}
    {10273904.6, 4},   // 96x512x512 x 7 tiles; Mvoxels/s by lanes {1: 16360, 2: 18194, 4: 18498}
};

}  // namespace cle
