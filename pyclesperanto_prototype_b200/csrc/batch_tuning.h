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
    {0.0, 16},   // 64x64 x 256 tiles; Mvoxels/s by lanes {1: 27, 2: 52, 4: 103, 8: 173, 12: 152, 16: 198}
    {16384.0, 16},   // 256x256 x 256 tiles; Mvoxels/s by lanes {1: 208, 2: 383, 4: 739, 8: 1399, 12: 1126, 16: 1460}
    {185363.8, 16},   // 32x128x128 x 256 tiles; Mvoxels/s by lanes {1: 722, 2: 1375, 4: 2621, 8: 4594, 12: 3898, 16: 4787}
    {1482910.4, 8},   // 64x256x256 x 47 tiles; Mvoxels/s by lanes {1: 6074, 2: 10318, 4: 15401, 8: 19116, 12: 17063, 16: 17449}
    {10273904.6, 4},   // 96x512x512 x 7 tiles; Mvoxels/s by lanes {1: 13956, 2: 16871, 4: 17555}
};

}  // namespace cle
