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

// initial table (8 lanes measured best on the mixed 2D/3D tile batch before
// the tuner ran); regenerated by autotune.py
static const BatchTuning kBatchTuning[] = {
    {0.0, 8},
};

}  // namespace cle
