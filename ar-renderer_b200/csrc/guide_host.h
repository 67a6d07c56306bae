// Host-side interface of the guide network's kernels (guide.cu) for the path tracer's driver.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "device.cuh"
#include "guide.cuh"

namespace prb {

// Makes the device's guide state ready; reset (or a first use) draws fresh weights from `seed`.
void guide_prepare(DeviceState &ds, int device, bool reset, uint64_t seed);
// Inference over the rows of `features` (FP16, [n x 128]); n is read from dcount on the device,
// maxRows bounds it. out: FP32 [n x 48].
void guide_infer_rows(cudaStream_t st, int device, const __half *features, const int *dcount, int maxRows, float *out);
// One online training step (forward, backward, Adam at learning rate lr, or the device's setting
// when lr <= 0) on records [offset, offset + maxRows) of the
// recorded samples (count on the device); weights are normalised to mean 1 within the batch.
void guide_train_records(cudaStream_t st, int device, const GuideTrainRec *recs, const int *dcount, int offset,
                         int maxRows, float lr);
// The device's sampling and training settings (prgpu_guide_set_options) and learning rate.
GuideOpts guide_options(int device);
float guide_learning_rate(int device);
// Allocates the staging buffers of guide_train_records for batches of up to maxRows, so that its
// launches can be captured into a graph (no allocation during capture); their address.
void guide_reserve_training(int device, int maxRows);
const void *guide_training_buffer(int device);
// True (and cleared) when a guide kernel gave up waiting for its tensor-core work.
bool guide_failed(DeviceState &ds, int device);
// Launch bookkeeping: kernels per inference / training step.
constexpr int kGuideInferLaunches = 1, kGuideTrainLaunches = 5;

} // namespace prb
