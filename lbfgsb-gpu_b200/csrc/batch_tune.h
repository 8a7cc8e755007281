// batch_tune.h -- tiles per CTA of the batched passes by instance size, the table that
// lbfgsb-gpu_b200/autotune.py writes after timing batched solves on the GPU.
// Buckets: n <= 4096, <= 16384, <= 65536, <= 262144, larger.
#pragma once

namespace lbfgsb_b200 {
constexpr int kTuneBuckets = 5;
constexpr int kTunedTilesPerCta[kTuneBuckets] = {128, 1024, 64, 128, 32};
}  // namespace lbfgsb_b200
