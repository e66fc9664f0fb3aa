// selector.cuh -- sizes and parameter layout of the schedule-selector MLP.
#pragma once

namespace hpvcd {

constexpr int kFeatures = 16;     // per-batch statistics (k_features)
constexpr int kHidden = 64;       // two hidden layers of 64 units
constexpr int kMaxVariants = 32;  // outputs: one predicted cost per schedule variant
constexpr int kMlpTile = 16;      // samples per CTA of the forward kernel

// Offsets (in parameters) of W1 [H][F], b1 [H], W2 [H][H], b2 [H], W3 [K][H],
// b3 [K] in the flat parameter vector; weights are row-major [out][in].
struct MlpLayout {
    int w1, b1, w2, b2, w3, b3, total;
    __host__ __device__ explicit MlpLayout(int K)
        : w1(0),
          b1(kHidden * kFeatures),
          w2(b1 + kHidden),
          b2(w2 + kHidden * kHidden),
          w3(b2 + kHidden),
          b3(w3 + K * kHidden),
          total(b3 + K) {}
};

}  // namespace hpvcd
