// The learned far-field closure: shapes shared by its kernels (k_closure.cu)
// and the runtime.
//
// The closure has no counterpart in the reference.  On top of the order-1
// local expansion of the traversal (GRAD mode of k_traverse.cu) a small MLP
// predicts, per particle, the far-field force error left by the expansion,
// from the leaf's field L, field gradient G, the particle's offset in the
// leaf and the leaf's depth.  A sampled FP64 direct sum judges every tick
// whether the correction helps; otherwise the uncorrected forces stand.
//
// Network: 16 inputs (13 used) -> 64 -> 64 -> 64 -> 8 outputs (3 used), GELU
// (tanh form) after each hidden layer.  Weights BF16, biases and all
// accumulation FP32.
#pragma once

#include <cstdint>

namespace psg {

constexpr int kMlpIn = 16;
constexpr int kMlpInUsed = 13;
constexpr int kMlpHid = 64;
constexpr int kMlpOut = 8;
constexpr int kMlpOutUsed = 3;
constexpr float kMlpOutScale = 0.01f;  // dF = m * s * kMlpOutScale * y
constexpr int kJudgeSamples = 4096;  // the judge's largest sample
constexpr int kJudgeDefault = 1024;  // its sample unless set

// FP32 parameter vector, the layout every entry point uses:
//   W1[16][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64][8] b4[8]
// (W[in][out]; inputs 13..15 and outputs 3..7 are padding)
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpIn * kMlpHid;
constexpr int kOffW2 = kOffB1 + kMlpHid;
constexpr int kOffB2 = kOffW2 + kMlpHid * kMlpHid;
constexpr int kOffW3 = kOffB2 + kMlpHid;
constexpr int kOffB3 = kOffW3 + kMlpHid * kMlpHid;
constexpr int kOffW4 = kOffB3 + kMlpHid;
constexpr int kOffB4 = kOffW4 + kMlpHid * kMlpOut;
constexpr int kMlpParams = kOffB4 + kMlpOut;  // 9928

// Device copy used by the kernels: transposed BF16 weights Wt[out][in] with
// padded rows (conflict-free B-fragment loads), FP32 biases.
constexpr int kLd1 = 24;  // row stride (bf16) of Wt1 (16 inputs)
constexpr int kLdH = 72;  // row stride of Wt2, Wt3, Wt4 (64 inputs)
struct MlpPacked {
    uint16_t wt1[kMlpHid * kLd1];
    uint16_t wt2[kMlpHid * kLdH];
    uint16_t wt3[kMlpHid * kLdH];
    uint16_t wt4[kMlpOut * kLdH];
    float b1[kMlpHid];
    float b2[kMlpHid];
    float b3[kMlpHid];
    float b4[kMlpOut];
};

// what the judge reports for a tick
struct JudgeOut {
    double median_base;  // median relative error of the order-1 forces
    double median_mlp;   // ... with the learned correction added
    int use_mlp;         // 1: the correction was applied
    int samples;
};

}  // namespace psg
