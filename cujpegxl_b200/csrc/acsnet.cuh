// Transform-decision network: a 4-layer convolutional network over one 32x32
// region of XYB pixels (with a 1-pixel ring of its neighbours, clamped at the
// image border) that predicts the region's DCT32/DCT16/DCT8 split (17
// classes) and the log2 quant field of each of its 16 blocks.
//
// Layers (BF16 weights and activations, FP32 accumulation):
//   L1  3x3 stride 2   8 -> 32 channels   34x34 -> 16x16   ReLU (no padding)
//   L2  3x3 stride 2  32 -> 32            16x16 ->  8x8    ReLU
//   L3  3x3 stride 2  32 -> 32             8x8  ->  4x4    ReLU
//   L4  3x3 stride 1  32 -> 32             4x4  ->  4x4    (linear)
// (L2..L4 zero-pad by 1.)
// Input channels: X, Y, B and log2(distance), each normalised as
// (v - shift) * scale, then four zero channels. Output channel 0 of L4 at
// block position p is the block's log2 quant field; channels 1..17 averaged
// over the 16 positions are the split logits; channels 18..31 are unused
// (their weights stay zero).
//
// Split classes: 0 = one DCT32; 1 + m = four quadrants in raster order, bit q
// of m set when quadrant q is four DCT8 blocks and clear when it is one DCT16.
#pragma once

#include <cstddef>
#include <cstdint>

namespace jxb {

constexpr int kNetInW = 34;      // input side: the region and a 1-pixel ring
constexpr int kNetInPix = kNetInW * kNetInW;
constexpr int kNetC = 32;        // output channels of every layer
constexpr int kNetIn = 8;        // stored input channels
constexpr int kNetClasses = 17;
constexpr int kNetK1 = 80;       // L1 reduction: 9 taps x 8 channels + 8 zero columns
constexpr int kNetK = 288;       // L2..L4 reduction: 9 taps x 32 channels
constexpr int kNetOut = kNetClasses + 16;  // per region: 17 logits, 16 log2 quant fields

// Parameter vector, canonical order: W1[32][80], W2..W4[32][288] (row = output
// channel, column = tap * Cin + input channel, tap = ky * 3 + kx), then the
// four bias vectors [4][32].
constexpr int kNetW1 = 0;
constexpr int kNetW2 = kNetW1 + kNetC * kNetK1;
constexpr int kNetW3 = kNetW2 + kNetC * kNetK;
constexpr int kNetW4 = kNetW3 + kNetC * kNetK;
constexpr int kNetWeights = kNetW4 + kNetC * kNetK;  // 30208
constexpr int kNetBias = kNetWeights;
constexpr int kNetParams = kNetBias + 4 * kNetC;     // 30336

// Weights as the kernels read them.
struct NetParamsDev {
    const std::uint16_t* w;  // [kNetWeights] BF16 bit patterns, canonical order
    const float* bias;       // [4][32]
    float scale[4];          // input normalisation (X, Y, B, log2 distance)
    float shift[4];
};

// Per-sample activations kept by the training forward/backward kernel for the
// weight-gradient kernel (BF16, compact [position][channel]).
constexpr int kNetActX1 = 0;                       // [34*34][8]
constexpr int kNetActX2 = kNetActX1 + kNetInPix * 8;  // [256][32]
constexpr int kNetActX3 = kNetActX2 + 256 * 32;    // [64][32]
constexpr int kNetActX4 = kNetActX3 + 64 * 32;     // [16][32]
constexpr int kNetActG1 = kNetActX4 + 16 * 32;     // [256][32] dL/d(L1 pre-activation)
constexpr int kNetActG2 = kNetActG1 + 256 * 32;    // [64][32]
constexpr int kNetActG3 = kNetActG2 + 64 * 32;     // [16][32]
constexpr int kNetActG4 = kNetActG3 + 16 * 32;     // [16][32] dL/d(L4 output)
constexpr int kNetActPerSample = kNetActG4 + 16 * 32;  // 31264 BF16 values

// One training or evaluation batch in device memory.
struct NetBatchDev {
    const float* tiles;          // [ntiles][3][34][34] XYB
    const std::int32_t* tile_index;  // [n] tile of each sample
    const float* log2_distance;  // [n]
    const std::int8_t* label_class;  // [n] or null (forward only)
    const float* label_qf;       // [n][16] log2 quant field, or null
    const float* label_soft;     // [n][17] target distribution replacing the one-hot class, or null
    std::uint32_t n;
};

// Inference inside an encode: the decisions of every region of the frame.
struct NetDecisionsDev {
    std::int8_t* cls;    // [rh][rw] split class, -1 where the heuristic decides
    std::int16_t* qf;    // [bh][bw] quant field of blocks in decided regions
    // Null, or [ntiles + 2]: the raster indices of the 64x64 tiles, those
    // whose regions inside the image are all decided from the front, the
    // others from the back (the last two words count them).
    std::uint32_t* tile_order;
};

struct FrontendInputs;

// Launches the inference kernel over the frame of `in` (one CTA per 64x64
// tile, as the frontend). Regions that are not a full 32x32 inside the image,
// and regions whose top-two softmax margin is below `margin`, get class -1.
bool acsnet_infer_launch(const FrontendInputs& in, const NetParamsDev& p, float log2_distance, float margin,
                         const NetDecisionsDev& out, void* stream);

bool acsnet_kernels_init();

}  // namespace jxb
