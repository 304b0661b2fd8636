// Fused frontend: one CTA per 64x64 chroma-from-luma tile runs
// NV12 -> XYB -> adaptive quant field -> inverse gaborish -> transform
// selection -> variable DCT -> chroma-from-luma -> quantisation, keeping every
// intermediate in shared memory. Only the NV12 tile (plus a 2-pixel halo) is
// read from HBM and only the quantised planes and side information are
// written back.
#pragma once

#include <cstddef>
#include <cstdint>

namespace jxb {

// Distance-derived scalars, computed on the host exactly as the reference's
// host code does (src/frontend_fused.cu:349-380, src/quant_calibration.h:49-88,
// src/frontend_quantize.cu:251-260, src/transform_select.cu:470-479).
struct FrontendScalars {
    float km0, km1, km2, km3;  // FuzzyErosion weights
    float mul_pb, add_pb;      // per-block modulation -> field mapping
    float inv_global_scale;    // 2^16 / global_scale
    float mask_sqrt_mul;       // sqrtf(211.66567973503678f * 1e8f)
    float qgsf_select;         // raw_quant_field * global_scale / 2^16 (selection proxy)
    float gsf;                 // global_scale / 2^16
    float dc_scale;            // gsf * quant_dc
};

// Device outputs of the frontend for one frame (B = (W/8)*(H/8) blocks,
// T = ceil(W/64)*ceil(H/64) colour tiles). All planes are block-raster.
struct FrontendOutputs {
    std::int16_t* ac;     // [3][B*64] quantised AC, covered-block layout, X,Y,B
    std::int32_t* dc;     // [3][B] quantised DC, X,Y,B
    std::int8_t* acs;     // [B] 8/16/32 at first-blocks, 0 at covered blocks
    std::int32_t* qf;     // [B] adaptive quant field (1..256)
    std::int8_t* ytox;    // [T]
    std::int8_t* ytob;    // [T]
    std::uint8_t* nzn;    // [3][B] normalised non-zero count, written at every covered position
    std::uint16_t* nzc;   // [3][B] non-zero AC count at first-blocks (0 elsewhere)
    // Optional stage dumps for tests (null in production).
    float* dbg_xyb;       // [3][H][W] XYB before sharpening
    float* dbg_sharp;     // [3][H][W] XYB after inverse gaborish
    std::uint16_t* dbg_coeff;  // [3][B*64] FP16 bit patterns, covered-block layout
    float* dbg_cost;      // [3][B] selection costs: DCT8, DCT16 at quad and DCT32 at region first blocks
};

struct FrontendInputs {
    const std::uint8_t* luma;
    const std::uint8_t* chroma;
    std::size_t luma_pitch;
    std::size_t chroma_pitch;
    int width;
    int height;
    // Learned decisions (both null without a network): the split class of
    // every 32x32 region ([ceil(bh/4)][ceil(bw/4)], -1 where the RD heuristic
    // decides) and, if net_qf is set, the quant field of the blocks of
    // decided regions ([bh][bw]).
    const std::int8_t* net_class;
    const std::int16_t* net_qf;
    // Null, or the order in which the single-frame kernel takes the 64x64
    // tiles (raster indices; its CTA b runs entries 2b and 2b + 1): with
    // learned decisions, the tiles whose regions are all decided come first,
    // so that a CTA's two tiles, which it waits for together, cost alike.
    const std::uint32_t* tile_order;
};

// Read-only tables in device memory (built once per device by
// frontend_tables_init).
// Offset of the reciprocals RN(1 / w) that follow the dequantisation weights.
constexpr int kDequantInv = 3 * 3 * 1024;

struct FrontendTables {
    const float* dequant;     // [3 sizes][3 ch][1024] stride 1024 (size 8, 16, 32), then their reciprocals
    const float* sel_weight;  // [3 sizes][1024] DCT8 Y weight sampled at round(f*8/N)
    const float* log2_1p;     // [kLog2TableSize] log2f(1 + i)
    const double* llf_basis;  // [2][4][4] orthonormal m-point basis for m = 2, 4
};

constexpr int kLog2TableSize = 1 << 19;

// Builds the constant-memory bases and the device tables for the current
// device. Returns false on a CUDA error.
bool frontend_tables_init(FrontendTables* tables);

FrontendScalars frontend_scalars(float distance, std::uint32_t* global_scale,
                                 std::uint32_t* quant_dc);

// Launches the fused frontend on `stream`.
bool frontend_launch(const FrontendInputs& in, const FrontendScalars& s, const FrontendTables& t,
                     const FrontendOutputs& out, void* stream);

// Frames of one batched frontend launch (the launch's parameter block holds
// them, so one launch takes at most kBatchFrames frames).
constexpr int kBatchFrames = 64;

struct FrontendJob {
    FrontendInputs in;
    FrontendScalars sc;
    FrontendOutputs out;
    int tiles_x;               // 64x64 tiles per row
    std::uint32_t tile_begin;  // first work item of the frame
};

struct FrontendBatch {
    FrontendTables tb;
    int nframes;
    int chunk;                   // tiles per claim
    std::uint32_t total_tiles;
    std::uint32_t* counter;      // claim counter, zero at launch; null: static round-robin claims
    FrontendJob jobs[kBatchFrames];
};

// Launches `ctas` resident CTAs that run every tile of every frame in `b`:
// paired, CTAs of two tiles at a time (one per half, claimed together; one
// CTA per SM), else CTAs of one tile at a time (two per SM).
bool frontend_batch_launch(const FrontendBatch& b, int ctas, bool paired, void* stream);

}  // namespace jxb
