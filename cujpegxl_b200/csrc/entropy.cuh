// Device entropy coding and frame assembly: quantised planes -> .jxl bytes in
// device memory, with no host round trip.
//
// The codestream is modelled as a list of sections (DcGlobal, the DcGroups,
// AcGlobal, the AcGroups, in TOC order), each a list of "items" whose bit
// lengths are data dependent but whose number is fixed by the frame geometry:
// a header blob, one AC block-channel, one DC sample, one AcMetadata sample.
// Per frame:
//   1. token pass over all items: the AC stripes' tokens are counted into
//      the 32 cluster histograms and stored once in a token pool; the other
//      items fill the per-DC-group DC and AcMetadata histograms;
//   2. prefix codes built on the device, one warp per histogram;
//   3. bit-length pass over all items, then a two-level exclusive scan;
//   4. a layout CTA sizes every section, writes the container, headers and
//      TOC, and places the sections;
//   5. an emit pass writes every item's bits at its final position.
// Passes 1, 3 and 5 are one launch each: a CTA per AC stripe (one warp per
// block-channel while tokenising, stored tokens afterwards), then a CTA per
// 512 other items (two per thread); passes 3 and 5 take stripes whose
// tokens did not fit the pool in one more launch each, with their
// coefficients staged again. A clear kernel zeroes the histograms and the
// pool fill first.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

namespace jxb {

enum SectionKind : int { kSecDcGlobal = 0, kSecDcGroup = 1, kSecAcGlobal = 2, kSecAcGroup = 3 };

struct Section {
    std::uint32_t first;   // first global item index
    std::uint32_t count;   // items in the section
    int kind;
    int group;             // DC or AC group index
};

// Up to kStripeRows block rows of one AC group: the unit one CTA stages in
// shared memory for the AC passes. Rows start at multiples of 4 inside the
// group, so every DCT16/DCT32 transform lies inside one stripe.
constexpr int kStripeRows = 4;
struct Stripe {
    std::uint32_t item0;   // global index of the stripe's first item
    std::int32_t section;  // section index of the AC group
    std::uint16_t group;   // AC group index
    std::uint8_t r0;       // first block row inside the group
    std::uint8_t rows;     // block rows, 1..kStripeRows
};

// Geometry and per-frame device state of the entropy stage. All pointers are
// device memory owned by the encoder.
struct EntropyDev {
    // geometry
    int width, height, bw, bh, nblocks, xg, nac, xdg, ndc, cmw, nsec;
    std::uint32_t total_items;
    std::uint32_t ac_first;          // first item of the first AcGroup; AC block-channels follow
    std::uint32_t num_tiles;         // scan tiles of kScanTile items
    const Section* sections;
    const Stripe* stripes;
    int nstripes;

    // inputs (frontend outputs)
    const std::int16_t* ac;
    const std::int32_t* dc;
    const std::int8_t* acs;
    const std::int32_t* qf;
    const std::int8_t* ytox;
    const std::int8_t* ytob;
    const std::uint8_t* nzn;
    const std::uint16_t* nzc;

    // constant tables
    const std::uint16_t* order;      // natural orders: 64 (DCT8) | 256 (DCT16) | 1024 (DCT32)
    const std::uint8_t* pre_const;   // DcGroup header bits before the DC code description
    std::uint32_t pre_const_bits;
    const std::uint8_t* mid_const;   // AcMetadata header bits after the count field
    std::uint32_t mid_const_bits;
    const std::uint8_t* ac_prefix;   // AcGlobal bits before the per-cluster sizes
    std::uint32_t ac_prefix_bits;
    const std::uint8_t* dc_global;   // DcGlobal section bits (per distance)
    std::uint32_t dc_global_bits;

    // per-frame scratch
    std::uint32_t* ac_hist;          // [32][256]
    std::uint32_t* dc_hist;          // [ndc][256]
    std::uint32_t* am_hist;          // [ndc][256]
    std::uint32_t* fb_count;         // [ndc]
    std::uint8_t* ac_depth;          // [32][256]
    std::uint16_t* ac_bits;
    std::uint8_t* dc_depth;          // [ndc][256]
    std::uint16_t* dc_bits;
    std::uint8_t* am_depth;          // [ndc][256]
    std::uint16_t* am_bits;
    std::uint32_t* ac_alpha;         // [32]
    std::uint8_t* desc;              // [32 + 2*ndc][kDescBytes] code descriptions
    std::uint32_t* desc_bits;        // [32 + 2*ndc]
    std::uint32_t* item_bits;        // [total_items]
    std::uint32_t* item_pre;         // [total_items] exclusive prefix within its scan tile
    std::uint32_t* tile_sum;         // [num_tiles]
    unsigned long long* tile_off;    // [num_tiles + 1]
    unsigned long long* sec_pos;     // [nsec] absolute bit offset of each section in `out`
    unsigned long long* result;      // [4]: total bytes, body start, status, 0

    // AC tokens, written once by the histogram pass and read by the bit-length
    // and emission passes: each stripe reserves a contiguous run of the pool
    // (stream order); a stripe that finds the pool full keeps its tokens
    // unstored and the later passes tokenise its coefficients again.
    std::uint32_t* tok_pool;         // [tok_capacity] packed tokens (pack_ac_token)
    std::uint32_t tok_capacity;
    std::uint32_t* tok_count;        // [1] pool fill, zeroed per frame
    std::uint32_t* stripe_tok;       // [2 * nstripes]: pool offset or kNoTokens, token count
    std::uint8_t* out;               // output buffer (container + codestream)
    std::size_t out_capacity;
};

constexpr int kDescBytes = 256;
constexpr int kScanTile = 4096;
// Token pool capacity per 8x8 block: 4K frames at distance 0.5 use about 27,
// at distance 1 about 11.
constexpr std::uint32_t kTokensPerBlock = 32;
constexpr std::uint32_t kNoTokens = 0xffffffffu;

// Shared memory of the layout kernel: one 32-bit size per section, then the
// codestream header, which is at most 64 bytes before the TOC plus 4 bytes
// per TOC entry.
__host__ __device__ constexpr std::uint32_t layout_sizes_bytes(int nsec) {
    return (static_cast<std::uint32_t>(nsec) * 4 + 15) & ~15u;
}
__host__ __device__ constexpr std::uint32_t layout_head_bytes(int nsec) {
    return 64 + static_cast<std::uint32_t>(nsec) * 4;
}
constexpr std::uint32_t kLayoutSmemLimit = 200 * 1024;
constexpr int kMaxSections = static_cast<int>(kLayoutSmemLimit / 8) - 16;

// Builds the constant header blobs and section table for a geometry. Fills the
// host-side vectors; the caller uploads them.
struct EntropyHostPlan {
    std::vector<Section> sections;
    std::vector<Stripe> stripes;
    std::uint32_t total_items{0};
    std::uint32_t ac_first{0};
    std::vector<std::uint8_t> pre_const;
    std::uint32_t pre_const_bits{0};
    std::vector<std::uint8_t> mid_const;
    std::uint32_t mid_const_bits{0};
    std::vector<std::uint8_t> ac_prefix;
    std::uint32_t ac_prefix_bits{0};
    std::vector<std::uint16_t> order;
};
EntropyHostPlan entropy_plan(int width, int height);

// DcGlobal section bits for the quantiser state.
std::vector<std::uint8_t> dc_global_bits(std::uint32_t global_scale, std::uint32_t quant_dc,
                                         std::uint32_t* nbits);

// Worst-case output size (same bound as the reference's cujpegxl.cc:50-59).
std::size_t worst_case_output(std::uint32_t width, std::uint32_t height);

// Enqueues the whole entropy + assembly stage on `stream`. After completion
// result[0] holds the file size and result[2] a status (0 = ok, 1 = output
// capacity exceeded).
bool entropy_launch(const EntropyDev& e, void* stream);

// Several frames' entropy stages as one launch per pass: each pass runs the
// blocks of every frame, frame f owning blocks begin[phase][f] ..
// begin[phase][f + 1] - 1. The frames live in the launch's parameter block.
constexpr int kEntropyBatchFrames = 64;
enum EntropyPhase : int {
    kPhaseItems = 0,    // item passes: one block per AC stripe, then one per 512 other items
    kPhaseCodes = 1,    // prefix codes: one block per histogram
    kPhaseScan = 2,     // item scan tiles
    kPhaseFrame = 3,    // one block per frame
    kPhaseZero = 4,     // body zeroing
    kPhaseStripes = 5,  // AC stripes whose tokens did not fit the pool
    kEntropyPhases = 6
};
struct EntropyBatch {
    int nframes;
    std::uint32_t begin[kEntropyPhases][kEntropyBatchFrames + 1];
    EntropyDev frames[kEntropyBatchFrames];
};

// Fills b.begin from b.frames[0 .. b.nframes).
void entropy_batch_plan(EntropyBatch& b);

// Enqueues every frame's entropy stage on `stream` (b planned).
bool entropy_batch_launch(const EntropyBatch& b, void* stream);

// The device prefix-code builder on one histogram of `length` (1..256)
// symbols, synchronously on the current device (test hook): depths, codes and
// the header (header_cap >= kDescBytes), its length in bits.
bool prefix_code_test(const std::uint32_t* hist, int length, std::uint8_t* depth, std::uint16_t* bits,
                      std::uint8_t* header, std::size_t header_cap, std::uint32_t* nbits);

}  // namespace jxb
