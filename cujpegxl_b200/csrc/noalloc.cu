// Entropy coding and assembly from device planes without any allocation.
//
// Some callers cannot allocate device memory while they encode: a real-time
// loop where cudaMalloc would synchronise the whole device and stall other
// streams, or an embedder whose device memory is entirely reserved by its own
// pool allocator. For them, cujpegxl_b200_encode_planes_noalloc takes the
// quantised planes and the output buffer from the caller and keeps every
// intermediate (non-zero counts, section table, histograms, prefix codes,
// per-item bit lengths and their scan) in one file-scope __device__ array of
// kScratchBytes. Every GPU that loads the library holds that array until the
// process exits. The call synchronises its stream before it returns.

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <vector>

#include "cujpegxl/cujpegxl.h"
#include "cujpegxl_b200/cujpegxl_b200.h"
#include "entropy.cuh"
#include "jxl_constants.cuh"

namespace jxb {
bool entropy_kernels_init();
bool launch_nz_counts(const std::int16_t* ac, const std::int8_t* acs, int bw, int bh, std::uint8_t* nzn,
                      std::uint16_t* nzc, void* stream);
}  // namespace jxb

namespace {

// Frames up to kMaxPixels (4 megapixels, e.g. 2560x1600 or 2048x2048) fit in
// the scratch array; larger frames are rejected.
constexpr std::size_t kMaxPixels = std::size_t{1} << 22;
constexpr std::size_t kScratchBytes = std::size_t{7} << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mutex;
unsigned char* g_scratch_addr[64] = {};

// Device address of the scratch array on the current device. A host-side
// name of a __device__ array is not a device address, so it is looked up
// once per device with that device current.
unsigned char* scratch_for_current_device() {
    int dev{0};
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_addr[dev] == nullptr) {
        void* p{nullptr};
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return nullptr;
        if (!jxb::entropy_kernels_init()) return nullptr;
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    return g_scratch_addr[dev];
}

struct Carve {
    unsigned char* base;
    std::size_t used{0};
    bool ok{true};
    template <typename T>
    T* take(std::size_t count) {
        const std::size_t at{(used + 255) & ~static_cast<std::size_t>(255)};
        const std::size_t bytes{count * sizeof(T)};
        if (at + bytes > kScratchBytes) {
            ok = false;
            return nullptr;
        }
        used = at + bytes;
        return reinterpret_cast<T*>(base + at);
    }
};

}  // namespace

extern "C" {

// No counterpart in the reference. Entropy coding and assembly of one frame
// from quantised planes already in device memory into a caller-owned device
// buffer, exactly as cujpegxl_b200_encode_planes, with no allocation. See
// include/cujpegxl_b200/cujpegxl_b200.h for the contract.
cujpegxl_status cujpegxl_b200_encode_planes_noalloc(const cujpegxl_b200_device_planes* planes,
                                                    uint32_t width, uint32_t height,
                                                    uint32_t global_scale, uint32_t quant_dc,
                                                    uint8_t* out_device, size_t out_capacity,
                                                    size_t* out_size, uintptr_t stream) {
    if (planes == nullptr || out_device == nullptr || out_size == nullptr || planes->ac == 0 ||
        planes->dc == 0 || planes->acs == 0 || planes->qf == 0 || planes->ytox == 0 || planes->ytob == 0 ||
        (reinterpret_cast<std::uintptr_t>(out_device) & 15u) != 0 || (planes->ac & 15u) != 0 ||
        (planes->dc & 3u) != 0 || (planes->qf & 3u) != 0) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    if (width == 0 || height == 0 || width % 8 != 0 || height % 8 != 0 ||
        ((width / 8 + 31) / 32) * static_cast<std::size_t>((height / 8 + 31) / 32) <= 1) {
        return CUJPEGXL_UNSUPPORTED_RESOLUTION;
    }
    if (static_cast<std::size_t>(width) * height > kMaxPixels) return CUJPEGXL_UNSUPPORTED_RESOLUTION;
    unsigned char* base{scratch_for_current_device()};
    if (base == nullptr) return CUJPEGXL_INTERNAL_ERROR;
    cudaStream_t st{reinterpret_cast<cudaStream_t>(stream)};

    const int W{static_cast<int>(width)};
    const int H{static_cast<int>(height)};
    const int bw{W / 8};
    const int bh{H / 8};
    const std::size_t nb{static_cast<std::size_t>(bw) * bh};
    const jxb::EntropyHostPlan plan{jxb::entropy_plan(W, H)};
    const int ndc{((bw + 255) / 256) * ((bh + 255) / 256)};
    const std::uint32_t tiles{(plan.total_items + jxb::kScanTile - 1) / jxb::kScanTile};
    std::uint32_t dcg_bits{0};
    const std::vector<std::uint8_t> dcg{jxb::dc_global_bits(global_scale, quant_dc, &dcg_bits)};

    Carve c{base};
    jxb::EntropyDev e{};
    e.width = W;
    e.height = H;
    e.bw = bw;
    e.bh = bh;
    e.nblocks = static_cast<int>(nb);
    e.xg = (bw + 31) / 32;
    e.nac = e.xg * ((bh + 31) / 32);
    e.xdg = (bw + 255) / 256;
    e.ndc = ndc;
    e.cmw = (bw + 7) / 8;
    e.nsec = static_cast<int>(plan.sections.size());
    e.total_items = plan.total_items;
    e.ac_first = plan.ac_first;
    e.num_tiles = tiles;
    auto* sections{c.take<jxb::Section>(plan.sections.size())};
    auto* stripes{c.take<jxb::Stripe>(plan.stripes.size())};
    auto* order{c.take<std::uint16_t>(plan.order.size())};
    auto* pre{c.take<std::uint8_t>(plan.pre_const.size())};
    auto* mid{c.take<std::uint8_t>(plan.mid_const.size())};
    auto* acp{c.take<std::uint8_t>(plan.ac_prefix.size())};
    auto* dcgd{c.take<std::uint8_t>(dcg.size())};
    std::uint8_t* nzn{c.take<std::uint8_t>(3 * nb)};
    std::uint16_t* nzc{c.take<std::uint16_t>(3 * nb)};
    e.ac_hist = c.take<std::uint32_t>(32 * 256);
    e.dc_hist = c.take<std::uint32_t>(static_cast<std::size_t>(ndc) * 256);
    e.am_hist = c.take<std::uint32_t>(static_cast<std::size_t>(ndc) * 256);
    e.fb_count = c.take<std::uint32_t>(static_cast<std::size_t>(ndc));
    e.ac_depth = c.take<std::uint8_t>(32 * 256);
    e.ac_bits = c.take<std::uint16_t>(32 * 256);
    e.dc_depth = c.take<std::uint8_t>(static_cast<std::size_t>(ndc) * 256);
    e.dc_bits = c.take<std::uint16_t>(static_cast<std::size_t>(ndc) * 256);
    e.am_depth = c.take<std::uint8_t>(static_cast<std::size_t>(ndc) * 256);
    e.am_bits = c.take<std::uint16_t>(static_cast<std::size_t>(ndc) * 256);
    e.ac_alpha = c.take<std::uint32_t>(32);
    e.desc = c.take<std::uint8_t>(static_cast<std::size_t>(32 + 2 * ndc) * jxb::kDescBytes);
    e.desc_bits = c.take<std::uint32_t>(static_cast<std::size_t>(32 + 2 * ndc));
    e.item_bits = c.take<std::uint32_t>(plan.total_items);
    e.item_pre = c.take<std::uint32_t>(plan.total_items);
    e.tile_sum = c.take<std::uint32_t>(tiles);
    e.tile_off = c.take<unsigned long long>(tiles + 1);
    e.sec_pos = c.take<unsigned long long>(plan.sections.size());
    e.result = c.take<unsigned long long>(4);
    e.tok_count = c.take<std::uint32_t>(1);
    e.stripe_tok = c.take<std::uint32_t>(2 * plan.stripes.size());
    if (!c.ok) return CUJPEGXL_UNSUPPORTED_RESOLUTION;
    // The rest of the array holds AC tokens; stripes that find it full are
    // tokenised again from their coefficients.
    const std::size_t tok_at{(c.used + 255) & ~static_cast<std::size_t>(255)};
    e.tok_capacity = tok_at < kScratchBytes ? static_cast<std::uint32_t>((kScratchBytes - tok_at) / 4) : 0u;
    e.tok_pool = reinterpret_cast<std::uint32_t*>(base + (tok_at < kScratchBytes ? tok_at : 0));

    e.sections = sections;
    e.stripes = stripes;
    e.nstripes = static_cast<int>(plan.stripes.size());
    e.order = order;
    e.pre_const = pre;
    e.pre_const_bits = plan.pre_const_bits;
    e.mid_const = mid;
    e.mid_const_bits = plan.mid_const_bits;
    e.ac_prefix = acp;
    e.ac_prefix_bits = plan.ac_prefix_bits;
    e.dc_global = dcgd;
    e.dc_global_bits = dcg_bits;
    e.ac = reinterpret_cast<const std::int16_t*>(planes->ac);
    e.dc = reinterpret_cast<const std::int32_t*>(planes->dc);
    e.acs = reinterpret_cast<const std::int8_t*>(planes->acs);
    e.qf = reinterpret_cast<const std::int32_t*>(planes->qf);
    e.ytox = reinterpret_cast<const std::int8_t*>(planes->ytox);
    e.ytob = reinterpret_cast<const std::int8_t*>(planes->ytob);
    e.nzn = nzn;
    e.nzc = nzc;
    e.out = out_device;
    e.out_capacity = out_capacity & ~static_cast<std::size_t>(15);

    // The tables change with the geometry and the quantiser, so they are
    // written on every call; everything else is recomputed or cleared by the
    // entropy stage itself.
    const bool uploaded{
        cudaMemcpyAsync(sections, plan.sections.data(), plan.sections.size() * sizeof(jxb::Section),
                        cudaMemcpyHostToDevice, st) == cudaSuccess &&
        cudaMemcpyAsync(stripes, plan.stripes.data(), plan.stripes.size() * sizeof(jxb::Stripe),
                        cudaMemcpyHostToDevice, st) == cudaSuccess &&
        cudaMemcpyAsync(order, plan.order.data(), plan.order.size() * 2, cudaMemcpyHostToDevice, st) == cudaSuccess &&
        cudaMemcpyAsync(pre, plan.pre_const.data(), plan.pre_const.size(), cudaMemcpyHostToDevice, st) == cudaSuccess &&
        cudaMemcpyAsync(mid, plan.mid_const.data(), plan.mid_const.size(), cudaMemcpyHostToDevice, st) == cudaSuccess &&
        cudaMemcpyAsync(acp, plan.ac_prefix.data(), plan.ac_prefix.size(), cudaMemcpyHostToDevice, st) == cudaSuccess &&
        cudaMemcpyAsync(dcgd, dcg.data(), dcg.size(), cudaMemcpyHostToDevice, st) == cudaSuccess};
    if (!uploaded || !jxb::launch_nz_counts(e.ac, e.acs, bw, bh, nzn, nzc, st) || !jxb::entropy_launch(e, st)) {
        return CUJPEGXL_INTERNAL_ERROR;
    }
    unsigned long long result[4]{};
    if (cudaMemcpyAsync(result, e.result, sizeof(result), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        return CUJPEGXL_INTERNAL_ERROR;
    }
    if (result[2] == 1) {
        *out_size = static_cast<std::size_t>(result[0]);
        return CUJPEGXL_BUFFER_TOO_SMALL;
    }
    if (result[2] != 0) return CUJPEGXL_INTERNAL_ERROR;
    *out_size = static_cast<std::size_t>(result[0]);
    return CUJPEGXL_OK;
}

}  // extern "C"
