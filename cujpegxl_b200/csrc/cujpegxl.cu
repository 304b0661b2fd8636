// The C ABI of libcujpegxl.so.1: the reference's nine entry points
// (include/cujpegxl/cujpegxl.h:66-82 in m-pilia/cujpegxl, implemented there in
// src/cujpegxl.cc) plus the additional entry points of
// include/cujpegxl_b200/cujpegxl_b200.h, over a per-encoder CUDA stream and
// device arena allocated once per geometry.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "cujpegxl/cujpegxl.h"
#include "cujpegxl_b200/cujpegxl_b200.h"
#include "encoder_internal.h"
#include "acsnet.cuh"
#include "entropy.cuh"
#include "frontend.cuh"
#include "jxl_constants.cuh"

namespace jxb {
bool entropy_kernels_init();
}

struct cujpegxl_encoder {
    cujpegxl_config config{};
    int device{0};
    cudaStream_t stream{nullptr};
    void* arena{nullptr};
    std::uint32_t geo_w{0};
    std::uint32_t geo_h{0};
    float geo_distance{-1.0f};
    bool debug{false};
    jxb::FrontendOutputs fo{};
    jxb::EntropyDev ed{};
    jxb::FrontendScalars fs{};
    std::uint32_t global_scale{0};
    std::uint32_t quant_dc{0};
    std::uint8_t* dc_global_dev{nullptr};
    float* dbg_xyb{nullptr};
    float* dbg_sharp{nullptr};
    std::uint16_t* dbg_coeff{nullptr};
    float* dbg_cost{nullptr};
    std::uint8_t* nv12_dev{nullptr};
    std::uint8_t* nv12_pinned{nullptr};
    unsigned long long* result_pinned{nullptr};
    std::size_t arena_bytes{0};
    bool pending{false};
    // Learned decisions: the attached network (not owned), its margin and
    // flags, and the per-frame decision buffers in the arena.
    const cujpegxl_b200_acsnet* net{nullptr};
    float net_margin{0.2f};
    std::uint32_t net_flags{0};
    std::int8_t* net_class{nullptr};
    std::uint32_t* tile_order{nullptr};  // [64x64 tiles + 2], written by the inference kernel
    std::int16_t* net_qf{nullptr};
    bool allow_single{false};  // created with CUJPEGXL_B200_ENCODER_SINGLE_GROUP
};

namespace {

struct DeviceTables {
    bool ready{false};
    jxb::FrontendTables ft{};
};

std::mutex g_mutex;
DeviceTables g_tables[64];

// Encoder resources (device arenas, pinned host buffers, streams) go through
// these wrappers: they count what is live, and a test hook can make the n-th
// acquisition fail as a real out-of-memory would, to exercise the error paths
// of create and configure (cujpegxl_b200_debug_fail_allocation).
std::atomic<std::uint32_t> g_fail_countdown{0};
std::atomic<std::uint64_t> g_live{0};

bool injected_failure() {
    std::uint32_t n{g_fail_countdown.load()};
    while (n != 0) {
        if (g_fail_countdown.compare_exchange_weak(n, n - 1)) return n == 1;
    }
    return false;
}

bool acquire_device(void** p, std::size_t bytes) {
    if (injected_failure() || cudaMalloc(p, bytes) != cudaSuccess) {
        *p = nullptr;
        return false;
    }
    ++g_live;
    return true;
}

bool acquire_pinned(void** p, std::size_t bytes) {
    if (injected_failure() || cudaHostAlloc(p, bytes, cudaHostAllocDefault) != cudaSuccess) {
        *p = nullptr;
        return false;
    }
    ++g_live;
    return true;
}

bool acquire_stream(cudaStream_t* s) {
    if (injected_failure() || cudaStreamCreateWithFlags(s, cudaStreamNonBlocking) != cudaSuccess) {
        *s = nullptr;
        return false;
    }
    ++g_live;
    return true;
}

void release_device(void* p) {
    if (p != nullptr && cudaFree(p) == cudaSuccess) --g_live;
}

void release_pinned(void* p) {
    if (p != nullptr && cudaFreeHost(p) == cudaSuccess) --g_live;
}

void release_stream(cudaStream_t s) {
    if (s != nullptr && cudaStreamDestroy(s) == cudaSuccess) --g_live;
}

// Restores the caller's current device on scope exit.
class DeviceScope {
public:
    explicit DeviceScope(int device) {
        ok_ = cudaGetDevice(&prev_) == cudaSuccess && cudaSetDevice(device) == cudaSuccess;
    }
    ~DeviceScope() { cudaSetDevice(prev_); }
    bool ok() const { return ok_; }

private:
    int prev_{0};
    bool ok_{false};
};

bool device_tables(int device, jxb::FrontendTables* out) {
    if (device < 0 || device >= 64) return false;
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceTables& t{g_tables[device]};
    if (!t.ready) {
        if (!jxb::frontend_tables_init(&t.ft) || !jxb::entropy_kernels_init() || !jxb::acsnet_kernels_init()) {
            return false;
        }
        t.ready = true;
    }
    *out = t.ft;
    return true;
}

bool device_exists(std::int32_t ordinal, int* major, int* minor) {
    int count{0};
    if (cudaGetDeviceCount(&count) != cudaSuccess || ordinal < 0 || ordinal >= count) return false;
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, ordinal) != cudaSuccess) return false;
    *major = prop.major;
    *minor = prop.minor;
    return true;
}

// src/cujpegxl.cc:36-48: distance must be positive and finite; width and
// height positive multiples of 8 spanning more than one 256x256 AC group.
// allow_single: frames of one AC group (at most 256x256), which the reference
// rejects, are accepted and written with the combined-section layout.
cujpegxl_status validate_config(const cujpegxl_config& c, bool allow_single = false) {
    if (!(c.distance > 0.0f) || !std::isfinite(c.distance)) return CUJPEGXL_INVALID_ARGUMENT;
    if (c.width == 0 || c.height == 0 || c.width % 8 != 0 || c.height % 8 != 0) {
        return CUJPEGXL_UNSUPPORTED_RESOLUTION;
    }
    const std::size_t nac{((c.width / 8 + 31) / 32) * static_cast<std::size_t>((c.height / 8 + 31) / 32)};
    if (nac <= 1 && !allow_single) return CUJPEGXL_UNSUPPORTED_RESOLUTION;
    // The TOC is written in one CTA's shared memory: about 25,000 sections
    // (1.6 gigapixels) at most.
    const std::size_t ndc{((c.width / 8 + 255) / 256) * static_cast<std::size_t>((c.height / 8 + 255) / 256)};
    if (2 + ndc + nac > static_cast<std::size_t>(jxb::kMaxSections)) return CUJPEGXL_UNSUPPORTED_RESOLUTION;
    return CUJPEGXL_OK;
}

std::size_t align256(std::size_t v) { return (v + 255) & ~static_cast<std::size_t>(255); }

// Sub-allocates the encoder's device buffers from one arena.
struct ArenaPlan {
    std::size_t total{0};
    std::size_t take(std::size_t bytes) {
        const std::size_t at{total};
        total += align256(bytes);
        return at;
    }
};

void release(cujpegxl_encoder* e) {
    release_device(e->arena);
    release_pinned(e->nv12_pinned);
    e->arena = nullptr;
    e->nv12_pinned = nullptr;
    e->geo_w = e->geo_h = 0;
}

// Allocates every per-geometry buffer (nothing is allocated per frame).
bool allocate(cujpegxl_encoder* e) {
    release(e);
    const std::uint32_t W{e->config.width};
    const std::uint32_t H{e->config.height};
    const std::size_t bw{W / 8};
    const std::size_t bh{H / 8};
    const std::size_t nb{bw * bh};
    const std::size_t nt{((bw + 7) / 8) * ((bh + 7) / 8)};
    const jxb::EntropyHostPlan plan{jxb::entropy_plan(static_cast<int>(W), static_cast<int>(H))};
    const int ndc{static_cast<int>(((bw + 255) / 256) * ((bh + 255) / 256))};
    const int nac{static_cast<int>(((bw + 31) / 32) * ((bh + 31) / 32))};
    const std::uint32_t tiles{(plan.total_items + jxb::kScanTile - 1) / jxb::kScanTile};
    const std::size_t out_cap{(jxb::worst_case_output(W, H) + 15) & ~static_cast<std::size_t>(15)};

    ArenaPlan a;
    const std::size_t o_ac{a.take(3 * nb * 64 * 2)};
    const std::size_t o_dc{a.take(3 * nb * 4)};
    const std::size_t o_acs{a.take(nb)};
    const std::size_t o_qf{a.take(nb * 4)};
    const std::size_t o_tx{a.take(nt)};
    const std::size_t o_tb{a.take(nt)};
    const std::size_t o_nzn{a.take(3 * nb)};
    const std::size_t o_nzc{a.take(3 * nb * 2)};
    const std::size_t o_sec{a.take(plan.sections.size() * sizeof(jxb::Section))};
    const std::size_t o_str{a.take(plan.stripes.size() * sizeof(jxb::Stripe))};
    const std::size_t o_ord{a.take(plan.order.size() * 2)};
    const std::size_t o_pre{a.take(plan.pre_const.size())};
    const std::size_t o_mid{a.take(plan.mid_const.size())};
    const std::size_t o_acp{a.take(plan.ac_prefix.size())};
    const std::size_t o_dcg{a.take(64)};
    const std::size_t o_ach{a.take(32 * 256 * 4)};
    const std::size_t o_dch{a.take(static_cast<std::size_t>(ndc) * 256 * 4)};
    const std::size_t o_amh{a.take(static_cast<std::size_t>(ndc) * 256 * 4)};
    const std::size_t o_fb{a.take(static_cast<std::size_t>(ndc) * 4)};
    const std::size_t o_acd{a.take(32 * 256)};
    const std::size_t o_acb{a.take(32 * 256 * 2)};
    const std::size_t o_dcd{a.take(static_cast<std::size_t>(ndc) * 256)};
    const std::size_t o_dcb{a.take(static_cast<std::size_t>(ndc) * 256 * 2)};
    const std::size_t o_amd{a.take(static_cast<std::size_t>(ndc) * 256)};
    const std::size_t o_amb{a.take(static_cast<std::size_t>(ndc) * 256 * 2)};
    const std::size_t o_alpha{a.take(32 * 4)};
    const std::size_t o_desc{a.take(static_cast<std::size_t>(32 + 2 * ndc) * jxb::kDescBytes)};
    const std::size_t o_descb{a.take(static_cast<std::size_t>(32 + 2 * ndc) * 4)};
    const std::size_t o_ib{a.take(static_cast<std::size_t>(plan.total_items) * 4)};
    const std::size_t o_ip{a.take(static_cast<std::size_t>(plan.total_items) * 4)};
    const std::size_t o_ts{a.take(static_cast<std::size_t>(tiles) * 4)};
    const std::size_t o_to{a.take(static_cast<std::size_t>(tiles + 1) * 8)};
    const std::size_t o_sp{a.take(plan.sections.size() * 8)};
    const std::size_t o_res{a.take(4 * 8)};
    const std::uint32_t tok_cap{static_cast<std::uint32_t>(std::min<std::size_t>(nb * jxb::kTokensPerBlock, 0xfffffff0u))};
    const std::size_t o_tok{a.take(static_cast<std::size_t>(tok_cap) * 4)};
    const std::size_t o_tokn{a.take(4)};
    const std::size_t o_stok{a.take(plan.stripes.size() * 8)};
    const std::size_t o_out{a.take(out_cap)};
    const std::size_t o_nv12{a.take(static_cast<std::size_t>(W) * H * 3 / 2)};
    const std::size_t o_ncls{a.take(((bw + 3) / 4) * ((bh + 3) / 4))};
    const std::size_t o_nqf{a.take(nb * 2)};
    const std::size_t o_tord{a.take((nt + 2) * 4)};
    std::size_t o_dbg{0};
    if (e->debug) {
        o_dbg = a.take(2 * 3 * static_cast<std::size_t>(W) * H * 4 + 3 * nb * 64 * 2 + 3 * nb * 4);
    }
    void* base{nullptr};
    if (!acquire_device(&base, a.total)) return false;
    e->arena = base;
    e->arena_bytes = a.total;
    auto* b{static_cast<std::uint8_t*>(base)};

    jxb::FrontendOutputs& fo{e->fo};
    fo.ac = reinterpret_cast<std::int16_t*>(b + o_ac);
    fo.dc = reinterpret_cast<std::int32_t*>(b + o_dc);
    fo.acs = reinterpret_cast<std::int8_t*>(b + o_acs);
    fo.qf = reinterpret_cast<std::int32_t*>(b + o_qf);
    fo.ytox = reinterpret_cast<std::int8_t*>(b + o_tx);
    fo.ytob = reinterpret_cast<std::int8_t*>(b + o_tb);
    fo.nzn = b + o_nzn;
    fo.nzc = reinterpret_cast<std::uint16_t*>(b + o_nzc);
    e->dbg_xyb = e->debug ? reinterpret_cast<float*>(b + o_dbg) : nullptr;
    e->dbg_sharp = e->debug ? e->dbg_xyb + 3 * static_cast<std::size_t>(W) * H : nullptr;
    e->dbg_coeff = e->debug ? reinterpret_cast<std::uint16_t*>(e->dbg_sharp + 3 * static_cast<std::size_t>(W) * H)
                            : nullptr;
    fo.dbg_xyb = e->dbg_xyb;
    fo.dbg_sharp = e->dbg_sharp;
    fo.dbg_coeff = e->dbg_coeff;
    e->dbg_cost = e->debug ? reinterpret_cast<float*>(e->dbg_coeff + 3 * nb * 64) : nullptr;
    fo.dbg_cost = e->dbg_cost;

    jxb::EntropyDev& ed{e->ed};
    ed = jxb::EntropyDev{};
    ed.width = static_cast<int>(W);
    ed.height = static_cast<int>(H);
    ed.bw = static_cast<int>(bw);
    ed.bh = static_cast<int>(bh);
    ed.nblocks = static_cast<int>(nb);
    ed.xg = static_cast<int>((bw + 31) / 32);
    ed.nac = nac;
    ed.xdg = static_cast<int>((bw + 255) / 256);
    ed.ndc = ndc;
    ed.cmw = static_cast<int>((bw + 7) / 8);
    ed.nsec = static_cast<int>(plan.sections.size());
    ed.total_items = plan.total_items;
    ed.ac_first = plan.ac_first;
    ed.num_tiles = tiles;
    ed.sections = reinterpret_cast<const jxb::Section*>(b + o_sec);
    ed.stripes = reinterpret_cast<const jxb::Stripe*>(b + o_str);
    ed.nstripes = static_cast<int>(plan.stripes.size());
    ed.ac = fo.ac;
    ed.dc = fo.dc;
    ed.acs = fo.acs;
    ed.qf = fo.qf;
    ed.ytox = fo.ytox;
    ed.ytob = fo.ytob;
    ed.nzn = fo.nzn;
    ed.nzc = fo.nzc;
    ed.order = reinterpret_cast<const std::uint16_t*>(b + o_ord);
    ed.pre_const = b + o_pre;
    ed.pre_const_bits = plan.pre_const_bits;
    ed.mid_const = b + o_mid;
    ed.mid_const_bits = plan.mid_const_bits;
    ed.ac_prefix = b + o_acp;
    ed.ac_prefix_bits = plan.ac_prefix_bits;
    e->dc_global_dev = b + o_dcg;
    ed.dc_global = e->dc_global_dev;
    ed.ac_hist = reinterpret_cast<std::uint32_t*>(b + o_ach);
    ed.dc_hist = reinterpret_cast<std::uint32_t*>(b + o_dch);
    ed.am_hist = reinterpret_cast<std::uint32_t*>(b + o_amh);
    ed.fb_count = reinterpret_cast<std::uint32_t*>(b + o_fb);
    ed.ac_depth = b + o_acd;
    ed.ac_bits = reinterpret_cast<std::uint16_t*>(b + o_acb);
    ed.dc_depth = b + o_dcd;
    ed.dc_bits = reinterpret_cast<std::uint16_t*>(b + o_dcb);
    ed.am_depth = b + o_amd;
    ed.am_bits = reinterpret_cast<std::uint16_t*>(b + o_amb);
    ed.ac_alpha = reinterpret_cast<std::uint32_t*>(b + o_alpha);
    ed.desc = b + o_desc;
    ed.desc_bits = reinterpret_cast<std::uint32_t*>(b + o_descb);
    ed.item_bits = reinterpret_cast<std::uint32_t*>(b + o_ib);
    ed.item_pre = reinterpret_cast<std::uint32_t*>(b + o_ip);
    ed.tile_sum = reinterpret_cast<std::uint32_t*>(b + o_ts);
    ed.tile_off = reinterpret_cast<unsigned long long*>(b + o_to);
    ed.sec_pos = reinterpret_cast<unsigned long long*>(b + o_sp);
    ed.result = reinterpret_cast<unsigned long long*>(b + o_res);
    ed.tok_pool = reinterpret_cast<std::uint32_t*>(b + o_tok);
    ed.tok_capacity = tok_cap;
    ed.tok_count = reinterpret_cast<std::uint32_t*>(b + o_tokn);
    ed.stripe_tok = reinterpret_cast<std::uint32_t*>(b + o_stok);
    ed.out = b + o_out;
    ed.out_capacity = out_cap;
    e->nv12_dev = b + o_nv12;
    e->net_class = reinterpret_cast<std::int8_t*>(b + o_ncls);
    e->net_qf = reinterpret_cast<std::int16_t*>(b + o_nqf);
    e->tile_order = reinterpret_cast<std::uint32_t*>(b + o_tord);

    bool ok{cudaMemcpy(b + o_sec, plan.sections.data(), plan.sections.size() * sizeof(jxb::Section),
                       cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(b + o_str, plan.stripes.data(), plan.stripes.size() * sizeof(jxb::Stripe),
                       cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(b + o_ord, plan.order.data(), plan.order.size() * 2, cudaMemcpyHostToDevice) ==
                cudaSuccess &&
            cudaMemcpy(b + o_pre, plan.pre_const.data(), plan.pre_const.size(), cudaMemcpyHostToDevice) ==
                cudaSuccess &&
            cudaMemcpy(b + o_mid, plan.mid_const.data(), plan.mid_const.size(), cudaMemcpyHostToDevice) ==
                cudaSuccess &&
            cudaMemcpy(b + o_acp, plan.ac_prefix.data(), plan.ac_prefix.size(), cudaMemcpyHostToDevice) ==
                cudaSuccess};
    ok = ok && acquire_pinned(reinterpret_cast<void**>(&e->nv12_pinned), static_cast<std::size_t>(W) * H * 3 / 2 + 64);
    if (!ok) {
        release(e);
        return false;
    }
    e->result_pinned = reinterpret_cast<unsigned long long*>(e->nv12_pinned + static_cast<std::size_t>(W) * H * 3 / 2);
    e->geo_w = W;
    e->geo_h = H;
    e->geo_distance = -1.0f;
    return true;
}

// Per-distance state: quantiser scalars and the DcGlobal section.
bool set_distance(cujpegxl_encoder* e) {
    if (e->geo_distance == e->config.distance) return true;
    e->fs = jxb::frontend_scalars(e->config.distance, &e->global_scale, &e->quant_dc);
    std::uint32_t nbits{0};
    const std::vector<std::uint8_t> dcg{jxb::dc_global_bits(e->global_scale, e->quant_dc, &nbits)};
    if (dcg.size() > 64 || cudaMemcpy(e->dc_global_dev, dcg.data(), dcg.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        return false;
    }
    e->ed.dc_global_bits = nbits;
    e->geo_distance = e->config.distance;
    return true;
}

bool prepare(cujpegxl_encoder* e) {
    if (e->geo_w != e->config.width || e->geo_h != e->config.height || e->arena == nullptr) {
        if (!allocate(e)) return false;
    }
    return set_distance(e);
}

bool enqueue_frame(cujpegxl_encoder* e, const std::uint8_t* luma, std::size_t lp, const std::uint8_t* chroma,
                   std::size_t cp, std::uint32_t stages = 3u, cudaStream_t stream = nullptr) {
    jxb::FrontendTables ft{};
    if (!device_tables(e->device, &ft)) return false;
    jxb::FrontendInputs in{luma, chroma, lp, cp, static_cast<int>(e->config.width),
                           static_cast<int>(e->config.height), nullptr, nullptr, nullptr};
    cudaStream_t st{stream != nullptr ? stream : e->stream};
    if ((stages & 1u) && e->net != nullptr) {
        const jxb::NetDecisionsDev dec{e->net_class, (e->net_flags & CUJPEGXL_B200_ACSNET_QF) ? e->net_qf : nullptr,
                                       e->tile_order};
        if (!jxb::acsnet_infer_launch(in, *jxb::acsnet_params(e->net), std::log2(e->config.distance),
                                      e->net_margin, dec, st)) {
            return false;
        }
        in.net_class = dec.cls;
        in.net_qf = dec.qf;
        in.tile_order = dec.tile_order;
    }
    if ((stages & 1u) && !jxb::frontend_launch(in, e->fs, ft, e->fo, st)) return false;
    return (stages & 2u) == 0 || jxb::entropy_launch(e->ed, st);
}

cujpegxl_status finish(cujpegxl_encoder* e, cujpegxl_output* output);

// Waits for the encode and copies the file into `output`.
// Non-zero counts of uploaded planes (the frontend computes these itself):
// per first-block and channel the count over its non-LLF coefficients, and
// its normalised value at every covered position (src/entropy.cu:686-721).
__global__ void nz_kernel(const std::int16_t* ac, const std::int8_t* acs, int bw, int bh,
                          std::uint8_t* nzn, std::uint16_t* nzc) {
    const int blk{static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x)};
    const int nb{bw * bh};
    if (blk >= nb) return;
    const int n{acs[blk]};
    for (int c{0}; c < 3; ++c) nzc[c * nb + blk] = 0;
    if (n == 0) return;
    const int bx{blk % bw};
    const int by{blk / bw};
    const int side{n / 8};
    const int l2{n == 16 ? 2 : (n == 32 ? 4 : 0)};
    for (int c{0}; c < 3; ++c) {
        const std::int16_t* p{ac + static_cast<std::size_t>(c) * nb * 64};
        int cnt{0};
        for (int raw{0}; raw < n * n; ++raw) {
            if ((raw / n) < side && (raw % n) < side) continue;
            if (p[jxb::covered_slot(n, bx, by, bw, raw)] != 0) ++cnt;
        }
        const int norm{(cnt + side * side - 1) >> l2};
        for (int dy{0}; dy < side; ++dy) {
            for (int dx{0}; dx < side; ++dx) {
                nzn[c * nb + (by + dy) * bw + bx + dx] = static_cast<std::uint8_t>(norm);
            }
        }
        nzc[c * nb + blk] = static_cast<std::uint16_t>(cnt);
    }
}

// Copies a finished file from device memory into pinned host memory that the
// device reaches through unified addressing, with the file's size taken from
// the result words on the device, so that no host round trip sits between the
// encode and the copy. words_out receives {file bytes, status}: status 0 =
// copied, 1 = the file exceeds `capacity` (nothing copied), 2 = the encode
// failed.
__global__ void __launch_bounds__(256) readback_kernel(const unsigned long long* result, const std::uint8_t* src,
                                                       std::uint8_t* dst, unsigned long long capacity,
                                                       unsigned long long* words_out) {
    const unsigned long long total{result[0]};
    const unsigned long long status{result[2] != 0 ? 2ull : (total > capacity ? 1ull : 0ull)};
    const unsigned long long tid{static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x};
    const unsigned long long stride{static_cast<unsigned long long>(gridDim.x) * blockDim.x};
    if (status == 0) {
        if ((reinterpret_cast<std::uintptr_t>(dst) & 15u) == 0) {
            const unsigned long long nvec{total / 16};
            const uint4* s4{reinterpret_cast<const uint4*>(src)};
            uint4* d4{reinterpret_cast<uint4*>(dst)};
            for (unsigned long long i{tid}; i < nvec; i += stride) d4[i] = s4[i];
            for (unsigned long long i{nvec * 16 + tid}; i < total; i += stride) dst[i] = src[i];
        } else {
            for (unsigned long long i{tid}; i < total; i += stride) dst[i] = src[i];
        }
    }
    if (tid == 0) {
        words_out[0] = total;
        words_out[1] = status;
    }
}

constexpr unsigned kReadbackBlocks = 64;

// True when [p, p + bytes) starts in page-locked host memory that the current
// device can address (cudaHostAlloc / cudaHostRegister / torch pin_memory).
bool device_reachable_host(const void* p) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (attr.type != cudaMemoryTypeHost) return false;
    void* dp{nullptr};
    if (cudaHostGetDevicePointer(&dp, const_cast<void*>(p), 0) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return dp == p;
}

bool enqueue_readback(cujpegxl_encoder* e, std::uint8_t* dst, std::size_t capacity, unsigned long long* words,
                      cudaStream_t st) {
    readback_kernel<<<kReadbackBlocks, 256, 0, st>>>(e->ed.result, e->ed.out, dst, capacity, words);
    return cudaGetLastError() == cudaSuccess;
}

// A pageable output buffer: the file is copied on the device side into the
// encoder's page-locked NV12 staging buffer (free again once the encode has
// read its input) behind the encode, so the call waits once, and then to the
// caller's memory by a host copy; a pageable device-to-host copy would go
// through the driver's own staging after a second wait. A file larger than
// the staging buffer is copied from device memory instead.
cujpegxl_status finish_pageable(cujpegxl_encoder* e, cujpegxl_output* output) {
    const std::size_t staging{static_cast<std::size_t>(e->config.width) * e->config.height * 3 / 2};
    if (!enqueue_readback(e, e->nv12_pinned, staging, e->result_pinned, e->stream) ||
        cudaStreamSynchronize(e->stream) != cudaSuccess) {
        return CUJPEGXL_INTERNAL_ERROR;
    }
    if (e->result_pinned[1] == 2) return CUJPEGXL_INTERNAL_ERROR;
    const std::size_t total{static_cast<std::size_t>(e->result_pinned[0])};
    if (total > output->capacity) {
        output->size = total;
        return CUJPEGXL_BUFFER_TOO_SMALL;
    }
    if (e->result_pinned[1] == 0) {
        std::memcpy(output->data, e->nv12_pinned, total);
    } else if (cudaMemcpyAsync(output->data, e->ed.out, total, cudaMemcpyDeviceToHost, e->stream) != cudaSuccess ||
               cudaStreamSynchronize(e->stream) != cudaSuccess) {
        return CUJPEGXL_INTERNAL_ERROR;
    }
    output->size = total;
    return CUJPEGXL_OK;
}

// Waits for the encode and copies the file into `output`. A page-locked
// output buffer is written by readback_kernel right behind the encode, so the
// call waits once; other buffers are reached through the encoder's
// page-locked staging buffer (finish_pageable), also after one wait.
cujpegxl_status finish(cujpegxl_encoder* e, cujpegxl_output* output) {
    if (!device_reachable_host(output->data)) return finish_pageable(e, output);
    if (!enqueue_readback(e, output->data, output->capacity, e->result_pinned, e->stream) ||
        cudaStreamSynchronize(e->stream) != cudaSuccess) {
        return CUJPEGXL_INTERNAL_ERROR;
    }
    if (e->result_pinned[1] == 2) return CUJPEGXL_INTERNAL_ERROR;
    output->size = static_cast<std::size_t>(e->result_pinned[0]);
    return e->result_pinned[1] == 1 ? CUJPEGXL_BUFFER_TOO_SMALL : CUJPEGXL_OK;
}

}  // namespace

namespace jxb {

bool encoder_prepare(cujpegxl_encoder* e) {
    DeviceScope scope{e->device};
    return scope.ok() && prepare(e);
}

bool encoder_launch(cujpegxl_encoder* e, const cujpegxl_nv12_input& input, cudaStream_t stream) {
    if (input.luma == 0 || input.chroma == 0 || input.luma_pitch < e->config.width ||
        input.chroma_pitch < e->config.width) {
        return false;
    }
    return enqueue_frame(e, reinterpret_cast<const std::uint8_t*>(input.luma), input.luma_pitch,
                         reinterpret_cast<const std::uint8_t*>(input.chroma), input.chroma_pitch, 3u, stream);
}

bool encoder_frontend_job(cujpegxl_encoder* e, const cujpegxl_nv12_input& input, cudaStream_t stream,
                          FrontendJob* job, FrontendTables* tables) {
    if (!device_tables(e->device, tables)) return false;
    FrontendInputs in{reinterpret_cast<const std::uint8_t*>(input.luma), reinterpret_cast<const std::uint8_t*>(input.chroma),
                      input.luma_pitch, input.chroma_pitch, static_cast<int>(e->config.width),
                      static_cast<int>(e->config.height), nullptr, nullptr, nullptr};
    if (e->net != nullptr) {
        // The batched frontend takes tiles from its own work list.
        const NetDecisionsDev dec{e->net_class, (e->net_flags & CUJPEGXL_B200_ACSNET_QF) ? e->net_qf : nullptr,
                                  nullptr};
        if (!acsnet_infer_launch(in, *acsnet_params(e->net), std::log2(e->config.distance), e->net_margin, dec,
                                 stream)) {
            return false;
        }
        in.net_class = dec.cls;
        in.net_qf = dec.qf;
    }
    job->in = in;
    job->sc = e->fs;
    job->out = e->fo;
    job->tiles_x = static_cast<int>((e->config.width + 63) / 64);
    job->tile_begin = 0;
    return true;
}

const EntropyDev& encoder_entropy(const cujpegxl_encoder* e) { return e->ed; }

bool encoder_has_network(const cujpegxl_encoder* e) { return e->net != nullptr; }

const unsigned long long* encoder_result_words(const cujpegxl_encoder* e) { return e->ed.result; }

const std::uint8_t* encoder_output(const cujpegxl_encoder* e) { return e->ed.out; }

}  // namespace jxb

namespace jxb {
// Launches the non-zero-count kernel above on `stream` (used by entry points
// that take quantised planes from the caller).
bool launch_nz_counts(const std::int16_t* ac, const std::int8_t* acs, int bw, int bh, std::uint8_t* nzn,
                      std::uint16_t* nzc, void* stream) {
    const int nb{bw * bh};
    nz_kernel<<<static_cast<unsigned>((nb + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        ac, acs, bw, bh, nzn, nzc);
    return cudaGetLastError() == cudaSuccess;
}
}  // namespace jxb

extern "C" {

uint32_t cujpegxl_api_version(void) { return CUJPEGXL_API_VERSION; }

const char* cujpegxl_status_string(cujpegxl_status status) {
    switch (status) {
        case CUJPEGXL_OK: return "ok";
        case CUJPEGXL_NOT_IMPLEMENTED: return "not-implemented";
        case CUJPEGXL_INVALID_ARGUMENT: return "invalid-argument";
        case CUJPEGXL_UNSUPPORTED_RESOLUTION: return "unsupported-resolution";
        case CUJPEGXL_NO_DEVICE: return "no-device";
        case CUJPEGXL_INTERNAL_ERROR: return "internal-error";
        case CUJPEGXL_BUFFER_TOO_SMALL: return "buffer-too-small";
    }
    return "internal-error";
}

const char* cujpegxl_backend_string(cujpegxl_backend backend) {
    switch (backend) {
        case CUJPEGXL_BACKEND_FP32_SIMT: return "fp32-simt";
        case CUJPEGXL_BACKEND_FP16_TENSOR: return "fp16-tensor";
        case CUJPEGXL_BACKEND_UNKNOWN: return "unknown";
    }
    return "unknown";
}

// Same label rule as the reference (src/capability.h:25-34): compute
// capability >= 8.0 -> FP16_TENSOR, >= 6.0 -> FP32_SIMT.
cujpegxl_status cujpegxl_query_backend(int32_t device_ordinal, cujpegxl_backend* out_backend) {
    if (out_backend == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    int major{0};
    int minor{0};
    if (!device_exists(device_ordinal, &major, &minor)) return CUJPEGXL_NO_DEVICE;
    const int cc{major * 10 + minor};
    *out_backend = cc >= 80 ? CUJPEGXL_BACKEND_FP16_TENSOR
                            : (cc >= 60 ? CUJPEGXL_BACKEND_FP32_SIMT : CUJPEGXL_BACKEND_UNKNOWN);
    return CUJPEGXL_OK;
}

cujpegxl_status cujpegxl_max_output_size(const cujpegxl_config* config, size_t* out_bytes) {
    return cujpegxl_b200_max_output_size_ex(config, 0u, out_bytes);
}

cujpegxl_status cujpegxl_b200_max_output_size_ex(const cujpegxl_config* config, uint32_t flags, size_t* out_bytes) {
    if (config == nullptr || out_bytes == nullptr || (flags & ~CUJPEGXL_B200_ENCODER_SINGLE_GROUP) != 0) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    const cujpegxl_status st{validate_config(*config, (flags & CUJPEGXL_B200_ENCODER_SINGLE_GROUP) != 0)};
    if (st != CUJPEGXL_OK) return st;
    *out_bytes = jxb::worst_case_output(config->width, config->height);
    return CUJPEGXL_OK;
}

cujpegxl_status cujpegxl_encoder_create(const cujpegxl_config* config, cujpegxl_encoder** out_encoder) {
    return cujpegxl_b200_encoder_create_ex(config, 0u, out_encoder);
}

cujpegxl_status cujpegxl_b200_encoder_create_ex(const cujpegxl_config* config, uint32_t flags,
                                                cujpegxl_encoder** out_encoder) {
    if (config == nullptr || out_encoder == nullptr || (flags & ~CUJPEGXL_B200_ENCODER_SINGLE_GROUP) != 0) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    *out_encoder = nullptr;
    const bool allow_single{(flags & CUJPEGXL_B200_ENCODER_SINGLE_GROUP) != 0};
    const cujpegxl_status st{validate_config(*config, allow_single)};
    if (st != CUJPEGXL_OK) return st;
    int major{0};
    int minor{0};
    if (!device_exists(config->device_ordinal, &major, &minor)) return CUJPEGXL_NO_DEVICE;
    auto* e{new (std::nothrow) cujpegxl_encoder{}};
    if (e == nullptr) return CUJPEGXL_INTERNAL_ERROR;
    e->config = *config;
    e->device = config->device_ordinal;
    e->allow_single = allow_single;
    DeviceScope scope{e->device};
    jxb::FrontendTables ft{};
    if (!scope.ok() || !device_tables(e->device, &ft) ||
        !acquire_stream(&e->stream) || !prepare(e)) {
        release_stream(e->stream);
        release(e);
        delete e;
        return CUJPEGXL_INTERNAL_ERROR;
    }
    *out_encoder = e;
    return CUJPEGXL_OK;
}

cujpegxl_status cujpegxl_encoder_configure(cujpegxl_encoder* encoder, const cujpegxl_config* config) {
    if (encoder == nullptr || config == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    const cujpegxl_status st{validate_config(*config, encoder->allow_single)};
    if (st != CUJPEGXL_OK) return st;
    if (config->device_ordinal != encoder->config.device_ordinal) {
        int major{0};
        int minor{0};
        if (!device_exists(config->device_ordinal, &major, &minor)) return CUJPEGXL_NO_DEVICE;
        DeviceScope old{encoder->device};
        cudaStreamSynchronize(encoder->stream);
        release_stream(encoder->stream);
        encoder->stream = nullptr;
        release(encoder);
        encoder->device = config->device_ordinal;
        encoder->net = nullptr;  // a network lives on one device
        DeviceScope scope{encoder->device};
        if (!acquire_stream(&encoder->stream)) return CUJPEGXL_INTERNAL_ERROR;
    }
    encoder->config = *config;
    DeviceScope scope{encoder->device};
    cudaStreamSynchronize(encoder->stream);
    return prepare(encoder) ? CUJPEGXL_OK : CUJPEGXL_INTERNAL_ERROR;
}

cujpegxl_status cujpegxl_encoder_encode(cujpegxl_encoder* encoder, const cujpegxl_nv12_input* input,
                                        cujpegxl_output* output) {
    if (encoder == nullptr || input == nullptr || output == nullptr || output->data == nullptr ||
        input->luma == 0 || input->chroma == 0) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    const cujpegxl_status st{validate_config(encoder->config, encoder->allow_single)};
    if (st != CUJPEGXL_OK) return st;
    if (input->luma_pitch < encoder->config.width || input->chroma_pitch < encoder->config.width) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    DeviceScope scope{encoder->device};
    if (!scope.ok() || !prepare(encoder)) return CUJPEGXL_INTERNAL_ERROR;
    if (!enqueue_frame(encoder, reinterpret_cast<const std::uint8_t*>(input->luma), input->luma_pitch,
                       reinterpret_cast<const std::uint8_t*>(input->chroma), input->chroma_pitch)) {
        return CUJPEGXL_INTERNAL_ERROR;
    }
    return finish(encoder, output);
}

void cujpegxl_encoder_destroy(cujpegxl_encoder* encoder) {
    if (encoder == nullptr) return;
    {
        DeviceScope scope{encoder->device};
        if (encoder->stream) {
            cudaStreamSynchronize(encoder->stream);
            release_stream(encoder->stream);
        }
        release(encoder);
    }
    delete encoder;
}

cujpegxl_status cujpegxl_b200_encoder_set_debug(cujpegxl_encoder* encoder, int32_t enable) {
    if (encoder == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    const bool want{enable != 0};
    if (want == encoder->debug) return CUJPEGXL_OK;
    DeviceScope scope{encoder->device};
    cudaStreamSynchronize(encoder->stream);
    encoder->debug = want;
    release(encoder);
    return prepare(encoder) ? CUJPEGXL_OK : CUJPEGXL_INTERNAL_ERROR;
}

cujpegxl_status cujpegxl_b200_encoder_read_planes(cujpegxl_encoder* encoder, const cujpegxl_b200_planes* host) {
    if (encoder == nullptr || host == nullptr || encoder->arena == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    DeviceScope scope{encoder->device};
    if (cudaStreamSynchronize(encoder->stream) != cudaSuccess) return CUJPEGXL_INTERNAL_ERROR;
    const std::size_t W{encoder->config.width};
    const std::size_t H{encoder->config.height};
    const std::size_t nb{(W / 8) * (H / 8)};
    const std::size_t nt{((W / 8 + 7) / 8) * ((H / 8 + 7) / 8)};
    struct Copy {
        void* dst;
        const void* src;
        std::size_t bytes;
    };
    const Copy copies[]{
        {host->ac, encoder->fo.ac, 3 * nb * 64 * 2},
        {host->dc, encoder->fo.dc, 3 * nb * 4},
        {host->acs, encoder->fo.acs, nb},
        {host->qf, encoder->fo.qf, nb * 4},
        {host->ytox, encoder->fo.ytox, nt},
        {host->ytob, encoder->fo.ytob, nt},
        {host->xyb, encoder->dbg_xyb, 3 * W * H * 4},
        {host->sharp, encoder->dbg_sharp, 3 * W * H * 4},
        {host->coeff, encoder->dbg_coeff, 3 * nb * 64 * 2},
        {host->cost, encoder->dbg_cost, 3 * nb * 4},
    };
    for (const Copy& c : copies) {
        if (c.dst == nullptr) continue;
        if (c.src == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
        if (cudaMemcpy(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost) != cudaSuccess) return CUJPEGXL_INTERNAL_ERROR;
    }
    return CUJPEGXL_OK;
}

cujpegxl_status cujpegxl_b200_encode_planes(cujpegxl_encoder* encoder, const cujpegxl_b200_planes* host,
                                            uint32_t global_scale, uint32_t quant_dc, cujpegxl_output* output) {
    if (encoder == nullptr || host == nullptr || output == nullptr || output->data == nullptr ||
        host->ac == nullptr || host->dc == nullptr || host->acs == nullptr || host->qf == nullptr ||
        host->ytox == nullptr || host->ytob == nullptr) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    DeviceScope scope{encoder->device};
    if (!scope.ok() || !prepare(encoder)) return CUJPEGXL_INTERNAL_ERROR;
    const std::size_t W{encoder->config.width};
    const std::size_t H{encoder->config.height};
    const std::size_t nb{(W / 8) * (H / 8)};
    const std::size_t nt{((W / 8 + 7) / 8) * ((H / 8 + 7) / 8)};
    std::uint32_t nbits{0};
    const std::vector<std::uint8_t> dcg{jxb::dc_global_bits(global_scale, quant_dc, &nbits)};
    cudaStream_t st{encoder->stream};
    bool ok{cudaMemcpyAsync(encoder->fo.ac, host->ac, 3 * nb * 64 * 2, cudaMemcpyHostToDevice, st) == cudaSuccess &&
            cudaMemcpyAsync(encoder->fo.dc, host->dc, 3 * nb * 4, cudaMemcpyHostToDevice, st) == cudaSuccess &&
            cudaMemcpyAsync(encoder->fo.acs, host->acs, nb, cudaMemcpyHostToDevice, st) == cudaSuccess &&
            cudaMemcpyAsync(encoder->fo.qf, host->qf, nb * 4, cudaMemcpyHostToDevice, st) == cudaSuccess &&
            cudaMemcpyAsync(encoder->fo.ytox, host->ytox, nt, cudaMemcpyHostToDevice, st) == cudaSuccess &&
            cudaMemcpyAsync(encoder->fo.ytob, host->ytob, nt, cudaMemcpyHostToDevice, st) == cudaSuccess &&
            cudaMemcpyAsync(encoder->dc_global_dev, dcg.data(), dcg.size(), cudaMemcpyHostToDevice, st) == cudaSuccess &&
            cudaStreamSynchronize(st) == cudaSuccess};
    if (!ok) return CUJPEGXL_INTERNAL_ERROR;
    // The DcGlobal blob now belongs to these planes; force a refresh on the next encode.
    encoder->geo_distance = -1.0f;
    const std::uint32_t saved_bits{encoder->ed.dc_global_bits};
    encoder->ed.dc_global_bits = nbits;
    nz_kernel<<<static_cast<unsigned>((nb + 255) / 256), 256, 0, st>>>(
        encoder->fo.ac, encoder->fo.acs, static_cast<int>(W / 8), static_cast<int>(H / 8), encoder->fo.nzn,
        encoder->fo.nzc);
    ok = cudaGetLastError() == cudaSuccess && jxb::entropy_launch(encoder->ed, st);
    encoder->ed.dc_global_bits = saved_bits;
    if (!ok) return CUJPEGXL_INTERNAL_ERROR;
    return finish(encoder, output);
}

cujpegxl_status cujpegxl_b200_encode_host(cujpegxl_encoder* encoder, const uint8_t* nv12, size_t nv12_size,
                                          cujpegxl_output* output) {
    if (encoder == nullptr || nv12 == nullptr || output == nullptr || output->data == nullptr) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    const std::size_t W{encoder->config.width};
    const std::size_t H{encoder->config.height};
    if (nv12_size != W * H * 3 / 2) return CUJPEGXL_INVALID_ARGUMENT;
    DeviceScope scope{encoder->device};
    if (!scope.ok() || !prepare(encoder)) return CUJPEGXL_INTERNAL_ERROR;
    std::memcpy(encoder->nv12_pinned, nv12, nv12_size);
    if (cudaMemcpyAsync(encoder->nv12_dev, encoder->nv12_pinned, nv12_size, cudaMemcpyHostToDevice,
                        encoder->stream) != cudaSuccess ||
        !enqueue_frame(encoder, encoder->nv12_dev, W, encoder->nv12_dev + W * H, W)) {
        return CUJPEGXL_INTERNAL_ERROR;
    }
    return finish(encoder, output);
}

cujpegxl_status cujpegxl_b200_encoder_enqueue(cujpegxl_encoder* encoder, const cujpegxl_nv12_input* input) {
    if (encoder == nullptr || input == nullptr || input->luma == 0 || input->chroma == 0 ||
        input->luma_pitch < encoder->config.width || input->chroma_pitch < encoder->config.width) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    DeviceScope scope{encoder->device};
    if (!scope.ok() || !prepare(encoder)) return CUJPEGXL_INTERNAL_ERROR;
    if (!enqueue_frame(encoder, reinterpret_cast<const std::uint8_t*>(input->luma), input->luma_pitch,
                       reinterpret_cast<const std::uint8_t*>(input->chroma), input->chroma_pitch)) {
        return CUJPEGXL_INTERNAL_ERROR;
    }
    encoder->pending = true;
    return CUJPEGXL_OK;
}

cujpegxl_status cujpegxl_b200_encoder_enqueue_stages(cujpegxl_encoder* encoder,
                                                     const cujpegxl_nv12_input* input, uint32_t stages) {
    if (encoder == nullptr || input == nullptr || input->luma == 0 || input->chroma == 0 ||
        input->luma_pitch < encoder->config.width || input->chroma_pitch < encoder->config.width ||
        stages == 0 || stages > 3) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    DeviceScope scope{encoder->device};
    if (!scope.ok() || !prepare(encoder)) return CUJPEGXL_INTERNAL_ERROR;
    if (!enqueue_frame(encoder, reinterpret_cast<const std::uint8_t*>(input->luma), input->luma_pitch,
                       reinterpret_cast<const std::uint8_t*>(input->chroma), input->chroma_pitch, stages)) {
        return CUJPEGXL_INTERNAL_ERROR;
    }
    encoder->pending = true;
    return CUJPEGXL_OK;
}

cujpegxl_status cujpegxl_b200_encoder_result(cujpegxl_encoder* encoder, size_t* out_size,
                                             uintptr_t* out_device_bytes) {
    if (encoder == nullptr || out_size == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    DeviceScope scope{encoder->device};
    if (cudaMemcpyAsync(encoder->result_pinned, encoder->ed.result, 4 * 8, cudaMemcpyDeviceToHost,
                        encoder->stream) != cudaSuccess ||
        cudaStreamSynchronize(encoder->stream) != cudaSuccess) {
        return CUJPEGXL_INTERNAL_ERROR;
    }
    encoder->pending = false;
    if (encoder->result_pinned[2] != 0) return CUJPEGXL_INTERNAL_ERROR;
    *out_size = static_cast<std::size_t>(encoder->result_pinned[0]);
    if (out_device_bytes != nullptr) *out_device_bytes = reinterpret_cast<uintptr_t>(encoder->ed.out);
    return CUJPEGXL_OK;
}

cujpegxl_status cujpegxl_b200_encoder_enqueue_readback(cujpegxl_encoder* encoder, uint8_t* host_dst,
                                                      size_t capacity, uint64_t* host_words) {
    if (encoder == nullptr || host_dst == nullptr || host_words == nullptr || encoder->arena == nullptr) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    DeviceScope scope{encoder->device};
    if (!scope.ok()) return CUJPEGXL_INTERNAL_ERROR;
    if ((reinterpret_cast<std::uintptr_t>(host_words) & 7u) != 0 || !device_reachable_host(host_dst) ||
        !device_reachable_host(host_words)) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    return enqueue_readback(encoder, host_dst, capacity, reinterpret_cast<unsigned long long*>(host_words),
                            encoder->stream)
               ? CUJPEGXL_OK
               : CUJPEGXL_INTERNAL_ERROR;
}

cujpegxl_status cujpegxl_b200_encoder_stream(cujpegxl_encoder* encoder, uintptr_t* out_stream) {
    if (encoder == nullptr || out_stream == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    *out_stream = reinterpret_cast<uintptr_t>(encoder->stream);
    return CUJPEGXL_OK;
}

cujpegxl_status cujpegxl_b200_encoder_memory(cujpegxl_encoder* encoder, size_t* device_bytes,
                                             size_t* pinned_host_bytes) {
    if (encoder == nullptr || device_bytes == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    *device_bytes = encoder->arena_bytes;
    if (pinned_host_bytes != nullptr) {
        *pinned_host_bytes = encoder->nv12_pinned != nullptr
                                 ? static_cast<std::size_t>(encoder->geo_w) * encoder->geo_h * 3 / 2 + 64
                                 : 0;
    }
    return CUJPEGXL_OK;
}

uint32_t cujpegxl_b200_kernels_per_encode(void) { return 12u; }

void cujpegxl_b200_debug_fail_allocation(uint32_t nth) { g_fail_countdown.store(nth); }

uint64_t cujpegxl_b200_debug_live_allocations(void) { return g_live.load(); }

cujpegxl_status cujpegxl_b200_debug_prefix_code(int32_t device_ordinal, const uint32_t* hist, uint32_t length,
                                                uint8_t* depth, uint16_t* bits, uint8_t* header,
                                                size_t header_cap, uint32_t* header_bits) {
    if (hist == nullptr || depth == nullptr || bits == nullptr || header == nullptr || header_bits == nullptr ||
        length == 0 || length > 256 || header_cap < static_cast<size_t>(jxb::kDescBytes)) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    int major{0};
    int minor{0};
    if (!device_exists(device_ordinal, &major, &minor)) return CUJPEGXL_NO_DEVICE;
    DeviceScope scope{device_ordinal};
    if (!scope.ok()) return CUJPEGXL_INTERNAL_ERROR;
    return jxb::prefix_code_test(hist, static_cast<int>(length), depth, bits, header, header_cap, header_bits)
               ? CUJPEGXL_OK
               : CUJPEGXL_INTERNAL_ERROR;
}

cujpegxl_status cujpegxl_b200_encoder_set_acsnet(cujpegxl_encoder* encoder, const cujpegxl_b200_acsnet* net,
                                                 float margin, uint32_t flags) {
    if (encoder == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    if (net == nullptr) {
        encoder->net = nullptr;
        encoder->net_flags = 0;
        return CUJPEGXL_OK;
    }
    if (!(margin >= 0.0f && margin <= 1.0f) || (flags & CUJPEGXL_B200_ACSNET_SPLIT) == 0 ||
        (flags & ~(CUJPEGXL_B200_ACSNET_SPLIT | CUJPEGXL_B200_ACSNET_QF)) != 0 ||
        jxb::acsnet_device(net) != encoder->device) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    encoder->net = net;
    encoder->net_margin = margin;
    encoder->net_flags = flags;
    return CUJPEGXL_OK;
}

cujpegxl_status cujpegxl_b200_encoder_acsnet_stats(cujpegxl_encoder* encoder, uint32_t* decided,
                                                   uint32_t* regions) {
    if (encoder == nullptr || decided == nullptr || regions == nullptr || encoder->arena == nullptr) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    DeviceScope scope{encoder->device};
    const std::size_t rw{(encoder->geo_w / 8 + 3) / 4};
    const std::size_t rh{(encoder->geo_h / 8 + 3) / 4};
    std::vector<std::int8_t> cls(rw * rh);
    if (!scope.ok() || cudaStreamSynchronize(encoder->stream) != cudaSuccess ||
        cudaMemcpy(cls.data(), encoder->net_class, cls.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
        return CUJPEGXL_INTERNAL_ERROR;
    }
    std::uint32_t d{0};
    for (const std::int8_t c : cls) d += c >= 0 ? 1u : 0u;
    *decided = encoder->net != nullptr ? d : 0u;
    *regions = static_cast<std::uint32_t>((encoder->geo_w / 32) * (encoder->geo_h / 32));
    return CUJPEGXL_OK;
}

}  // extern "C"
