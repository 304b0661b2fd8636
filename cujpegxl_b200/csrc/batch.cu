// Batched encode: many frames, each with its own geometry and distance, in one
// CUDA graph launch.
//
// Every frame keeps its own encoder (arena, tables, output buffer), but the
// work is not run frame by frame: the graph holds one persistent frontend
// launch whose resident CTAs take the 64x64 tiles of all frames from one work
// list (frontend_batch_launch), then one launch per entropy pass that runs
// every frame's blocks of that pass (entropy_batch_launch), then a gather of
// every frame's result words and their copy to pinned host memory. With a
// transform-decision network attached, each frame's inference runs in front of
// the frontend launch.
//
// The schedule of the frontend launch (resident CTAs, tiles per claim,
// claims from a counter or round-robin, frames largest-first or in the given
// order) is picked on the first encode by timing every candidate graph, and
// cached per geometry mix for later batches. A later encode with the same
// input addresses relaunches the graph as it is; new addresses are captured
// again and the executable graph is updated in place.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <numeric>
#include <vector>

#include "cujpegxl/cujpegxl.h"
#include "cujpegxl_b200/cujpegxl_b200.h"
#include "encoder_internal.h"

namespace {

constexpr int kResultWords = 3;  // total bytes, body start, status

__global__ void gather_results(const unsigned long long* const* src, int count, unsigned long long* dst) {
    const int i{static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x)};
    if (i >= count) return;
    for (int w{0}; w < kResultWords; ++w) dst[kResultWords * i + w] = src[i][w];
}

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

bool same_inputs(const std::vector<cujpegxl_nv12_input>& a, const cujpegxl_nv12_input* b) {
    for (std::size_t i{0}; i < a.size(); ++i) {
        if (a[i].luma != b[i].luma || a[i].chroma != b[i].chroma || a[i].luma_pitch != b[i].luma_pitch ||
            a[i].chroma_pitch != b[i].chroma_pitch) {
            return false;
        }
    }
    return true;
}

// The frontend launch schedule the autotuner chooses among: CTAs of two
// tiles at a time (paired, one per SM) or of one tile (ctas_per_sm per SM).
struct Schedule {
    bool paired{true};
    int ctas_per_sm{1};
    int chunk{1};
    bool dynamic{true};
    bool largest_first{true};
    float ms{0.0f};  // measured time of one batch with it
};

// Tuned schedules of earlier batches, keyed by device, network use and the
// frames' geometries in order.
std::mutex g_cache_mutex;
std::map<std::vector<std::uint64_t>, Schedule> g_cache;

}  // namespace

struct cujpegxl_b200_batch {
    int device{0};
    int sms{0};
    std::vector<cujpegxl_encoder*> encs;
    std::vector<std::size_t> pixels;
    std::vector<std::uint32_t> widths;
    cudaStream_t root{nullptr};
    std::uint32_t* counters{nullptr};                 // device, one frontend claim counter per group
    const unsigned long long** result_ptrs{nullptr};  // device [count]
    unsigned long long* gathered{nullptr};            // device [count][3]
    unsigned long long* gathered_host{nullptr};       // pinned [count][3]
    cudaGraphExec_t exec{nullptr};
    std::vector<cujpegxl_nv12_input> bound;
    Schedule schedule{};
    bool tuned{false};
    bool from_cache{false};
    bool launched{false};
};

namespace {

void release(cujpegxl_b200_batch* b) {
    DeviceScope scope{b->device};
    if (b->root) cudaStreamSynchronize(b->root);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->root) cudaStreamDestroy(b->root);
    if (b->counters) cudaFree(b->counters);
    if (b->result_ptrs) cudaFree(b->result_ptrs);
    if (b->gathered) cudaFree(b->gathered);
    if (b->gathered_host) cudaFreeHost(b->gathered_host);
    for (cujpegxl_encoder* e : b->encs) cujpegxl_encoder_destroy(e);
}

std::size_t groups_of(std::size_t count) {
    return (count + jxb::kBatchFrames - 1) / jxb::kBatchFrames;
}

// Records the whole batch on the root stream as a graph with schedule `sc`:
// frames in groups of at most kBatchFrames, each group one frontend launch
// and one launch per entropy pass.
bool capture(cujpegxl_b200_batch* b, const cujpegxl_nv12_input* inputs, const Schedule& sc, cudaGraph_t* graph) {
    const std::size_t count{b->encs.size()};
    std::vector<std::size_t> order(count);
    std::iota(order.begin(), order.end(), std::size_t{0});
    if (sc.largest_first) {
        std::stable_sort(order.begin(), order.end(),
                         [&](std::size_t x, std::size_t y) { return b->pixels[x] > b->pixels[y]; });
    }
    if (cudaStreamBeginCapture(b->root, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return false;
    bool ok{true};
    auto* fb{new (std::nothrow) jxb::FrontendBatch{}};
    auto* eb{new (std::nothrow) jxb::EntropyBatch{}};
    ok = fb != nullptr && eb != nullptr;
    for (std::size_t g0{0}, grp{0}; ok && g0 < count; g0 += jxb::kBatchFrames, ++grp) {
        const std::size_t n{std::min<std::size_t>(jxb::kBatchFrames, count - g0)};
        std::uint32_t tiles{0};
        for (std::size_t k{0}; ok && k < n; ++k) {
            const std::size_t i{order[g0 + k]};
            jxb::FrontendJob& job{fb->jobs[k]};
            ok = jxb::encoder_frontend_job(b->encs[i], inputs[i], b->root, &job, &fb->tb);
            job.tile_begin = tiles;
            const std::uint32_t th{(static_cast<std::uint32_t>(job.in.height) + 63) / 64};
            tiles += static_cast<std::uint32_t>(job.tiles_x) * th;
            eb->frames[k] = jxb::encoder_entropy(b->encs[i]);
        }
        if (!ok) break;
        fb->nframes = static_cast<int>(n);
        fb->chunk = sc.chunk;
        fb->total_tiles = tiles;
        fb->counter = sc.dynamic ? b->counters + grp : nullptr;
        eb->nframes = static_cast<int>(n);
        jxb::entropy_batch_plan(*eb);
        ok = (!sc.dynamic || cudaMemsetAsync(fb->counter, 0, sizeof(std::uint32_t), b->root) == cudaSuccess) &&
             jxb::frontend_batch_launch(*fb, sc.ctas_per_sm * b->sms, sc.paired, b->root) &&
             jxb::entropy_batch_launch(*eb, b->root);
    }
    delete fb;
    delete eb;
    const int icount{static_cast<int>(count)};
    if (ok) {
        gather_results<<<(icount + 127) / 128, 128, 0, b->root>>>(b->result_ptrs, icount, b->gathered);
        ok = cudaGetLastError() == cudaSuccess &&
             cudaMemcpyAsync(b->gathered_host, b->gathered, sizeof(unsigned long long) * kResultWords * count,
                             cudaMemcpyDeviceToHost, b->root) == cudaSuccess;
    }
    cudaGraph_t g{nullptr};
    const bool ended{cudaStreamEndCapture(b->root, &g) == cudaSuccess};
    if (!ok || !ended) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return false;
    }
    *graph = g;
    return true;
}

bool instantiate(cujpegxl_b200_batch* b, const cujpegxl_nv12_input* inputs, const Schedule& sc,
                 cudaGraphExec_t* exec) {
    cudaGraph_t g{nullptr};
    if (!capture(b, inputs, sc, &g)) return false;
    const bool ok{cudaGraphInstantiate(exec, g, 0) == cudaSuccess};
    cudaGraphDestroy(g);
    return ok;
}

// The CTA shape the environment restricts the candidates to, if any
// (CUJPEGXL_B200_BATCH_TILES_PER_CTA = 1 or 2), so that tests can check both
// shapes' output; 0 otherwise.
int forced_tiles_per_cta() {
    const char* v{std::getenv("CUJPEGXL_B200_BATCH_TILES_PER_CTA")};
    if (v == nullptr) return 0;
    return std::strcmp(v, "1") == 0 ? 1 : (std::strcmp(v, "2") == 0 ? 2 : 0);
}

std::vector<std::uint64_t> cache_key(const cujpegxl_b200_batch* b) {
    std::vector<std::uint64_t> key{static_cast<std::uint64_t>(b->device)};
    for (cujpegxl_encoder* e : b->encs) {
        const jxb::EntropyDev& ed{jxb::encoder_entropy(e)};
        key.push_back((static_cast<std::uint64_t>(ed.width) << 32) | static_cast<std::uint64_t>(ed.height));
    }
    key.push_back(jxb::encoder_has_network(b->encs.front()) ? 1u : 0u);
    key.push_back(static_cast<std::uint64_t>(forced_tiles_per_cta()));
    return key;
}

// The candidates: paired CTAs (one per SM, two tiles at a time) and
// single-tile CTAs (two per SM), each with dynamic claims of 1, 2 or 4 tiles
// (per half, when paired) or round-robin claims of single tiles, and the
// frames largest-first or in the given order.
std::vector<Schedule> candidates() {
    const int forced{forced_tiles_per_cta()};
    std::vector<Schedule> out;
    for (const bool largest : {true, false}) {
        for (const bool paired : {true, false}) {
            if (forced != 0 && forced != (paired ? 2 : 1)) continue;
            const int per_sm{paired ? 1 : 2};
            for (const int chunk : {1, 2, 4}) out.push_back(Schedule{paired, per_sm, chunk, true, largest, 0.0f});
            out.push_back(Schedule{paired, per_sm, 1, false, largest, 0.0f});
        }
    }
    return out;
}

// Times every candidate schedule on the given inputs (one warm-up and two
// timed launches each) and keeps the fastest graph; a geometry mix tuned
// before reuses its schedule without timing.
bool autotune(cujpegxl_b200_batch* b, const cujpegxl_nv12_input* inputs) {
    const std::vector<std::uint64_t> key{cache_key(b)};
    {
        std::lock_guard<std::mutex> lock(g_cache_mutex);
        const auto it{g_cache.find(key)};
        if (it != g_cache.end()) {
            cudaGraphExec_t exec{nullptr};
            if (!instantiate(b, inputs, it->second, &exec)) return false;
            b->exec = exec;
            b->schedule = it->second;
            b->tuned = true;
            b->from_cache = true;
            return true;
        }
    }
    cudaEvent_t t0{nullptr};
    cudaEvent_t t1{nullptr};
    if (cudaEventCreate(&t0) != cudaSuccess || cudaEventCreate(&t1) != cudaSuccess) return false;
    cudaGraphExec_t best{nullptr};
    Schedule best_sc{};
    bool ok{true};
    for (Schedule sc : candidates()) {
        cudaGraphExec_t exec{nullptr};
        if (!instantiate(b, inputs, sc, &exec)) {
            ok = false;
            break;
        }
        float ms{0.0f};
        ok = cudaGraphLaunch(exec, b->root) == cudaSuccess && cudaEventRecord(t0, b->root) == cudaSuccess;
        for (int r{0}; ok && r < 2; ++r) ok = cudaGraphLaunch(exec, b->root) == cudaSuccess;
        ok = ok && cudaEventRecord(t1, b->root) == cudaSuccess && cudaEventSynchronize(t1) == cudaSuccess &&
             cudaEventElapsedTime(&ms, t0, t1) == cudaSuccess;
        if (!ok) {
            cudaGraphExecDestroy(exec);
            break;
        }
        sc.ms = ms / 2.0f;
        if (best == nullptr || sc.ms < best_sc.ms) {
            if (best) cudaGraphExecDestroy(best);
            best = exec;
            best_sc = sc;
        } else {
            cudaGraphExecDestroy(exec);
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (!ok || best == nullptr) {
        if (best) cudaGraphExecDestroy(best);
        return false;
    }
    b->exec = best;
    b->schedule = best_sc;
    b->tuned = true;
    b->from_cache = false;
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    g_cache[key] = best_sc;
    return true;
}

}  // namespace

extern "C" {

cujpegxl_status cujpegxl_b200_batch_create(const cujpegxl_config* frames, size_t count,
                                           cujpegxl_b200_batch** out_batch) {
    if (frames == nullptr || out_batch == nullptr || count == 0) return CUJPEGXL_INVALID_ARGUMENT;
    *out_batch = nullptr;
    for (size_t i{0}; i < count; ++i) {
        if (frames[i].device_ordinal != frames[0].device_ordinal) return CUJPEGXL_INVALID_ARGUMENT;
    }
    auto* b{new (std::nothrow) cujpegxl_b200_batch{}};
    if (b == nullptr) return CUJPEGXL_INTERNAL_ERROR;
    b->device = frames[0].device_ordinal;
    for (size_t i{0}; i < count; ++i) {
        cujpegxl_encoder* e{nullptr};
        const cujpegxl_status st{cujpegxl_encoder_create(&frames[i], &e)};
        if (st != CUJPEGXL_OK) {
            release(b);
            delete b;
            return st;
        }
        b->encs.push_back(e);
        b->pixels.push_back(static_cast<std::size_t>(frames[i].width) * frames[i].height);
        b->widths.push_back(frames[i].width);
    }
    DeviceScope scope{b->device};
    bool ok{scope.ok() && cudaStreamCreateWithFlags(&b->root, cudaStreamNonBlocking) == cudaSuccess &&
            cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device) == cudaSuccess};
    std::vector<const unsigned long long*> ptrs(count);
    for (size_t i{0}; i < count; ++i) ptrs[i] = jxb::encoder_result_words(b->encs[i]);
    ok = ok && cudaMalloc(reinterpret_cast<void**>(&b->counters), sizeof(std::uint32_t) * groups_of(count)) ==
                   cudaSuccess &&
         cudaMalloc(reinterpret_cast<void**>(&b->result_ptrs), sizeof(void*) * count) == cudaSuccess &&
         cudaMalloc(reinterpret_cast<void**>(&b->gathered), sizeof(unsigned long long) * kResultWords * count) ==
             cudaSuccess &&
         cudaHostAlloc(reinterpret_cast<void**>(&b->gathered_host), sizeof(unsigned long long) * kResultWords * count,
                       cudaHostAllocDefault) == cudaSuccess &&
         cudaMemcpy(b->result_ptrs, ptrs.data(), sizeof(void*) * count, cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) {
        release(b);
        delete b;
        return CUJPEGXL_INTERNAL_ERROR;
    }
    *out_batch = b;
    return CUJPEGXL_OK;
}

cujpegxl_status cujpegxl_b200_batch_encode(cujpegxl_b200_batch* batch, const cujpegxl_nv12_input* inputs) {
    if (batch == nullptr || inputs == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    for (size_t i{0}; i < batch->encs.size(); ++i) {
        if (inputs[i].luma == 0 || inputs[i].chroma == 0 || inputs[i].luma_pitch < batch->widths[i] ||
            inputs[i].chroma_pitch < batch->widths[i]) {
            return CUJPEGXL_INVALID_ARGUMENT;
        }
    }
    DeviceScope scope{batch->device};
    if (!scope.ok()) return CUJPEGXL_INTERNAL_ERROR;
    for (cujpegxl_encoder* e : batch->encs) {
        if (!jxb::encoder_prepare(e)) return CUJPEGXL_INTERNAL_ERROR;
    }
    if (batch->exec == nullptr) {
        if (!autotune(batch, inputs)) return CUJPEGXL_INTERNAL_ERROR;
        batch->bound.assign(inputs, inputs + batch->encs.size());
    } else if (!same_inputs(batch->bound, inputs)) {
        cudaGraph_t g{nullptr};
        if (!capture(batch, inputs, batch->schedule, &g)) return CUJPEGXL_INTERNAL_ERROR;
        cudaGraphExecUpdateResultInfo info{};
        if (cudaGraphExecUpdate(batch->exec, g, &info) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphExecDestroy(batch->exec);
            batch->exec = nullptr;
            const bool ok{cudaGraphInstantiate(&batch->exec, g, 0) == cudaSuccess};
            cudaGraphDestroy(g);
            if (!ok) return CUJPEGXL_INTERNAL_ERROR;
        } else {
            cudaGraphDestroy(g);
        }
        batch->bound.assign(inputs, inputs + batch->encs.size());
    }
    if (cudaGraphLaunch(batch->exec, batch->root) != cudaSuccess) return CUJPEGXL_INTERNAL_ERROR;
    batch->launched = true;
    return CUJPEGXL_OK;
}

cujpegxl_status cujpegxl_b200_batch_sync(cujpegxl_b200_batch* batch, size_t* sizes) {
    if (batch == nullptr || !batch->launched) return CUJPEGXL_INVALID_ARGUMENT;
    DeviceScope scope{batch->device};
    if (!scope.ok() || cudaStreamSynchronize(batch->root) != cudaSuccess) return CUJPEGXL_INTERNAL_ERROR;
    cujpegxl_status st{CUJPEGXL_OK};
    for (size_t i{0}; i < batch->encs.size(); ++i) {
        const unsigned long long* r{batch->gathered_host + kResultWords * i};
        if (sizes != nullptr) sizes[i] = static_cast<size_t>(r[0]);
        if (r[2] != 0) st = CUJPEGXL_INTERNAL_ERROR;
    }
    return st;
}

cujpegxl_status cujpegxl_b200_batch_frame(cujpegxl_b200_batch* batch, size_t index, size_t* size,
                                          uintptr_t* device_bytes) {
    if (batch == nullptr || index >= batch->encs.size() || size == nullptr || !batch->launched) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    const unsigned long long* r{batch->gathered_host + kResultWords * index};
    if (r[2] != 0) return CUJPEGXL_INTERNAL_ERROR;
    *size = static_cast<size_t>(r[0]);
    if (device_bytes != nullptr) {
        *device_bytes = reinterpret_cast<uintptr_t>(jxb::encoder_output(batch->encs[index]));
    }
    return CUJPEGXL_OK;
}

cujpegxl_status cujpegxl_b200_batch_copy(cujpegxl_b200_batch* batch, size_t index, cujpegxl_output* output) {
    if (output == nullptr || output->data == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    size_t size{0};
    uintptr_t dev{0};
    const cujpegxl_status st{cujpegxl_b200_batch_frame(batch, index, &size, &dev)};
    if (st != CUJPEGXL_OK) return st;
    if (size > output->capacity) {
        output->size = size;
        return CUJPEGXL_BUFFER_TOO_SMALL;
    }
    DeviceScope scope{batch->device};
    if (!scope.ok() ||
        cudaMemcpy(output->data, reinterpret_cast<const void*>(dev), size, cudaMemcpyDeviceToHost) != cudaSuccess) {
        return CUJPEGXL_INTERNAL_ERROR;
    }
    output->size = size;
    return CUJPEGXL_OK;
}

cujpegxl_status cujpegxl_b200_batch_set_acsnet(cujpegxl_b200_batch* batch, const cujpegxl_b200_acsnet* net,
                                               float margin, uint32_t flags) {
    if (batch == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    DeviceScope scope{batch->device};
    if (!scope.ok() || cudaStreamSynchronize(batch->root) != cudaSuccess) return CUJPEGXL_INTERNAL_ERROR;
    for (cujpegxl_encoder* e : batch->encs) {
        const cujpegxl_status st{cujpegxl_b200_encoder_set_acsnet(e, net, margin, flags)};
        if (st != CUJPEGXL_OK) {
            for (cujpegxl_encoder* u : batch->encs) cujpegxl_b200_encoder_set_acsnet(u, nullptr, 0.0f, 0u);
            return st;
        }
    }
    // The captured launch sequence changes: the next encode captures (and
    // tunes) the graph again.
    if (batch->exec != nullptr) {
        cudaGraphExecDestroy(batch->exec);
        batch->exec = nullptr;
    }
    batch->launched = false;
    return CUJPEGXL_OK;
}

cujpegxl_status cujpegxl_b200_batch_stream(const cujpegxl_b200_batch* batch, uintptr_t* stream) {
    if (batch == nullptr || stream == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    *stream = reinterpret_cast<uintptr_t>(batch->root);
    return CUJPEGXL_OK;
}

uint32_t cujpegxl_b200_batch_lanes(const cujpegxl_b200_batch* batch) {
    return batch == nullptr || !batch->tuned ? 0u : 1u;
}

cujpegxl_status cujpegxl_b200_batch_schedule(const cujpegxl_b200_batch* batch,
                                             cujpegxl_b200_batch_schedule_info* out) {
    if (batch == nullptr || out == nullptr || !batch->tuned) return CUJPEGXL_INVALID_ARGUMENT;
    out->frontend_ctas = static_cast<uint32_t>(batch->schedule.ctas_per_sm * batch->sms);
    out->tiles_per_cta = batch->schedule.paired ? 2u : 1u;
    out->tiles_per_claim = static_cast<uint32_t>(batch->schedule.chunk);
    out->dynamic_claims = batch->schedule.dynamic ? 1u : 0u;
    out->largest_first = batch->schedule.largest_first ? 1u : 0u;
    out->from_cache = batch->from_cache ? 1u : 0u;
    out->candidates = static_cast<uint32_t>(candidates().size());
    out->tuned_ms = batch->schedule.ms;
    return CUJPEGXL_OK;
}

void cujpegxl_b200_batch_destroy(cujpegxl_b200_batch* batch) {
    if (batch == nullptr) return;
    release(batch);
    delete batch;
}

}  // extern "C"
