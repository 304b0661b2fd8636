// Batched encode: many frames, each with its own geometry and distance, in one
// CUDA graph launch.
//
// Every frame has its own encoder (arena, tables, output buffer). The graph
// forks from a root stream into L lanes, encodes the frames on the lanes
// (largest frames first, each to the lane with the least work so far), joins
// the lanes, gathers every frame's result words with one small kernel and
// copies them to pinned host memory. L is chosen on the first encode by
// timing graphs with 1, 2, 4 and 8 lanes. A later encode with the same input
// addresses relaunches the graph as it is; new addresses are captured again
// and the executable graph is updated in place.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "cujpegxl/cujpegxl.h"
#include "cujpegxl_b200/cujpegxl_b200.h"
#include "encoder_internal.h"

namespace {

constexpr int kMaxLanes = 8;
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

}  // namespace

struct cujpegxl_b200_batch {
    int device{0};
    std::vector<cujpegxl_encoder*> encs;
    std::vector<std::size_t> order;  // frames by pixel count, largest first
    std::vector<std::size_t> pixels;
    std::vector<std::uint32_t> widths;
    cudaStream_t root{nullptr};
    cudaStream_t lanes[kMaxLanes]{};
    cudaEvent_t fork{nullptr};
    cudaEvent_t join[kMaxLanes]{};
    const unsigned long long** result_ptrs{nullptr};  // device [count]
    unsigned long long* gathered{nullptr};            // device [count][3]
    unsigned long long* gathered_host{nullptr};       // pinned [count][3]
    cudaGraphExec_t exec{nullptr};
    std::vector<cujpegxl_nv12_input> bound;
    int lanes_used{0};
    bool launched{false};
};

namespace {

void release(cujpegxl_b200_batch* b) {
    DeviceScope scope{b->device};
    if (b->root) cudaStreamSynchronize(b->root);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    for (int l{0}; l < kMaxLanes; ++l) {
        if (b->lanes[l]) cudaStreamDestroy(b->lanes[l]);
        if (b->join[l]) cudaEventDestroy(b->join[l]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->root) cudaStreamDestroy(b->root);
    if (b->result_ptrs) cudaFree(b->result_ptrs);
    if (b->gathered) cudaFree(b->gathered);
    if (b->gathered_host) cudaFreeHost(b->gathered_host);
    for (cujpegxl_encoder* e : b->encs) cujpegxl_encoder_destroy(e);
}

// Records the whole batch on the root stream as a graph with `lanes` lanes.
bool capture(cujpegxl_b200_batch* b, const cujpegxl_nv12_input* inputs, int lanes, cudaGraph_t* graph) {
    if (cudaStreamBeginCapture(b->root, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return false;
    bool ok{cudaEventRecord(b->fork, b->root) == cudaSuccess};
    for (int l{0}; ok && l < lanes; ++l) ok = cudaStreamWaitEvent(b->lanes[l], b->fork, 0) == cudaSuccess;
    std::vector<std::size_t> load(static_cast<std::size_t>(lanes), 0);
    for (std::size_t k{0}; ok && k < b->order.size(); ++k) {
        const std::size_t i{b->order[k]};
        const int l{static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin())};
        load[static_cast<std::size_t>(l)] += b->pixels[i];
        ok = jxb::encoder_launch(b->encs[i], inputs[i], b->lanes[l]);
    }
    for (int l{0}; ok && l < lanes; ++l) {
        ok = cudaEventRecord(b->join[l], b->lanes[l]) == cudaSuccess &&
             cudaStreamWaitEvent(b->root, b->join[l], 0) == cudaSuccess;
    }
    const int count{static_cast<int>(b->encs.size())};
    if (ok) {
        gather_results<<<(count + 127) / 128, 128, 0, b->root>>>(b->result_ptrs, count, b->gathered);
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

bool instantiate(cujpegxl_b200_batch* b, const cujpegxl_nv12_input* inputs, int lanes, cudaGraphExec_t* exec) {
    cudaGraph_t g{nullptr};
    if (!capture(b, inputs, lanes, &g)) return false;
    const bool ok{cudaGraphInstantiate(exec, g, 0) == cudaSuccess};
    cudaGraphDestroy(g);
    return ok;
}

// Times candidate lane counts on the given inputs and keeps the fastest graph.
bool autotune(cujpegxl_b200_batch* b, const cujpegxl_nv12_input* inputs) {
    const int count{static_cast<int>(b->encs.size())};
    cudaEvent_t t0{nullptr};
    cudaEvent_t t1{nullptr};
    if (cudaEventCreate(&t0) != cudaSuccess || cudaEventCreate(&t1) != cudaSuccess) return false;
    float best_ms{0.0f};
    cudaGraphExec_t best{nullptr};
    int best_lanes{0};
    bool ok{true};
    for (int lanes{1}; ok && lanes <= kMaxLanes; lanes *= 2) {
        if (lanes > 1 && lanes > count) break;
        cudaGraphExec_t exec{nullptr};
        if (!instantiate(b, inputs, lanes, &exec)) {
            ok = false;
            break;
        }
        float ms{0.0f};
        ok = cudaGraphLaunch(exec, b->root) == cudaSuccess && cudaEventRecord(t0, b->root) == cudaSuccess;
        for (int r{0}; ok && r < 2; ++r) ok = cudaGraphLaunch(exec, b->root) == cudaSuccess;
        ok = ok && cudaEventRecord(t1, b->root) == cudaSuccess && cudaEventSynchronize(t1) == cudaSuccess &&
             cudaEventElapsedTime(&ms, t0, t1) == cudaSuccess;
        if (ok && (best == nullptr || ms < best_ms)) {
            if (best) cudaGraphExecDestroy(best);
            best = exec;
            best_ms = ms;
            best_lanes = lanes;
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
    b->lanes_used = best_lanes;
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
    b->order.resize(count);
    std::iota(b->order.begin(), b->order.end(), std::size_t{0});
    std::stable_sort(b->order.begin(), b->order.end(),
                     [&](std::size_t x, std::size_t y) { return b->pixels[x] > b->pixels[y]; });
    DeviceScope scope{b->device};
    bool ok{scope.ok() && cudaStreamCreateWithFlags(&b->root, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess};
    for (int l{0}; ok && l < kMaxLanes; ++l) {
        ok = cudaStreamCreateWithFlags(&b->lanes[l], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&b->join[l], cudaEventDisableTiming) == cudaSuccess;
    }
    std::vector<const unsigned long long*> ptrs(count);
    for (size_t i{0}; i < count; ++i) ptrs[i] = jxb::encoder_result_words(b->encs[i]);
    ok = ok && cudaMalloc(reinterpret_cast<void**>(&b->result_ptrs), sizeof(void*) * count) == cudaSuccess &&
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
        if (!capture(batch, inputs, batch->lanes_used, &g)) return CUJPEGXL_INTERNAL_ERROR;
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
    return batch == nullptr ? 0u : static_cast<uint32_t>(batch->lanes_used);
}

void cujpegxl_b200_batch_destroy(cujpegxl_b200_batch* batch) {
    if (batch == nullptr) return;
    release(batch);
    delete batch;
}

}  // extern "C"
