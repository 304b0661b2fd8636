// Library-internal access to an encoder for the batch entry points: launch a
// whole encode on a caller-chosen stream (also inside a stream capture) and
// find its device-side result words and output bytes.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "cujpegxl/cujpegxl.h"
#include "cujpegxl_b200/cujpegxl_b200.h"
#include "entropy.cuh"
#include "frontend.cuh"

namespace jxb {

struct NetParamsDev;

// Device weights and device ordinal of a transform-decision network.
const NetParamsDev* acsnet_params(const cujpegxl_b200_acsnet* net);
int acsnet_device(const cujpegxl_b200_acsnet* net);

// Allocates or refreshes the per-geometry and per-distance state; not
// capturable (it may allocate and upload tables).
bool encoder_prepare(cujpegxl_encoder* e);

// Enqueues one full encode (frontend + entropy + assembly) of `input` on
// `stream`; issues only kernel launches and memsets, so it may be captured.
bool encoder_launch(cujpegxl_encoder* e, const cujpegxl_nv12_input& input, cudaStream_t stream);

// Device words written by the encode: total bytes, body start, status (0 ok).
const unsigned long long* encoder_result_words(const cujpegxl_encoder* e);

// Device address of the encoded file.
const std::uint8_t* encoder_output(const cujpegxl_encoder* e);

// The frontend work of one encode of `input` (validated by the caller) as a
// job of a batched frontend launch, and the device tables it uses. With a
// network attached, its inference is enqueued on `stream` here and the job
// reads the decisions. Issues only kernel launches, so it may be captured.
bool encoder_frontend_job(cujpegxl_encoder* e, const cujpegxl_nv12_input& input, cudaStream_t stream,
                          FrontendJob* job, FrontendTables* tables);

// The encoder's entropy-stage state (valid after encoder_prepare).
const EntropyDev& encoder_entropy(const cujpegxl_encoder* e);

// Whether a transform-decision network is attached.
bool encoder_has_network(const cujpegxl_encoder* e);

}  // namespace jxb
