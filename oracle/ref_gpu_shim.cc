// C entry points over the reference's own device code, for use as a checker
// on a GPU only (test infrastructure; never linked into the product).
//
// build_ref_gpu.py compiles, where they lie under the reference checkout, the
// reference's CUDA translation units that nvcc accepts unchanged and that
// carry the device-only float stages:
//   src/xyb.cu                NV12 -> XYB through the texture unit's bilinear
//                             chroma (nv12_to_xyb);
//   src/frontend_fused.cu     the fused adaptive-quantisation kernel
//                             (encode_frontend -> quant field);
//   src/frontend_transform.cu inverse gaborish and the variable DCT
//                             (frontend_transform, variable_forward_dct).
// The reference builds them with clang as its CUDA compiler. Three of its
// translation units (src/transform_select.cu, src/frontend_quantize.cu,
// src/entropy.cu) read constexpr tables from device code, which nvcc rejects,
// so they are not built: the quantiser and the device entropy coder have no
// reference-device pin here. frontend_transform calls select_transforms,
// which lives in src/transform_select.cu; this file supplies it from the
// reference's host twin of the same decision (src/transform_select_impl.cuh
// decide_region, the code the reference's own test holds equal to its device
// selection), or copies decisions the caller gives, so the DCT can also be
// timed on a fixed transform layout.

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "src/frontend_fused.h"
#include "src/frontend_transform.h"
#include "src/quant_calibration.h"
#include "src/transform_select_impl.cuh"
#include "src/xyb.h"

namespace {
// Device address of caller-given transform decisions for the next
// frontend_transform call, or null for the reference's own decisions.
const std::int8_t* g_given_acs{nullptr};
}  // namespace

namespace cujpegxl {

// The entry point of src/transform_select.cu (transform_select.h:21-22) with
// the reference's host decision loop (select_transforms_host restated: every
// 4x4-block region through decide_region at the calibrated qgsf).
bool select_transforms(const float* y, std::size_t width, std::size_t height, float distance,
                       std::int8_t* acs) {
    const std::size_t bw{width / 8};
    const std::size_t bh{height / 8};
    if (g_given_acs != nullptr) {
        return cudaMemcpy(acs, g_given_acs, bw * bh, cudaMemcpyDeviceToDevice) == cudaSuccess;
    }
    std::vector<float> plane(width * height);
    if (cudaMemcpy(plane.data(), y, plane.size() * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
        return false;
    }
    std::vector<std::int8_t> out(bw * bh, 0);
    const QuantCalibration cal{calibrate_quant(distance)};
    const float qgsf{static_cast<float>(cal.raw_quant_field) * cal.global_scale_float};
    for (std::size_t ry{0}; ry < (bh + 3) / 4; ++ry) {
        for (std::size_t rx{0}; rx < (bw + 3) / 4; ++rx) {
            decide_region(plane.data(), width, bw, bh, rx * 4, ry * 4, qgsf, TRANSFORM_SELECT_LAMBDA, out.data());
        }
    }
    return cudaMemcpy(acs, out.data(), out.size(), cudaMemcpyHostToDevice) == cudaSuccess;
}

}  // namespace cujpegxl

extern "C" {

// All addresses are device memory; each call returns 1 on success.
int refgpu_nv12_to_xyb(std::uintptr_t luma, std::size_t luma_pitch, std::uintptr_t chroma,
                       std::size_t chroma_pitch, std::size_t width, std::size_t height, std::uintptr_t xyb) {
    return cujpegxl::nv12_to_xyb(reinterpret_cast<const std::uint8_t*>(luma), luma_pitch,
                                 reinterpret_cast<const std::uint8_t*>(chroma), chroma_pitch, width, height,
                                 reinterpret_cast<float*>(xyb))
               ? 1
               : 0;
}

int refgpu_encode_frontend(std::uintptr_t luma, std::size_t luma_pitch, std::uintptr_t chroma,
                           std::size_t chroma_pitch, std::size_t width, std::size_t height, float distance,
                           std::uintptr_t quant_field) {
    return cujpegxl::encode_frontend(reinterpret_cast<const std::uint8_t*>(luma), luma_pitch,
                                     reinterpret_cast<const std::uint8_t*>(chroma), chroma_pitch, width, height,
                                     distance, reinterpret_cast<std::int32_t*>(quant_field))
               ? 1
               : 0;
}

// given_acs: device decisions to use instead of the reference's selection
// (0 = the reference's host-twin selection on its own sharpened Y plane).
int refgpu_frontend_transform(std::uintptr_t luma, std::size_t luma_pitch, std::uintptr_t chroma,
                              std::size_t chroma_pitch, std::size_t width, std::size_t height, float distance,
                              std::uintptr_t coeffs, std::uintptr_t acs, std::uintptr_t given_acs) {
    g_given_acs = reinterpret_cast<const std::int8_t*>(given_acs);
    const bool ok{cujpegxl::frontend_transform(reinterpret_cast<const std::uint8_t*>(luma), luma_pitch,
                                               reinterpret_cast<const std::uint8_t*>(chroma), chroma_pitch, width,
                                               height, distance, reinterpret_cast<__half*>(coeffs),
                                               reinterpret_cast<std::int8_t*>(acs))};
    g_given_acs = nullptr;
    return ok ? 1 : 0;
}

int refgpu_variable_forward_dct(std::uintptr_t planes, std::size_t width, std::size_t height, std::uintptr_t acs,
                                std::uintptr_t coeffs) {
    return cujpegxl::variable_forward_dct(reinterpret_cast<const float*>(planes), width, height,
                                          reinterpret_cast<const std::int8_t*>(acs),
                                          reinterpret_cast<__half*>(coeffs))
               ? 1
               : 0;
}

}  // extern "C"
