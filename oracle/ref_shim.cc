// C entry points over the reference's own host-compilable code, for use as a
// checker only (test infrastructure; never linked into the product).
//
// build_ref.py compiles this file together with the reference sources where
// they lie (src/bitstream/*.cc, tools/bitstream/*.cc, src/coeff_order.cc,
// src/vardct_layout.cc) into oracle/_ref/libjxlref.so. The reference headers
// that carry __device__ helpers (src/xyb_impl.cuh, src/adaptive_quant_impl.cuh)
// compile as plain host code with g++, so their formulas run here with the
// host libm. Every function below either forwards to a reference function or
// drives one with a loop that restates the caller in the reference (cited).

#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>

#include "src/ac_context.h"
#include "src/adaptive_quant_impl.cuh"
#include "src/bitstream/bit_writer.h"
#include "src/bitstream/container.h"
#include "src/bitstream/field_coder.h"
#include "src/bitstream/frame_assembly.h"
#include "src/bitstream/prefix_code.h"
#include "src/cfl.h"
#include "src/coeff_order.h"
#include "src/dc_predict.h"
#include "src/gaborish.h"
#include "src/quant_calibration.h"
#include "src/quant_weights_dct16.h"
#include "src/quant_weights_dct32.h"
#include "src/quant_weights_dct8.h"
#include "src/transform_select_impl.cuh"
#include "src/vardct_layout.h"
#include "src/xyb_impl.cuh"
#include "tools/bitstream/modular.h"
#include "tools/bitstream/vardct_frame.h"

using namespace cujpegxl;
using namespace cujpegxl::bitstream;

namespace {

// Builds a FrameCoefficients from flat arrays (channel-major X, Y, B).
FrameCoefficients make_fc(std::size_t w, std::size_t h, const std::int32_t* ac,
                          const std::int32_t* dc, const std::int8_t* acs, const std::int8_t* ytox,
                          const std::int8_t* ytob, std::uint32_t gs, std::uint32_t qdc,
                          std::uint32_t rqf) {
    FrameCoefficients fc{};
    fc.width = w;
    fc.height = h;
    fc.global_scale = gs;
    fc.quant_dc = qdc;
    fc.raw_quant_field = rqf;
    const std::size_t blocks{(w / 8) * (h / 8)};
    for (int c{0}; c < 3; ++c) {
        fc.ac[c].assign(ac + c * blocks * 64, ac + (c + 1) * blocks * 64);
        fc.dc[c].assign(dc + c * blocks, dc + (c + 1) * blocks);
    }
    if (acs != nullptr) {
        fc.acs.assign(acs, acs + blocks);
    }
    if (ytox != nullptr) {
        const std::size_t cm{((w / 8 + 7) / 8) * ((h / 8 + 7) / 8)};
        fc.ytox_map.assign(ytox, ytox + cm);
        fc.ytob_map.assign(ytob, ytob + cm);
    }
    return fc;
}

std::size_t copy_out(const std::vector<std::uint8_t>& v, std::uint8_t* out, std::size_t cap) {
    if (out != nullptr) {
        std::memcpy(out, v.data(), v.size() < cap ? v.size() : cap);
    }
    return v.size();
}

std::size_t ceil_log2_nonzero(std::size_t x) {
    std::size_t bits{0};
    for (std::size_t v{x > 1 ? x - 1 : 0}; v != 0; v >>= 1) {
        ++bits;
    }
    return bits;
}

}  // namespace

extern "C" {

// --- constants and scalar formulas -------------------------------------------

// src/xyb_impl.cuh:49-70 evaluated with the host libm.
void ref_xyb_pixel(float yv, float cb, float cr, float* x, float* y, float* b) {
    nv12_pixel_to_xyb(yv, cb, cr, *x, *y, *b);
}

// src/xyb_impl.cuh:17-35 constants, in order M00..M22, bias, 4 chroma factors, centre.
void ref_xyb_constants(float* out) {
    const float v[]{M00, M01, M02, M10, M11, M12, M20, M21, M22, OPSIN_BIAS,
                    CR_TO_R, CB_TO_G, CR_TO_G, CB_TO_B, CHROMA_CENTER};
    std::memcpy(out, v, sizeof(v));
}

// src/gaborish.h:24-29 weights WC, WR, WR2, WD, WL, WD2.
void ref_gaborish_weights(float* out) {
    const float v[]{GAB_WC, GAB_WR, GAB_WR2, GAB_WD, GAB_WL, GAB_WD2};
    std::memcpy(out, v, sizeof(v));
}

// src/adaptive_quant_impl.cuh:30-70.
float ref_ratio_cbrt_gamma(float v, int invert) {
    return invert ? ratio_cbrt_gamma<true>(v) : ratio_cbrt_gamma<false>(v);
}
float ref_masking_sqrt(float v) { return masking_sqrt(v); }
float ref_compute_mask(float v) { return compute_mask(v); }

// src/quant_calibration.h:49-88.
void ref_calibrate(float distance, std::uint32_t* ints, float* floats) {
    const QuantCalibration c{calibrate_quant(distance)};
    ints[0] = c.global_scale;
    ints[1] = c.quant_dc;
    ints[2] = c.raw_quant_field;
    floats[0] = c.global_scale_float;
    floats[1] = c.inv_global_scale;
}

// src/coeff_order.cc:10-43.
void ref_natural_order(int n, std::uint32_t* out) {
    const std::vector<std::uint32_t> o{natural_coeff_order(static_cast<std::size_t>(n))};
    std::memcpy(out, o.data(), o.size() * sizeof(std::uint32_t));
}

// src/quant_weights_dct{8,16,32}.h tables for channel c (0=X, 1=Y, 2=B).
void ref_dequant_weights(int n, int c, float* out) {
    if (n == 8) {
        std::memcpy(out, DCT8_DEQUANT_WEIGHTS[c], 64 * sizeof(float));
    } else if (n == 16) {
        std::memcpy(out, DCT16_DEQUANT_WEIGHTS[c], 256 * sizeof(float));
    } else {
        std::memcpy(out, DCT32_DEQUANT_WEIGHTS[c], 1024 * sizeof(float));
    }
}

// src/ac_context.h:55-148.
int ref_ac_cluster(std::uint32_t ctx) { return ac_cluster(ctx); }
int ref_ac_block_context(int c, int ord) { return ac_block_context(c, ord); }
std::uint32_t ref_ac_nonzero_context(std::uint32_t pred, int block_ctx) {
    return ac_nonzero_context(pred, block_ctx);
}
std::uint32_t ref_ac_zero_density_context(std::uint32_t left, std::uint32_t k, std::uint32_t cb,
                                          std::uint32_t l2, std::uint32_t prev) {
    return ac_zero_density_context(left, k, cb, l2, prev);
}

// src/dc_predict.h:33-50.
std::int32_t ref_gradient_predict(int hl, int ht, std::int32_t w, std::int32_t n, std::int32_t nw) {
    return gradient_predict(hl != 0, ht != 0, w, n, nw);
}

// --- stage twins --------------------------------------------------------------

// Transform selection over a whole sharpened-Y plane: the loop of
// select_transforms_host (src/transform_select.cu:286-303) around the
// reference's decide_region (src/transform_select_impl.cuh:130-201).
void ref_select_transforms(const float* y, std::size_t width, std::size_t height, float distance,
                           std::int8_t* acs) {
    const std::size_t bw{width / 8};
    const std::size_t bh{height / 8};
    const QuantCalibration cal{calibrate_quant(distance)};
    const float qgsf{static_cast<float>(cal.raw_quant_field) * cal.global_scale_float};
    for (std::size_t ry{0}; ry < (bh + 3) / 4; ++ry) {
        for (std::size_t rx{0}; rx < (bw + 3) / 4; ++rx) {
            decide_region(y, width, bw, bh, rx * 4, ry * 4, qgsf, TRANSFORM_SELECT_LAMBDA, acs);
        }
    }
}

// One block cost (src/transform_select_impl.cuh:49-115).
float ref_block_ac_cost(const float* y, std::size_t width, std::size_t px0, std::size_t py0, int n,
                        float qgsf) {
    return block_ac_cost(y, width, px0, py0, n, qgsf, TRANSFORM_SELECT_LAMBDA);
}

// src/vardct_layout.h:88-111 on a compacted m*m corner.
void ref_dc_from_llf(int m, const float* llf, float* dc) {
    dc_from_llf_strided(static_cast<std::size_t>(m), llf, static_cast<std::size_t>(m), dc);
}

// src/cfl.h:71-77.
void ref_cfl_maps_from_sums(double sxy, double syy, double sby, int* mx, int* mb) {
    cfl_maps_from_sums(sxy, syy, sby, mx, mb);
}

// --- bitstream ----------------------------------------------------------------

// src/bitstream/prefix_code.cc:387-426. Returns the header length in bits.
std::size_t ref_huffman(const std::uint32_t* hist, std::size_t len, std::uint8_t* depth,
                        std::uint16_t* bits, std::uint8_t* out, std::size_t cap) {
    BitWriter w{};
    build_and_store_huffman_tree(hist, len, depth, bits, w);
    copy_out(w.bytes(), out, cap);
    return w.bits_written();
}

// tools/bitstream/vardct_frame.cc:563-607: pooled clustered histogram, codes and
// per-group byte streams. Streams are concatenated into `out`; `sizes` gets
// num_ac_groups entries. Returns the total stream bytes.
std::size_t ref_ac_encode(std::size_t w, std::size_t h, const std::int32_t* ac,
                          const std::int8_t* acs, std::uint32_t* hist, std::uint8_t* depth,
                          std::uint16_t* bits, std::uint8_t* out, std::size_t cap,
                          std::uint32_t* sizes) {
    const std::size_t blocks{(w / 8) * (h / 8)};
    std::vector<std::int32_t> dc(3 * blocks, 0);
    const FrameCoefficients fc{make_fc(w, h, ac, dc.data(), acs, nullptr, nullptr, 1, 1, 1)};
    const AcReference r{reference_ac_encode(fc)};
    std::memcpy(hist, r.histogram.data(), r.histogram.size() * 4);
    std::memcpy(depth, r.depth.data(), r.depth.size());
    std::memcpy(bits, r.bits.data(), r.bits.size() * 2);
    std::vector<std::uint8_t> all{};
    for (std::size_t g{0}; g < r.group_streams.size(); ++g) {
        sizes[g] = static_cast<std::uint32_t>(r.group_streams[g].size());
        all.insert(all.end(), r.group_streams[g].begin(), r.group_streams[g].end());
    }
    return copy_out(all, out, cap);
}

// tools/bitstream/vardct_frame.cc:609-664 with a uniform quant field: DcGroup
// sections concatenated into `out`, per-group sizes, DC and AcMetadata histograms.
std::size_t ref_dc_encode(std::size_t w, std::size_t h, const std::int32_t* dc,
                          const std::int8_t* acs, const std::int8_t* ytox, const std::int8_t* ytob,
                          std::uint32_t rqf, std::uint8_t* out, std::size_t cap,
                          std::uint32_t* sizes, std::uint32_t* dc_hist, std::uint32_t* am_hist) {
    const std::size_t blocks{(w / 8) * (h / 8)};
    std::vector<std::int32_t> ac(3 * blocks * 64, 0);
    const FrameCoefficients fc{make_fc(w, h, ac.data(), dc, acs, ytox, ytob, 1, 1, rqf)};
    const DcReference r{reference_dc_encode(fc)};
    std::vector<std::uint8_t> all{};
    for (std::size_t g{0}; g < r.groups.size(); ++g) {
        const DcGroupReference& gr{r.groups[g]};
        sizes[g] = static_cast<std::uint32_t>(gr.section.size());
        all.insert(all.end(), gr.section.begin(), gr.section.end());
        for (std::size_t s{0}; s < 256; ++s) {
            dc_hist[g * 256 + s] = s < gr.dc_histogram.size() ? gr.dc_histogram[s] : 0;
            am_hist[g * 256 + s] = s < gr.acmeta_histogram.size() ? gr.acmeta_histogram[s] : 0;
        }
    }
    return copy_out(all, out, cap);
}

// tools/bitstream/vardct_frame.cc:666-677 (clustered AC): the bare codestream
// for a frame with a uniform quant field.
std::size_t ref_write_codestream(std::size_t w, std::size_t h, const std::int32_t* ac,
                                 const std::int32_t* dc, const std::int8_t* acs,
                                 const std::int8_t* ytox, const std::int8_t* ytob,
                                 std::uint32_t gs, std::uint32_t qdc, std::uint32_t rqf,
                                 std::uint8_t* out, std::size_t cap) {
    const FrameCoefficients fc{make_fc(w, h, ac, dc, acs, ytox, ytob, gs, qdc, rqf)};
    return copy_out(write_vardct_codestream(fc, true), out, cap);
}

// The production assembly of src/frame_encoder.cu:88-292 from quantised planes
// with a per-block quant field, built from the reference's host pieces:
// reference_ac_encode + build_ac_global (AC groups, AcGlobal), build_dc_global,
// per DcGroup the modular images of tools/bitstream/modular.cc with the
// AcMetadata QF row taken from `qf` (src/entropy.cu:255-274), then
// build_codestream_head and container_framing. Returns the file size.
std::size_t ref_encode_frame(std::size_t w, std::size_t h, const std::int32_t* ac,
                             const std::int32_t* dc, const std::int8_t* acs,
                             const std::int8_t* ytox, const std::int8_t* ytob,
                             const std::int32_t* qf, std::uint32_t gs, std::uint32_t qdc,
                             std::uint8_t* out, std::size_t cap) {
    const std::size_t bw{w / 8};
    const std::size_t bh{h / 8};
    const FrameCoefficients fc{make_fc(w, h, ac, dc, acs, ytox, ytob, gs, qdc, 1)};
    const std::size_t num_ac{ac_group_count(w, h)};
    const std::size_t xdg{(bw + 255) / 256};
    const std::size_t num_dc{dc_group_count(w, h)};
    const std::size_t cmw{(bw + 7) / 8};

    const AcReference acr{reference_ac_encode(fc)};
    const AcGlobalResult acg{build_ac_global(acr.histogram.data(), num_ac)};
    const std::vector<std::uint8_t> dcg{build_dc_global(QuantParams{gs, qdc})};

    std::vector<std::vector<std::uint8_t>> dc_sections(num_dc);
    for (std::size_t g{0}; g < num_dc; ++g) {
        const std::size_t bx0{(g % xdg) * 256};
        const std::size_t by0{(g / xdg) * 256};
        const std::size_t dgw{std::min<std::size_t>(256, bw - bx0)};
        const std::size_t dgh{std::min<std::size_t>(256, bh - by0)};
        std::vector<ModularChannel> dch{};
        const int phys[3]{1, 0, 2};
        for (int p{0}; p < 3; ++p) {
            ModularChannel ch{dgw, dgh, std::vector<std::int32_t>(dgw * dgh)};
            for (std::size_t y{0}; y < dgh; ++y) {
                for (std::size_t x{0}; x < dgw; ++x) {
                    ch.pixels[y * dgw + x] = dc[phys[p] * bw * bh + (by0 + y) * bw + bx0 + x];
                }
            }
            dch.push_back(std::move(ch));
        }
        const std::size_t cw{(dgw + 7) / 8};
        const std::size_t chh{(dgh + 7) / 8};
        ModularChannel tx{cw, chh, std::vector<std::int32_t>(cw * chh, 0)};
        ModularChannel tb{cw, chh, std::vector<std::int32_t>(cw * chh, 0)};
        for (std::size_t y{0}; y < chh; ++y) {
            for (std::size_t x{0}; x < cw; ++x) {
                const std::size_t t{(by0 / 8 + y) * cmw + bx0 / 8 + x};
                tx.pixels[y * cw + x] = ytox == nullptr ? 0 : ytox[t];
                tb.pixels[y * cw + x] = ytob == nullptr ? 0 : ytob[t];
            }
        }
        std::vector<std::int32_t> row0{};
        std::vector<std::int32_t> row1{};
        for (std::size_t y{0}; y < dgh; ++y) {
            for (std::size_t x{0}; x < dgw; ++x) {
                const std::size_t blk{(by0 + y) * bw + bx0 + x};
                const int side{acs == nullptr ? 8 : acs[blk]};
                if (side == ACS_COVERED) {
                    continue;
                }
                row0.push_back(side == 16 ? 4 : (side == 32 ? 5 : 0));
                row1.push_back(qf[blk] - 1);
            }
        }
        const std::size_t count{row0.size()};
        ModularChannel aq{count, 2, row0};
        aq.pixels.insert(aq.pixels.end(), row1.begin(), row1.end());
        ModularChannel epf{dgw, dgh, std::vector<std::int32_t>(dgw * dgh, 0)};
        std::vector<ModularChannel> meta{};
        meta.push_back(std::move(tx));
        meta.push_back(std::move(tb));
        meta.push_back(std::move(aq));
        meta.push_back(std::move(epf));

        BitWriter bw_{};
        write_bits(bw_, 2, 0);
        write_modular_image(bw_, dch, DC_PREDICTOR_GRADIENT);
        write_bits(bw_, ceil_log2_nonzero(dgw * dgh), static_cast<std::uint32_t>(count - 1));
        write_modular_image(bw_, meta);
        bw_.zero_pad_to_byte();
        dc_sections[g] = bw_.bytes();
    }

    std::vector<std::uint32_t> sizes{};
    sizes.push_back(static_cast<std::uint32_t>(dcg.size()));
    for (const auto& s : dc_sections) {
        sizes.push_back(static_cast<std::uint32_t>(s.size()));
    }
    sizes.push_back(static_cast<std::uint32_t>(acg.section.size()));
    for (const auto& s : acr.group_streams) {
        sizes.push_back(static_cast<std::uint32_t>(s.size()));
    }
    const std::vector<std::uint8_t> head{build_codestream_head(
        static_cast<std::uint32_t>(w), static_cast<std::uint32_t>(h), sizes)};
    std::vector<std::uint8_t> body{dcg};
    for (const auto& s : dc_sections) {
        body.insert(body.end(), s.begin(), s.end());
    }
    body.insert(body.end(), acg.section.begin(), acg.section.end());
    for (const auto& s : acr.group_streams) {
        body.insert(body.end(), s.begin(), s.end());
    }
    std::vector<std::uint8_t> file{container_framing(head.size() + body.size())};
    file.insert(file.end(), head.begin(), head.end());
    file.insert(file.end(), body.begin(), body.end());
    return copy_out(file, out, cap);
}

}  // extern "C"
