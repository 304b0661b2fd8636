// C interface of the host subset decoder (libjxlsubset.so): the JPEG XL subset
// this encoder writes, decoded to XYB and sRGB planes for decodability checks
// and PSNR measurement. Not part of the drop-in ABI.
#pragma once

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Decodes a .jxl file (container or bare codestream). On success returns 0,
 * sets *width and *height and, when the frame fits in `capacity_pixels`, fills
 * xyb[3][H][W] and srgb[3][H][W] (either may be NULL; sRGB in [0, 1]). Returns
 * 2 when the frame is larger than capacity_pixels (sizes still set) and 1 when
 * the file is malformed or outside the subset, with a message in `error`. */
int jxlsubset_decode(const uint8_t* data, size_t size, uint32_t* width, uint32_t* height, float* xyb,
                     float* srgb, size_t capacity_pixels, char* error, size_t error_size);

/* Parses a file into its quantised planes (layouts of cujpegxl_b200_planes:
 * ac [3][B*64] covered-block slots in planes X, Y, B; dc [3][B]; acs [B]; qf
 * [B] at first blocks, 0 elsewhere; ytox/ytob [T]) and the quantiser state.
 * Any pointer may be NULL. Returns 0, or 2 when the frame has more than
 * capacity_blocks blocks (sizes still set), or 1 with a message. */
int jxlsubset_decode_planes(const uint8_t* data, size_t size, uint32_t* width, uint32_t* height, int16_t* ac,
                            int32_t* dc, int8_t* acs, int32_t* qf, int8_t* ytox, int8_t* ytob,
                            uint32_t* global_scale, uint32_t* quant_dc, size_t capacity_blocks, char* error,
                            size_t error_size);

#ifdef __cplusplus
}
#endif
