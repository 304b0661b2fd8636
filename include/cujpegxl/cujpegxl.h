/* cujpegxl drop-in C ABI, B200 implementation.
 *
 * This header declares the same nine entry points, enums and structs as the
 * reference library's public header (include/cujpegxl/cujpegxl.h:24-82 in
 * m-pilia/cujpegxl), with identical names, values, field order and types, so a
 * program compiled against the reference header links and runs against
 * libcujpegxl.so.1 built from this repository without recompilation.
 *
 * The header is plain C and pulls in no CUDA header: device memory is handed
 * over as integer addresses. */

#ifndef CUJPEGXL_CUJPEGXL_H_
#define CUJPEGXL_CUJPEGXL_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Matches the reference's CUJPEGXL_API_VERSION (cujpegxl.h:24). */
#define CUJPEGXL_API_VERSION 3u

/* Status codes; numeric values are part of the ABI (reference cujpegxl.h:26-34). */
typedef enum cujpegxl_status {
    CUJPEGXL_OK = 0,
    CUJPEGXL_NOT_IMPLEMENTED = 1,
    CUJPEGXL_INVALID_ARGUMENT = 2,
    CUJPEGXL_UNSUPPORTED_RESOLUTION = 3,
    CUJPEGXL_NO_DEVICE = 4,
    CUJPEGXL_INTERNAL_ERROR = 5,
    CUJPEGXL_BUFFER_TOO_SMALL = 6
} cujpegxl_status;

/* Backend label reported by cujpegxl_query_backend (reference cujpegxl.h:36-40). */
typedef enum cujpegxl_backend {
    CUJPEGXL_BACKEND_UNKNOWN = 0,
    CUJPEGXL_BACKEND_FP32_SIMT = 1,
    CUJPEGXL_BACKEND_FP16_TENSOR = 2
} cujpegxl_backend;

/* Opaque encoder handle. */
typedef struct cujpegxl_encoder cujpegxl_encoder;

/* Frame geometry, Butteraugli-style distance and CUDA device ordinal
 * (reference cujpegxl.h:44-49). */
typedef struct cujpegxl_config {
    uint32_t width;
    uint32_t height;
    float distance;
    int32_t device_ordinal;
} cujpegxl_config;

/* One NV12 frame (BT.709 full range, 8-bit 4:2:0) resident in device memory:
 * `luma` is width x height bytes with row pitch `luma_pitch`; `chroma` is the
 * interleaved Cb/Cr plane, width bytes per row over height/2 rows, with row
 * pitch `chroma_pitch` (reference cujpegxl.h:51-58). */
typedef struct cujpegxl_nv12_input {
    uintptr_t luma;
    uintptr_t chroma;
    size_t luma_pitch;
    size_t chroma_pitch;
} cujpegxl_nv12_input;

/* Host output buffer: `data` with `capacity` bytes; `size` receives the
 * file length, or the required length on CUJPEGXL_BUFFER_TOO_SMALL
 * (reference cujpegxl.h:60-64). */
typedef struct cujpegxl_output {
    uint8_t* data;
    size_t size;
    size_t capacity;
} cujpegxl_output;

uint32_t cujpegxl_api_version(void);
const char* cujpegxl_status_string(cujpegxl_status status);
const char* cujpegxl_backend_string(cujpegxl_backend backend);

cujpegxl_status cujpegxl_query_backend(int32_t device_ordinal, cujpegxl_backend* out_backend);

/* Upper bound on the encoded file size for `config`, for sizing the output
 * buffer before an encode. */
cujpegxl_status cujpegxl_max_output_size(const cujpegxl_config* config, size_t* out_bytes);

cujpegxl_status cujpegxl_encoder_create(const cujpegxl_config* config,
                                        cujpegxl_encoder** out_encoder);
cujpegxl_status cujpegxl_encoder_configure(cujpegxl_encoder* encoder,
                                           const cujpegxl_config* config);
cujpegxl_status cujpegxl_encoder_encode(cujpegxl_encoder* encoder, const cujpegxl_nv12_input* input,
                                        cujpegxl_output* output);
void cujpegxl_encoder_destroy(cujpegxl_encoder* encoder);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* CUJPEGXL_CUJPEGXL_H_ */
