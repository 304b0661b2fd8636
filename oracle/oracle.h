/* CPU restatement of the reference encoder's path (test infrastructure only:
 * the checker for the CUDA path and the timed CPU baseline; nothing in the
 * product links or calls it). See frontend_oracle.c and bitstream_oracle.c. */
#ifndef CUJPEGXL_B200_ORACLE_H_
#define CUJPEGXL_B200_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    const uint8_t* luma;
    const uint8_t* chroma;
    size_t luma_pitch;
    size_t chroma_pitch;
    int width;
    int height;
} OracleFrame;

typedef struct {
    uint32_t global_scale, quant_dc, raw_quant_field;
    float gsf, inv_global_scale, qgsf_select, dc_scale;
    float mul_pb, add_pb;
    float km[4];
} OracleScalars;

typedef struct {
    int16_t* ac;     /* [3][B*64] */
    int32_t* dc;     /* [3][B] */
    int8_t* acs;     /* [B] */
    int32_t* qf;     /* [B] */
    int8_t* ytox;    /* [T] */
    int8_t* ytob;    /* [T] */
    uint8_t* nzn;    /* [3][B] */
    uint16_t* nzc;   /* [3][B] */
    float* dbg_xyb;  /* optional [3][H][W] */
    float* dbg_sharp;
    uint16_t* dbg_coeff;
} OracleOutputs;

void oracle_scalars(float distance, OracleScalars* s);
int oracle_frontend(const OracleFrame* in, float distance, const OracleOutputs* out, int threads);

/* Entropy coding and assembly from the frontend's planes into a full .jxl
 * file (container + codestream). Returns the file size, or 0 on error; writes
 * min(size, cap) bytes to `out`. */
size_t oracle_assemble(int width, int height, const int16_t* ac, const int32_t* dc,
                       const int8_t* acs, const int32_t* qf, const int8_t* ytox,
                       const int8_t* ytob, uint32_t global_scale, uint32_t quant_dc,
                       uint8_t* out, size_t cap);

/* Whole path: NV12 -> .jxl bytes. */
size_t oracle_encode(const OracleFrame* in, float distance, uint8_t* out, size_t cap, int threads);

/* Pieces exposed for tests. */
float oracle_log2(float x);
float oracle_exp2(float x);
float oracle_exp(float x);
float oracle_cbrt(float x);
float oracle_pow24(float x);
uint16_t oracle_f2h(float f);
float oracle_h2f(uint16_t h);
void oracle_xyb_pixel(const OracleFrame* in, int gx, int gy, float* out3);
float oracle_ratio_gamma(float v, int invert);
float oracle_masking_sqrt(float v);
float oracle_compute_mask(float v);
void oracle_gaborish_weights(float* out6);
float oracle_sel_cost(const float* y, int stride, int n, float qgsf);
void oracle_select_plane(const float* y, int width, int height, float distance, int8_t* acs);
void oracle_dc_from_llf(int m, const float* llf, float* dc);
void oracle_cfl_maps(float sxy, float syy, float sby, int* mx, int* mb);
size_t oracle_huffman(const uint32_t* hist, size_t len, uint8_t* depth, uint16_t* bits,
                      uint8_t* out, size_t cap);

#ifdef __cplusplus
}
#endif

#endif
