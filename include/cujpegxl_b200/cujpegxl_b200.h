/* Additional entry points of libcujpegxl.so.1 beyond the reference's nine.
 *
 * None of these replaces a reference entry point; they expose the encoder's
 * stages and device buffers for parity testing, benchmarking and callers that
 * keep frames on the device. They use the same opaque encoder handle and
 * status codes as include/cujpegxl/cujpegxl.h. Plain C, no CUDA types. */

#ifndef CUJPEGXL_B200_H_
#define CUJPEGXL_B200_H_

#include <stddef.h>
#include <stdint.h>

#include "cujpegxl/cujpegxl.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Host views of the frontend's planes for one frame (B = (W/8)*(H/8)
 * blocks, T = ceil(W/64)*ceil(H/64) colour tiles). Any pointer may be NULL.
 * The optional float/FP16 stage dumps are filled only while debug dumps are
 * enabled on the encoder. */
typedef struct cujpegxl_b200_planes {
    int16_t* ac;      /* [3][B*64] quantised AC, covered-block layout, X,Y,B */
    int32_t* dc;      /* [3][B] quantised DC */
    int8_t* acs;      /* [B] transform side at first-blocks, 0 at covered blocks */
    int32_t* qf;      /* [B] adaptive quant field */
    int8_t* ytox;     /* [T] */
    int8_t* ytob;     /* [T] */
    float* xyb;       /* [3][H][W] XYB before sharpening */
    float* sharp;     /* [3][H][W] XYB after inverse gaborish */
    uint16_t* coeff;  /* [3][B*64] FP16 DCT coefficients (bit patterns) */
    float* cost;      /* [3][B] RD costs of the transform selection: DCT8 at every
                       * block, DCT16 at the first block of every 16x16 quad and
                       * DCT32 at the first block of every 32x32 region (0
                       * elsewhere); only where the RD search ran */
} cujpegxl_b200_planes;

/* cujpegxl_encoder_create with options. CUJPEGXL_B200_ENCODER_SINGLE_GROUP
 * also accepts frames of a single 256x256 AC group (width and height at most
 * 256 pixels), which the reference rejects with UNSUPPORTED_RESOLUTION
 * (src/cujpegxl.cc:36-48): their DcGlobal, DcGroup, AcGlobal and AcGroup are
 * written as one combined section with a single TOC entry, concatenated bit
 * by bit and padded once at the end, as the reference's own codestream tool
 * writes such frames (tools/bitstream/vardct_frame.cc:414-449). The option
 * stays with the encoder through cujpegxl_encoder_configure. */
#define CUJPEGXL_B200_ENCODER_SINGLE_GROUP 1u
cujpegxl_status cujpegxl_b200_encoder_create_ex(const cujpegxl_config* config, uint32_t flags,
                                                cujpegxl_encoder** out_encoder);

/* cujpegxl_max_output_size with the same options. */
cujpegxl_status cujpegxl_b200_max_output_size_ex(const cujpegxl_config* config, uint32_t flags,
                                                 size_t* out_bytes);

/* Enables (non-zero) or disables the float/FP16 stage dumps of the frontend.
 * Replaces no reference interface. */
cujpegxl_status cujpegxl_b200_encoder_set_debug(cujpegxl_encoder* encoder, int32_t enable);

/* Copies the planes of the most recent encode to host memory. Replaces no
 * reference interface. */
cujpegxl_status cujpegxl_b200_encoder_read_planes(cujpegxl_encoder* encoder,
                                                  const cujpegxl_b200_planes* host);

/* Entropy coding and assembly only: uploads quantised planes (ac, dc, acs,
 * qf, ytox, ytob must be non-NULL) and writes the .jxl file, exactly as
 * cujpegxl_encoder_encode does after its frontend. The stage the reference
 * runs as encode_frame (src/frame_encoder.h:49-53). */
cujpegxl_status cujpegxl_b200_encode_planes(cujpegxl_encoder* encoder,
                                            const cujpegxl_b200_planes* host,
                                            uint32_t global_scale, uint32_t quant_dc,
                                            cujpegxl_output* output);

/* Host NV12 in (width*height*3/2 bytes, pitch = width), .jxl out: uploads
 * through a pinned staging buffer, then encodes. The path of the reference's
 * Python binding (python/nv12_host_encode.cu:10-40). */
cujpegxl_status cujpegxl_b200_encode_host(cujpegxl_encoder* encoder, const uint8_t* nv12,
                                          size_t nv12_size, cujpegxl_output* output);

/* Enqueues one encode on the encoder's stream and returns without waiting;
 * the file stays in device memory. cujpegxl_b200_encoder_result waits and
 * reports its size and device address. For callers that keep bytes on the
 * device and for throughput measurement. Replaces no reference interface. */
cujpegxl_status cujpegxl_b200_encoder_enqueue(cujpegxl_encoder* encoder,
                                              const cujpegxl_nv12_input* input);
cujpegxl_status cujpegxl_b200_encoder_result(cujpegxl_encoder* encoder, size_t* out_size,
                                             uintptr_t* out_device_bytes);

/* Enqueues, behind the encoder's last enqueued encode, the copy of its file
 * into page-locked host memory (cudaHostAlloc, cudaHostRegister or torch's
 * pin_memory; other memory gives CUJPEGXL_INVALID_ARGUMENT) and returns
 * without waiting. The copy is made by a kernel that reads the file's size on
 * the device, so no host round trip separates encode and copy. When the
 * encoder's stream has reached it, host_words[0] holds the file's size and
 * host_words[1] a status: 0 = copied into host_dst, 1 = larger than
 * `capacity` (nothing copied), 2 = the encode failed. host_words is 8-byte
 * aligned page-locked memory of two words. cujpegxl_encoder_encode takes the
 * same path by itself when its output buffer is page-locked. Replaces no
 * reference interface. */
cujpegxl_status cujpegxl_b200_encoder_enqueue_readback(cujpegxl_encoder* encoder, uint8_t* host_dst,
                                                      size_t capacity, uint64_t* host_words);

/* As cujpegxl_b200_encoder_enqueue, restricted to the stages in `stages`
 * (bit 0: the fused frontend kernel, bit 1: entropy coding and assembly).
 * For timing one stage in isolation. Replaces no reference interface. */
#define CUJPEGXL_B200_STAGE_FRONTEND 1u
#define CUJPEGXL_B200_STAGE_ENTROPY 2u
cujpegxl_status cujpegxl_b200_encoder_enqueue_stages(cujpegxl_encoder* encoder,
                                                     const cujpegxl_nv12_input* input,
                                                     uint32_t stages);

/* The encoder's CUDA stream (a cudaStream_t as an integer), for callers that
 * order their own work or timing events against it. */
cujpegxl_status cujpegxl_b200_encoder_stream(cujpegxl_encoder* encoder, uintptr_t* out_stream);

/* Device views of quantised planes (layouts as cujpegxl_b200_planes), as
 * integer device addresses. */
typedef struct cujpegxl_b200_device_planes {
    uintptr_t ac;     /* int16_t [3][B*64] */
    uintptr_t dc;     /* int32_t [3][B] */
    uintptr_t acs;    /* int8_t [B] */
    uintptr_t qf;     /* int32_t [B] */
    uintptr_t ytox;   /* int8_t [T] */
    uintptr_t ytob;   /* int8_t [T] */
} cujpegxl_b200_device_planes;

/* No counterpart in the reference. Entropy coding and assembly of one frame
 * from quantised planes already in device memory, producing the same file as
 * cujpegxl_b200_encode_planes, for callers that cannot allocate device memory
 * while they encode: a real-time loop where cudaMalloc would synchronise the
 * whole device and stall other streams, or an embedder whose device memory is
 * entirely reserved by its own pool allocator. It allocates nothing: the
 * caller passes the planes and a device output buffer (`out_capacity` bytes),
 * and every intermediate lives in one fixed 7 MiB array that each GPU loading
 * the library holds until the process exits.
 *  - Alignment: the AC plane and the output buffer 16-byte aligned, the DC
 *    and quant-field planes 4-byte aligned (every cudaMalloc'd buffer is);
 *    other addresses give CUJPEGXL_INVALID_ARGUMENT.
 *  - Frames above 4,194,304 pixels (width*height) are rejected with
 *    CUJPEGXL_UNSUPPORTED_RESOLUTION; other geometry rules are those of
 *    cujpegxl_encoder_create.
 *  - The first call on a device also looks up the array's device address and
 *    sets kernel attributes (host runtime calls that later calls skip).
 *  - Calls share the array: calls that overlap on the GPU (different streams
 *    or threads without ordering) race and corrupt each other's output.
 *  - Work is enqueued on `stream` (a cudaStream_t as an integer, 0 for the
 *    default stream); the call then synchronises `stream`, reads the result
 *    words back and sets *out_size to the file length, or to the required
 *    length with CUJPEGXL_BUFFER_TOO_SMALL. */
cujpegxl_status cujpegxl_b200_encode_planes_noalloc(const cujpegxl_b200_device_planes* planes,
                                                    uint32_t width, uint32_t height,
                                                    uint32_t global_scale, uint32_t quant_dc,
                                                    uint8_t* out_device, size_t out_capacity,
                                                    size_t* out_size, uintptr_t stream);

/* Number of kernels one encode launches. */
uint32_t cujpegxl_b200_kernels_per_encode(void);

/* Test hooks for the error paths of encoder creation (the reference has no
 * counterpart; its tests cover only argument errors). After
 * cujpegxl_b200_debug_fail_allocation(n) with n > 0, the n-th device arena,
 * pinned host buffer or CUDA stream that an encoder acquires from then on fails
 * as an out-of-memory would; n = 0 turns the injection off. The count of such
 * resources that encoders currently hold is
 * cujpegxl_b200_debug_live_allocations(): a failed cujpegxl_encoder_create
 * must leave it where it was. */
void cujpegxl_b200_debug_fail_allocation(uint32_t nth);
uint64_t cujpegxl_b200_debug_live_allocations(void);

/* Test hook: the device's prefix-code builder (the one every encode runs) on
 * one histogram of `length` symbols (1..256, host memory), for comparison with
 * the reference's build_and_store_huffman_tree (src/bitstream/prefix_code.cc):
 * depth[length], bits[length] (bit-reversed canonical codes) and the code's
 * header in header[header_cap >= 256], *header_bits its length in bits.
 * Synchronous; allocates a small device buffer. */
cujpegxl_status cujpegxl_b200_debug_prefix_code(int32_t device_ordinal, const uint32_t* hist, uint32_t length,
                                                uint8_t* depth, uint16_t* bits, uint8_t* header,
                                                size_t header_cap, uint32_t* header_bits);

/* Device memory the encoder holds for its current geometry (one arena, all of
 * it allocated at create/configure) and its pinned host staging buffer
 * (`pinned_host_bytes` may be NULL), for admission control by callers that
 * run many encoders. Replaces no reference interface. */
cujpegxl_status cujpegxl_b200_encoder_memory(cujpegxl_encoder* encoder, size_t* device_bytes,
                                             size_t* pinned_host_bytes);

/* ---- Batched encode: frames of different sizes in one CUDA graph launch ----
 * No reference counterpart (the reference encodes one frame per call). A batch
 * owns one encoder per frame (each frame may have its own width, height and
 * distance; all on one device). cujpegxl_b200_batch_encode enqueues the whole
 * batch as one graph launch whose work is batched across frames: one
 * persistent frontend launch takes the 64x64 tiles of all frames from one
 * work list, then each entropy pass runs once for all frames (frames in
 * groups of 64 per launch). The first encode times the candidate frontend
 * schedules (cujpegxl_b200_batch_schedule) and keeps the fastest, and later
 * batches of the same geometry mix reuse it (the environment variable
 * CUJPEGXL_B200_BATCH_TILES_PER_CTA, 1 or 2, restricts the candidates to
 * one CTA shape, read when a batch tunes); later encodes with the same
 * input addresses relaunch that graph, new addresses are recaptured and the
 * graph updated in place. The call is asynchronous:
 * cujpegxl_b200_batch_sync waits and reports every frame's size, after which
 * each file can be read on the device or copied to the host. */
typedef struct cujpegxl_b200_batch cujpegxl_b200_batch;

cujpegxl_status cujpegxl_b200_batch_create(const cujpegxl_config* frames, size_t count,
                                           cujpegxl_b200_batch** out_batch);

/* inputs[count]: device NV12 frames, the same rules as cujpegxl_encoder_encode. */
cujpegxl_status cujpegxl_b200_batch_encode(cujpegxl_b200_batch* batch, const cujpegxl_nv12_input* inputs);

/* Waits for the last batch_encode; sizes[count] (may be NULL) receives the
 * file sizes. CUJPEGXL_INTERNAL_ERROR if any frame failed. */
cujpegxl_status cujpegxl_b200_batch_sync(cujpegxl_b200_batch* batch, size_t* sizes);

/* After batch_sync: size and device address of frame `index`'s file. */
cujpegxl_status cujpegxl_b200_batch_frame(cujpegxl_b200_batch* batch, size_t index, size_t* size,
                                          uintptr_t* device_bytes);

/* After batch_sync: copies frame `index`'s file to host memory (BUFFER_TOO_SMALL
 * sets output->size to the required length). */
cujpegxl_status cujpegxl_b200_batch_copy(cujpegxl_b200_batch* batch, size_t index, cujpegxl_output* output);

/* The stream the batch's graph is launched on (to order or time caller work
 * against it). */
cujpegxl_status cujpegxl_b200_batch_stream(const cujpegxl_b200_batch* batch, uintptr_t* stream);

/* 1 once the batch's graph exists (its work runs on one stream), else 0. */
uint32_t cujpegxl_b200_batch_lanes(const cujpegxl_b200_batch* batch);

/* The frontend schedule the batch's autotuner chose on its first encode (or
 * took from an earlier batch of the same geometry mix): resident CTAs of the
 * persistent frontend launch, tiles per claim (per tile slot of a CTA), claims
 * from a counter (1) or round-robin (0), frames largest-first (1) or in the
 * given order (0), the measured time of one batch with it, and the tiles
 * each CTA runs at a time (2: one per half of a 512-thread CTA, claimed
 * together; 1: 256-thread CTAs). */
typedef struct cujpegxl_b200_batch_schedule_info {
    uint32_t frontend_ctas;
    uint32_t tiles_per_claim;
    uint32_t dynamic_claims;
    uint32_t largest_first;
    uint32_t from_cache;
    uint32_t candidates;
    float tuned_ms;
    uint32_t tiles_per_cta;
} cujpegxl_b200_batch_schedule_info;
cujpegxl_status cujpegxl_b200_batch_schedule(const cujpegxl_b200_batch* batch,
                                             cujpegxl_b200_batch_schedule_info* out);

void cujpegxl_b200_batch_destroy(cujpegxl_b200_batch* batch);

/* ---- Learned transform decisions ----
 * No reference counterpart. A 4-layer BF16 convolutional network over each
 * 32x32 region of XYB pixels predicts the region's DCT32/DCT16/DCT8 split and
 * the quant field of its 16 blocks. Regions whose softmax margin (top
 * probability minus the runner-up) is below a threshold keep the RD
 * heuristic, as do regions that are not a full 32x32 inside the image. The
 * decisions only steer the encoder: the stream stays conformant and its
 * entropy coding exact.
 *
 * Weights blob (little-endian): "JXBN", uint32 version 2, uint32 parameter
 * count, uint32 channels 32, classes 17, K1 80, K 288, float32 scale[4] and
 * shift[4] (input normalisation of X, Y, B and log2 distance), float32
 * parameters[count], then the SHA-256 of every preceding byte. */
typedef struct cujpegxl_b200_acsnet cujpegxl_b200_acsnet;

#define CUJPEGXL_B200_ACSNET_SPLIT 1u /* use the predicted transform split */
#define CUJPEGXL_B200_ACSNET_QF 2u    /* also use the predicted quant field */

/* Parameters of the network (the length of a blob's parameter array). */
uint32_t cujpegxl_b200_acsnet_param_count(void);

/* Checks a weights blob (layout, sizes and SHA-256) without a device:
 * CUJPEGXL_OK or CUJPEGXL_INVALID_ARGUMENT. */
cujpegxl_status cujpegxl_b200_acsnet_check_blob(const void* blob, size_t size);

/* Uploads a checked blob to `device_ordinal`. */
cujpegxl_status cujpegxl_b200_acsnet_create(const void* blob, size_t size, int32_t device_ordinal,
                                            cujpegxl_b200_acsnet** out_net);
void cujpegxl_b200_acsnet_destroy(cujpegxl_b200_acsnet* net);

/* Attaches `net` (NULL detaches) to an encoder on the same device. `flags` is
 * CUJPEGXL_B200_ACSNET_SPLIT, optionally with CUJPEGXL_B200_ACSNET_QF;
 * `margin` in [0, 1]. The network must outlive its use by the encoder. */
cujpegxl_status cujpegxl_b200_encoder_set_acsnet(cujpegxl_encoder* encoder, const cujpegxl_b200_acsnet* net,
                                                 float margin, uint32_t flags);

/* After an encode with a network attached: regions the network decided and
 * full 32x32 regions of the frame. Waits for the encoder's stream. */
cujpegxl_status cujpegxl_b200_encoder_acsnet_stats(cujpegxl_encoder* encoder, uint32_t* decided,
                                                   uint32_t* regions);

/* Training. All pointers in a batch are device addresses; sample i uses tile
 * tiles[tile_index[i]] ([3][34][34] float X, Y, B planes: the region and a
 * 1-pixel ring, clamped at the image border) at log2 distance
 * log2_distance[i], with labels label_class[i] (split class 0..16) and
 * label_qf[i][16] (log2 quant field of the blocks in raster order).
 * label_soft (may be NULL) replaces the one-hot target of the split by a
 * distribution [n][17]; label_class then only feeds the accuracy statistic. */
typedef struct cujpegxl_b200_acsnet_batch {
    const float* tiles;
    const int32_t* tile_index;
    const float* log2_distance;
    const int8_t* label_class;
    const float* label_qf;
    uint32_t n;
    const float* label_soft;
} cujpegxl_b200_acsnet_batch;

typedef struct cujpegxl_b200_acsnet_trainer cujpegxl_b200_acsnet_trainer;

/* params[param_count] and norm[8] (scale[4] then shift[4]) are host arrays.
 * Batches passed later hold at most max_batch samples. */
cujpegxl_status cujpegxl_b200_acsnet_trainer_create(const float* params, const float* norm, uint32_t max_batch,
                                                    int32_t device_ordinal,
                                                    cujpegxl_b200_acsnet_trainer** out_trainer);
void cujpegxl_b200_acsnet_trainer_destroy(cujpegxl_b200_acsnet_trainer* trainer);

/* out[n][33] (device): the 17 split logits, then the 16 log2 quant fields. */
cujpegxl_status cujpegxl_b200_acsnet_trainer_forward(cujpegxl_b200_acsnet_trainer* trainer,
                                                     const cujpegxl_b200_acsnet_batch* batch, float* out,
                                                     uintptr_t stream);

/* Gradient of the batch-mean loss (cross-entropy of the split against its
 * one-hot label or label_soft, plus qf_weight times the mean squared log2
 * quant-field error) into grad[param_count] (device), without changing the
 * parameters. stats[n][4] (device, may be
 * NULL): cross-entropy, quant-field squared error, 1 if the arg-max class is
 * the label, softmax margin. */
cujpegxl_status cujpegxl_b200_acsnet_trainer_gradient(cujpegxl_b200_acsnet_trainer* trainer,
                                                      const cujpegxl_b200_acsnet_batch* batch, float qf_weight,
                                                      float* grad, float* stats, uintptr_t stream);

/* One Adam step (beta1 0.9, beta2 0.999, epsilon 1e-8) on the batch. */
cujpegxl_status cujpegxl_b200_acsnet_trainer_step(cujpegxl_b200_acsnet_trainer* trainer,
                                                  const cujpegxl_b200_acsnet_batch* batch, float qf_weight,
                                                  float learning_rate, float* stats, uintptr_t stream);

/* Attaches `net` (NULL detaches) to every frame of a batch, as
 * cujpegxl_b200_encoder_set_acsnet does; waits for the batch's last launch,
 * and the next cujpegxl_b200_batch_encode captures and tunes its graph anew. */
cujpegxl_status cujpegxl_b200_batch_set_acsnet(cujpegxl_b200_batch* batch, const cujpegxl_b200_acsnet* net,
                                               float margin, uint32_t flags);

/* Copies the FP32 parameters to params[param_count] (host); synchronous. */
cujpegxl_status cujpegxl_b200_acsnet_trainer_params(cujpegxl_b200_acsnet_trainer* trainer, float* params);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* CUJPEGXL_B200_H_ */
