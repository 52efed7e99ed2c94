/*
 * bimp_b200.h -- C ABI of the B200-native BIMP keypoint detector.
 *
 * Plain C types only (pointers, sizes, ints, floats); no CUDA, torch or
 * OpenCV types appear in the signatures.  Streams are passed as `void*`
 * holding a cudaStream_t (NULL = the legacy default stream).
 *
 * Each entry point names the daniel-koudouna/cuda-bimp interface it replaces
 * (paths relative to that project).
 */
#ifndef BIMP_B200_H
#define BIMP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BIMP_NUM_ORI 8            /* bimp/include/detection/cuda_bimp.hpp:10 */
#define BIMP_KP_VECTOR_LENGTH 7   /* bimp/include/detection/cuda_bimp.hpp:13 */
#define BIMP_KP_MAX_POINTS 8000   /* bimp/include/detection/cuda_bimp.hpp:14 */

/* Row indices of the 7 x N device keypoint matrix (cv::cuda::SURF_CUDA
 * KeypointLayout, consumed by bimp/src/utils.cpp:130-150).  Rows 2 and 3
 * hold int32 bit patterns, the others float32. */
enum bimp_kp_row {
  BIMP_X_ROW = 0,
  BIMP_Y_ROW = 1,
  BIMP_LAPLACIAN_ROW = 2,
  BIMP_OCTAVE_ROW = 3,
  BIMP_SIZE_ROW = 4,
  BIMP_ANGLE_ROW = 5,
  BIMP_HESSIAN_ROW = 6
};

/* Status codes.  The reference prints and exit()s on any CUDA error
 * (helper_cuda.h macros, bimp/src/cuda_bimp.cu:4-10) and warns + truncates
 * on keypoint overflow (bimp/src/cuda_bimp.cu:132-138). */
typedef enum bimp_status {
  BIMP_OK = 0,
  BIMP_ERR_INVALID = -1,      /* bad argument: null pointer, size, wavelength list */
  BIMP_ERR_CUDA = -2,         /* CUDA runtime error; see bimp_last_error() */
  BIMP_ERR_NOMEM = -3,        /* device or pinned-host allocation failed */
  BIMP_ERR_CAPACITY = -4,     /* more keypoints than `capacity`; the first
                                 `capacity` (in scale, y, x order) were written
                                 and *n_found holds the true count */
  BIMP_ERR_NO_DEVICE = -5,    /* no CUDA device / not an sm_100 device */
  BIMP_ERR_UNSUPPORTED = -6   /* parameters outside what the kernels support */
} bimp_status;

/* Model constants hard-coded in bimp/src/cuda_bimp.cu (defaults = reference). */
/* Doubles, so that the defaults are the reference's double literals. */
typedef struct bimp_params {
  double gamma;         /* 0.5   cuda_bimp.cu:241 (multiplies the squared term) */
  double sigma_ratio;   /* 0.56  cuda_bimp.cu:243 */
  double size_ratio;    /* 7     cuda_bimp.cu:245 */
  double offset_ratio;  /* 0.6   cuda_bimp.cu:535 */
  double level_max;     /* 7.5   cuda_bimp.cu:236 */
  double radial_gain;   /* 16    cuda_bimp.cuh:497 */
  double w_tan;         /* 1     cuda_bimp.cuh:514 (implicit weight) */
  double w_rad;         /* 1     cuda_bimp.cuh:514 (implicit weight) */
  double thresh_ratio;  /* 0.104 cuda_bimp.cu:721 */
} bimp_params;

/* Host keypoint record, byte-compatible with cv::KeyPoint
 * {Point2f pt; float size, angle, response; int octave, class_id;}. */
typedef struct bimp_keypoint {
  float x, y;
  float size;
  float angle;
  float response;
  int32_t octave;
  int32_t class_id;
} bimp_keypoint;

/* Geometry of one scale (fields of CudaKernels, cuda_bimp.hpp:38-73). */
typedef struct bimp_scale_info {
  float lambda_full;   /* lambda2: requested wavelength */
  float lambda_level;  /* lambda: wavelength at the pyramid level */
  float pyrstep;
  int kernel_w;        /* kernelW == kernelH */
  int kernel_x;        /* kernelX == kernelY */
  int data_w, data_h;
  int fft_w, fft_h;    /* torus the reference convolves on */
  int margin;          /* (int)lambda: keypoint border margin */
} bimp_scale_info;

typedef struct bimp_context bimp_context;

/* ---- library ------------------------------------------------------------ */
const char* bimp_version(void);
/* Message of the last error on the calling thread ("" if none). */
const char* bimp_last_error(void);
/* Fills the reference defaults. */
void bimp_default_params(bimp_params* p);

/* makeLambdasLog, bimp/src/cuda_bimp.cu:927-937 (float accumulation).
 * Writes up to `cap` wavelengths; *n = number generated. */
int bimp_make_lambdas_log(float start, float end, int scales_per_octave,
                          float* out, int cap, int* n);
/* makeLambdasLin, bimp/src/cuda_bimp.cu:905-921. */
int bimp_make_lambdas_lin(float start, float end, int num_scales,
                          float* out, int cap, int* n);
/* snapTransformSize, bimp/src/cuda_bimp.cu:200-219. */
int bimp_snap_transform_size(int data_size);

/* ---- context (replaces bimp::cuda::CudaStuff) ---------------------------
 * CudaStuff(int width, int height, std::vector<float> lambdas),
 * bimp/include/detection/cuda_bimp.hpp:97, bimp/src/cuda_bimp.cu:222-397:
 * sorts the wavelengths, builds the Gabor bank and all per-scale buffers on
 * the current CUDA device.  `params` may be NULL (reference defaults). */
int bimp_ctx_create(bimp_context** ctx, int width, int height,
                    const float* lambdas, int n_lambdas,
                    const bimp_params* params);
/* The reference's Context(cv::Mat&) builds its CudaStuff from the image's
 * own size (bimp/src/bimp.cpp:7-8) but detects on getGPUImage's output,
 * which is upscaled when a side is below 350 pixels
 * (bimp/src/cuda_bimp.cu:156-168).  Each scale then filters the top-left
 * data_w x data_h window of its pyramid level of the larger image (convertTo
 * and collectCVMemory, bimp/src/cuda_bimp.cu:481-486).  This creates such a
 * context: geometry from width x height, detections taking images of
 * input_width x input_height (>= width x height). */
int bimp_ctx_create_for_input(bimp_context** ctx, int width, int height, int input_width, int input_height,
                              const float* lambdas, int n_lambdas, const bimp_params* params);
/* ~CudaStuff, bimp/src/cuda_bimp.cu:399-460. */
int bimp_ctx_destroy(bimp_context* ctx);
int bimp_ctx_num_scales(const bimp_context* ctx);
int bimp_ctx_scale_info(const bimp_context* ctx, int scale, bimp_scale_info* out);

/* ---- detection -----------------------------------------------------------
 * int getKeypoints(GpuMat& input, GpuMat& output, CudaStuff&, bool, bool),
 * bimp/include/detection/cuda_bimp.hpp:111, bimp/src/cuda_bimp.cu:109-127.
 * `d_image`: device uint8 grayscale, `pitch` bytes per row, size must equal
 * the context's.  `d_kp`: device float matrix 7 x `ld` (row r at d_kp + r*ld)
 * receiving up to `capacity` keypoints in (scale, y, x) order.  `n_found`
 * (host) receives the total count; the call synchronises `stream`. */
int bimp_detect_device(bimp_context* ctx, const uint8_t* d_image, size_t pitch,
                       int width, int height, float* d_kp, size_t ld,
                       int capacity, int* n_found, void* stream);

/* Same as bimp_detect_device without any host synchronisation: the total
 * count is written to the device int `d_count` (stream-ordered). */
int bimp_detect_device_async(bimp_context* ctx, const uint8_t* d_image, size_t pitch,
                             int width, int height, float* d_kp, size_t ld,
                             int capacity, int* d_count, void* stream);

/* Context(cv::Mat&) + Context::getKeypointsAndDownload(),
 * bimp/include/detection/bimp.hpp:35,38, bimp/src/bimp.cpp:7-20,89-92,
 * for an already-grey image: host uint8 image in, host cv::KeyPoint-layout
 * records out (utils.cpp:130-150 downloadKeypoints).  The records are
 * written on the device in this layout and come back through the context's
 * pinned staging with the count: as many as the previous call found plus a
 * margin before the one synchronisation of `stream`, the rest (a count well
 * above the previous call's) with one more copy and synchronisation. */
int bimp_detect_host(bimp_context* ctx, const uint8_t* image, size_t pitch,
                     int width, int height, bimp_keypoint* out, int capacity,
                     int* n_found, void* stream);

/* ---- pipelined host frames (no counterpart in the reference) -------------
 * The reference handles one frame per call and synchronises the device at
 * entry and exit (bimp/src/bimp.cpp:62, bimp/src/cuda_bimp.cu:115), so a
 * frame's copies never overlap another frame's work.  A pipeline holds
 * `depth` (1..8) contexts of one image size, each with its own stream, used
 * round robin: push() enqueues a host frame (its copy to the device, the
 * detection and the copy back of its records) and returns at once; pop()
 * waits for the oldest frame and returns its records as bimp_detect_host
 * does.  Up to `depth` frames are in flight, so the copies of one overlap
 * the kernels of the others.
 *
 * The frame memory passed to push() must stay unchanged until that frame is
 * popped; pinned memory keeps its copy asynchronous (pageable memory makes
 * push() wait for the copy).  `capacity` records per frame at most;
 * pop(capacity) returns BIMP_ERR_CAPACITY with the true total in *n_found
 * when a frame had more than min(capacity, the pipeline's capacity). */
typedef struct bimp_pipeline bimp_pipeline;
int bimp_pipeline_create(bimp_pipeline** pipeline, int width, int height, const float* lambdas, int n_lambdas,
                         const bimp_params* params, int depth, int capacity);
int bimp_pipeline_destroy(bimp_pipeline* pipeline);
/* BIMP_ERR_INVALID when `depth` frames are already in flight. */
int bimp_pipeline_push(bimp_pipeline* pipeline, const uint8_t* image, size_t pitch, int width, int height);
/* Records of the oldest frame in flight, in (scale, y, x) order;
 * BIMP_ERR_INVALID when no frame is in flight. */
int bimp_pipeline_pop(bimp_pipeline* pipeline, bimp_keypoint* out, int capacity, int* n_found);
int bimp_pipeline_in_flight(const bimp_pipeline* pipeline);

/* Per-scale dense maps of the last detection (Context::getResponses,
 * bimp/src/bimp.cpp:94-104; k.d_ResultDouble / k.d_ResultSingle).
 * which = 0: summed keypoint map D (double-stopped minus inhibition),
 *         1: single-stopped map S minus inhibition.
 * Copies data_h x data_w floats to device memory `d_out` (row pitch `ld`
 * floats) on `stream`. */
int bimp_dense_map(bimp_context* ctx, int scale, int which, float* d_out,
                   size_t ld, void* stream);

/* Complex-cell map C_o of the last detection for one scale/orientation
 * (cs.im.d_complex[o], bimp/src/cuda_bimp.cu:518), restricted to the
 * (data_h+1) x (data_w+1) window the stencils read. */
int bimp_complex_map(bimp_context* ctx, int scale, int orientation, float* d_out,
                     size_t ld, void* stream);

/* Line and edge detection on one scale of the last detection
 * (detectLE / detectLE_kernel, bimp/src/cuda_bimp.cu:1343-1365,
 * bimp/include/detection/cuda_bimp.cuh:362-432; the reference defines it but
 * never calls it).  Per data pixel: where the summed complex response
 * (d_ch, data_h x data_w with row pitch ch_ld floats; NULL = the sum of the
 * scale's 8 complex-cell maps) is at least 0.1, the dominant orientation's
 * odd/even responses and complex cell are tested one pixel across it.
 * Outputs (data_h x data_w, row pitch ld): d_result = the complex response
 * at detected lines/edges, else 0; d_ori = the orientation angle there
 * (o * 0.392699), else 0; d_type = 1 positive line, 2 negative line,
 * 3 positive edge, 4 negative edge, else 0.  Pixels whose one-pixel step
 * leaves the data are not detected (the reference reads past the data
 * there).  Recomputes the scale's even/odd responses (its first call
 * allocates their buffer); synchronises the stream. */
int bimp_detect_lines_edges(bimp_context* ctx, int scale, const float* d_ch, size_t ch_ld,
                            float* d_result, float* d_ori, int8_t* d_type, size_t ld,
                            void* stream);

/* ---- input preprocessing and colour features ------------------------------
 * getGPUImage size rule, bimp/src/cuda_bimp.cu:156-168: images with fewer
 * than 350 rows (and >= 350 columns) are scaled by 350/rows, otherwise
 * images with fewer than 350 columns by 350/cols (float factor, sizes
 * rounded to nearest).  *scale may be NULL. */
int bimp_min_size_dims(int width, int height, int* out_w, int* out_h, double* scale);

/* getGPUImage(cv::Mat&, bool grayscale), bimp/src/cuda_bimp.cu:156-180, for
 * an image already on the device: bilinear upscale to bimp_min_size_dims
 * (cv::resize INTER_LINEAR, 11-bit weights) and, for 3-channel BGR input with
 * grayscale != 0, BGR -> grey (cv::cuda::cvtColor COLOR_BGR2GRAY).  d_dst
 * receives out_w x out_h x (1 or channels) bytes at `dst_pitch`. */
int bimp_gpu_image(const uint8_t* d_src, size_t src_pitch, int width, int height, int channels,
                   int grayscale, uint8_t* d_dst, size_t dst_pitch, void* stream);

/* addColorFeatures, bimp/src/cuda_bimp.cu:950-958 (kernel
 * bimp/include/detection/cuda_bimp.cuh:8-71): the 24-bin colour histogram of
 * each of the n keypoints in the device 7 x kp_ld matrix, over the BGR
 * device image, into row i of `d_desc` (row pitch desc_ld floats, 24 used). */
int bimp_color_features(const float* d_kp, size_t kp_ld, int n, const uint8_t* d_bgr, size_t bgr_pitch,
                        int width, int height, float* d_desc, size_t desc_ld, void* stream);

/* ---- keypoint extraction without allocation ------------------------------
 * No counterpart in the reference (its extraction, cuda_gpu_keypoints,
 * allocates GpuMats and thrust/NPP temporaries on every call).  For callers
 * that cannot allocate device memory while they run: real-time loops that
 * must never enter the allocator (an allocation can block on a device
 * synchronisation), or hosts whose device memory all belongs to a pool the
 * library may not touch.
 *
 * Threshold (thresh_ratio * max of the map), strict 8-neighbour maxima,
 * margin (int)lambda_level and parabolic subpixel refinement on one summed
 * keypoint map `d_map` (height x width floats, row pitch `ld` floats, at
 * most INT_MAX), records written to the 7 x kp_ld device matrix `d_kp` in
 * (y, x) order.  Identical results to the extraction step of
 * bimp_detect_device for the same map.
 *
 * `*d_count` (device int, stream-ordered) receives the TRUE total, which can
 * exceed `capacity`: only the first min(total, capacity) records, in (y, x)
 * order, are written.  The count is known only on the device, so this call
 * cannot return BIMP_ERR_CAPACITY: compare *d_count with `capacity` yourself.
 *
 * All scratch lives in one fixed device array of about 260 KB per device
 * (held until the process exits); maps with more than 16384 candidate rows
 * are rejected with BIMP_ERR_UNSUPPORTED.  Nothing is allocated: no
 * cudaMalloc, cudaFree or allocating library call.  The first call on a
 * device looks up the array's device address once (with that device
 * current); make that first call before any stream capture.  Every call
 * shares the array: calls whose GPU work overlaps (unordered streams) race. */
int bimp_extract_keypoints_noalloc(const float* d_map, size_t ld, int width, int height,
                                   float lambda_level, float pyrstep, double thresh_ratio,
                                   float* d_kp, size_t kp_ld, int capacity, int* d_count,
                                   void* stream);

/* ---- measurement hooks (no counterpart in the reference) -----------------
 * Number of kernel launches one detection enqueues (all scales). */
int bimp_ctx_kernel_launches(const bimp_context* ctx);
/* Re-enqueues one stage of the last detection on `stream`, for timing a
 * single kernel with events: 0 = pyramid, 1 = tiled-FFT Gabor filtering,
 * 2 = end-stopping/inhibition stencil, 3 = NMS + compaction (into the last
 * detection's keypoint destination).  Inputs of the stage are the buffers
 * left by the previous detection, so the results are unchanged. */
int bimp_ctx_run_stage(bimp_context* ctx, int stage, void* stream);

/* ---- device memory helpers ------------------------------------------------
 * For callers (such as the header-only C++ mirror) that do not include the
 * CUDA runtime: GpuMat::create / release and upload / download
 * (cv::cuda::GpuMat, used throughout bimp/src/bimp.cpp).  bimp_copy_2d copies
 * `rows` rows of `width_bytes` between any host or device memory (direction
 * from the pointers) on `stream` and synchronises it. */
int bimp_device_alloc(void** ptr, size_t bytes);
int bimp_device_free(void* ptr);
int bimp_copy_2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width_bytes, size_t rows,
                 void* stream);

/* downloadKeypoints, bimp/src/utils.cpp:130-150: device 7 x ld matrix with n
 * columns -> host records (synchronous). */
int bimp_download_keypoints(const float* d_kp, size_t ld, int n,
                            bimp_keypoint* out, void* stream);
/* uploadKeypoints, bimp/src/utils.cpp:109-128. */
int bimp_upload_keypoints(const bimp_keypoint* kps, int n, float* d_kp,
                          size_t ld, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* BIMP_B200_H */
