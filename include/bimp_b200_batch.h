/*
 * bimp_b200_batch.h -- batched detection over many images of mixed sizes.
 *
 * The reference processes one image per call (bimp::cuda::getKeypoints,
 * bimp/include/detection/cuda_bimp.hpp:109, looping over scales and
 * orientations with ~90 launches and a host round trip per scale,
 * bimp/src/cuda_bimp.cu:462-559).  A batch runs the same detector on N
 * images at once: each kernel type is launched once for all images and all
 * scales, and the whole sequence is captured in a CUDA graph at creation and
 * replayed by bimp_batch_run().  Per-image results equal N calls of
 * bimp_detect_device() on the same images.
 */
#ifndef BIMP_B200_BATCH_H
#define BIMP_B200_BATCH_H

#include "bimp_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bimp_batch bimp_batch;

/* Builds the bank, all buffers and the CUDA graph for `n_images` images of
 * sizes widths[i] x heights[i] on the current device.  Keypoints go to
 * internal 7 x kp_capacity matrices, one per image. */
int bimp_batch_create(bimp_batch** batch, const int* widths, const int* heights,
                      int n_images, const float* lambdas, int n_lambdas,
                      const bimp_params* params, int kp_capacity);
int bimp_batch_destroy(bimp_batch* batch);
int bimp_batch_num_images(const bimp_batch* batch);

/* Device input buffer of image i (uint8, `pitch` bytes per row); the caller
 * writes the image there before bimp_batch_run(). */
int bimp_batch_image(bimp_batch* batch, int i, uint8_t** d_image, size_t* pitch);

/* Replays the captured graph on `stream` (no host synchronisation). */
int bimp_batch_run(bimp_batch* batch, void* stream);

/* Copies the per-image keypoint totals (n_images ints) to device memory. */
int bimp_batch_counts(bimp_batch* batch, int* d_counts, void* stream);

/* Internal 7 x ld keypoint matrix of image i, (scale, y, x) order; only the
 * first min(count, ld) columns are written. */
int bimp_batch_keypoints_device(bimp_batch* batch, int i, const float** d_kp, size_t* ld);

/* Host images in, host keypoints out: uploads every image, replays the
 * graph, downloads totals and records.  n_found[i] receives each image's
 * total; returns BIMP_ERR_CAPACITY if any exceeded its capacity. */
int bimp_batch_detect_host(bimp_batch* batch, const uint8_t* const* images,
                           const size_t* pitches, bimp_keypoint* const* outs,
                           const int* capacities, int* n_found, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* BIMP_B200_BATCH_H */
