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

/* One tile plan of the tiled-FFT filtering: `policy` 0 uses the largest
 * valid block per 128 x 128 tile (128 - 2 kX outputs per side), 1 rounds it
 * down to a multiple of 32 where that keeps at least 3/4 of it (more tiles,
 * evenly split passes); `order` 0 queues tiles scale by scale, 1 interleaves
 * the scales' tiles; `kernel` 1 runs the warp-specialised tile kernel (the
 * inverse y-passes of one orientation overlap the x-passes of the previous
 * one; needs every valid block <= 104), 0 the phased one (all warps pass by
 * pass); `grid` 0 launches one CTA per tile, grid > 0 at most that many
 * persistent CTAs that share the (tile, orientation) pairs in contiguous runs
 * of equal estimated cost (a tile cut between two CTAs is transformed
 * forward by both; the default plan uses one CTA per SM).  `tiles` is the
 * plan's tile count.  `ms` is the measured time of one
 * detection of the batch with the plan. */
typedef struct {
  int policy;
  int order;
  int kernel;
  int grid;
  int tiles;
  float ms;
} bimp_tile_plan;

/* Autotuner (no counterpart in the reference): times every tile plan
 * (2 kernels x 2 policies x 2 orders x 3 grids: one CTA per tile, or the
 * split plan over one or two CTAs per SM)
 * over `reps` detections of the batch's current inputs on `stream`, keeps
 * the fastest and recaptures the graph with it.  Plans of one policy give
 * bitwise identical results; policy 1 moves tile boundaries, which changes
 * the float rounding of the filtered maps (well inside the parity
 * tolerance).  The fastest plan goes to *chosen, the first max_tried
 * timings to tried[], their number to *n_tried.  Synchronises the stream. */
int bimp_batch_autotune(bimp_batch* batch, void* stream, int reps, bimp_tile_plan* chosen,
                        bimp_tile_plan* tried, int max_tried, int* n_tried);

/* Uses the given tile plan (e.g. one the autotuner chose earlier) and
 * recaptures the graph; grid <= 0 means one CTA per tile, grid > 0 the split
 * plan over at most `grid` persistent CTAs (BIMP_ERR_INVALID if that plan's
 * work list exceeds the buffer sized at creation); kernel 1 falls back
 * to the phased kernel where the pipelined one does not fit. */
int bimp_batch_set_tile_plan(bimp_batch* batch, int policy, int order, int grid, int kernel);

/* Replays the captured graph on `stream` (no host synchronisation). */
int bimp_batch_run(bimp_batch* batch, void* stream);

/* Copies the per-image keypoint totals (n_images ints) to device memory. */
int bimp_batch_counts(bimp_batch* batch, int* d_counts, void* stream);

/* Internal 7 x ld keypoint matrix of image i, (scale, y, x) order; only the
 * first min(count, ld) columns are written. */
int bimp_batch_keypoints_device(bimp_batch* batch, int i, const float** d_kp, size_t* ld);

/* Geometry of image i at one scale (as bimp_ctx_scale_info for a context of
 * that image's size). */
int bimp_batch_scale_info(const bimp_batch* batch, int i, int scale, bimp_scale_info* out);

/* Summed keypoint map D of image i, scale `scale` from the last run
 * (Context::getResponses, bimp/src/bimp.cpp:94-104, for one image of the
 * batch): data_h x data_w floats to device memory `d_out` (row pitch `ld`
 * floats) on `stream`. */
int bimp_batch_dense_map(bimp_batch* batch, int i, int scale, float* d_out, size_t ld, void* stream);

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
