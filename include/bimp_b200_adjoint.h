/*
 * bimp_b200_adjoint.h -- gradient of a weighted sum of the summed keypoint
 * maps (the dense, pre-NMS output of the detector).
 *
 * No counterpart in the reference, which only runs forward.  For a batch of
 * n float images X_i (H x W, values in [0, 1] standing for u8/255) the
 * forward computes, per scale s, the summed keypoint map D_is through a float
 * pyramid (pyrDown without uint8 rounding) and the same Gabor / end-stopping /
 * inhibition path as bimp_detect_device, and the loss
 *
 *     L = sum_i sum_s sum_{y,x} M_is[y,x] * D_is[y,x].
 *
 * The backward returns dL/dX_i and dL/d(alpha, rho, w_tan, w_rad):
 *   alpha  scale factor of every wavelength (lambda -> alpha * lambda) at 1,
 *   rho    sigma / lambda at the bank's sigma_ratio (0.56),
 *   w_tan, w_rad  weights of tangential and radial inhibition in
 *          D = D_double - w_tan * T - w_rad * R, at the params' values (1, 1).
 * Kernel sizes, stencil offsets, pyramid steps and margins stay at their
 * nominal values (they are integer functions of lambda); ReLU derivatives
 * are 0 at 0, and a complex response |e + i o| <= 3e-5 passes no gradient
 * (exactly flat image regions give |e + i o| = 0 up to rounding, where the
 * magnitude has no derivative; the value assumes images on the [0, 1] scale).
 * The forward keeps the complex responses and each tile's image spectrum
 * for the backward.
 */
#ifndef BIMP_B200_ADJOINT_H
#define BIMP_B200_ADJOINT_H

#include "bimp_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bimp_adjoint bimp_adjoint;

/* n_images float images of width x height, one wavelength bank. */
int bimp_adjoint_create(bimp_adjoint** out, int width, int height, int n_images, const float* lambdas,
                        int n_lambdas, const bimp_params* params);
int bimp_adjoint_destroy(bimp_adjoint* a);
int bimp_adjoint_num_scales(const bimp_adjoint* a);

/* Layout of the loss weights: image i, scale s occupies data_h x data_w
 * floats at d_masks + i * mask_stride + offset. */
int bimp_adjoint_mask_layout(const bimp_adjoint* a, int scale, int* data_w, int* data_h, size_t* offset,
                             size_t* mask_stride);

/* Forward: images (n x height rows of `pitch` floats, image i starting at
 * d_images + i * height * pitch) and weights in; the loss (one double) is
 * written to the device pointer d_loss.  Stream-ordered, no host sync. */
int bimp_adjoint_forward(bimp_adjoint* a, const float* d_images, size_t pitch, const float* d_masks, double* d_loss,
                         void* stream);

/* Backward of the last forward: dL/dX into d_grad (same layout as the
 * images) and dL/d(alpha, rho, w_tan, w_rad) into 4 device doubles. */
int bimp_adjoint_backward(bimp_adjoint* a, float* d_grad, size_t pitch, double* d_grad_params, void* stream);

/* Summed keypoint map of image i, scale s of the last forward (device copy,
 * data_h x data_w, row pitch ld floats). */
int bimp_adjoint_dense_map(bimp_adjoint* a, int image, int scale, float* d_out, size_t ld, void* stream);

/* Complex cells |e + i o| of image i, scale s, orientation o of the last
 * forward over the stencil window: (data_h + 1) x (data_w + 1) floats, row
 * pitch ld, element (r, c) = the torus element r * fftW + c (so column data_w
 * is row r + 1, column 0 when fftW == data_w).  The backward's ReLU states and
 * magnitude floor are functions of these values. */
int bimp_adjoint_complex_map(bimp_adjoint* a, int image, int scale, int orientation, float* d_out, size_t ld,
                             void* stream);

/* Device bytes held by the adjoint's buffers. */
size_t bimp_adjoint_device_bytes(const bimp_adjoint* a);

#ifdef __cplusplus
}
#endif
#endif /* BIMP_B200_ADJOINT_H */
