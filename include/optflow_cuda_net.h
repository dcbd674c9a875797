/*
 * optflow_cuda_net.h -- the learned coarse proposal: a small convolutional network that predicts the displacement
 * field at 1/8 resolution from an image pair, trained and run on the GPU with bfloat16 tensor-core kernels and
 * float32 accumulation. It can replace the POC coarse stage of a pair (python/optflow_ref/poc.py:216-239,
 * rust/crates/optflow-core/src/poc.rs:694 coarse_flow, reached from track.rs:578); the phase refinement always
 * follows, and tiles whose refined result fails the confidence test fall back to POC (ofc_set_coarse_net below).
 * The reference has no counterpart: every entry point here is an extension.
 *
 * Network (weights in one float32 vector of ofc_net_param_count() values; per layer a [cout][kpad] weight matrix,
 * kpad = 9 cin rounded up to 16, column (ky * 3 + kx) * cin + c, then cout biases):
 *   encoder (both images): 3x3/2 1->16 ReLU, 3x3/2 16->32 ReLU, 3x3/2 32->32 ReLU, 3x3 32->32
 *   correlation of the two 1/8 feature maps over +-5 cells (121 channels)
 *   decoder on [correlation, features of image 1, 7 zero channels]: 3x3 160->64 ReLU, 3x3 dil 2 64->64 ReLU,
 *   3x3 dil 4 64->32 ReLU, 3x3 32->16 (2 used)
 *   flow = 8 * soft-argmax of the correlation + the decoder's two channels, in pixels at the cell centres
 *   (8 i + 3.5, 8 j + 3.5).
 * Device pointers and a caller stream throughout; errors as in optflow_cuda.h.
 */
#ifndef OPTFLOW_CUDA_NET_H
#define OPTFLOW_CUDA_NET_H

#include "optflow_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ofc_net ofc_net;

/* number of float32 parameters */
OFC_API size_t ofc_net_param_count(void);

/* a network on `device` with its parameters, Adam moments and work buffers (parameters zero until set) */
OFC_API ofc_net* ofc_net_create(int device, char* err, size_t errlen);
OFC_API void ofc_net_destroy(ofc_net* net);

/* host copies of the float32 parameters; setting them resets the Adam state */
OFC_API int ofc_net_set_params(ofc_net* net, const float* params, size_t n, char* err, size_t errlen);
OFC_API int ofc_net_get_params(ofc_net* net, float* params, size_t n, char* err, size_t errlen);

/* flow (nb x h/8 x w/8 x 2 floats) of nb pairs of h x w float32 images (i1, i2: nb images each, contiguous);
 * h, w multiples of 8, at least 16 */
OFC_API int ofc_net_forward(ofc_net* net, const float* i1, const float* i2, int nb, int h, int w, float* flow,
                            void* stream, char* err, size_t errlen);

/* forward + backward of loss = (1 / cells) sum over the cells with mask != 0 of sqrt(|flow - target|^2 + 0.01)
 * (target nb x h/8 x w/8 x 2 px, mask nb x h/8 x w/8 bytes); grads (device, ofc_net_param_count floats) receive
 * the gradient (NULL: the network's own buffer, which ofc_net_adam then reads), *loss the loss (host double; the
 * call then synchronises the stream). */
OFC_API int ofc_net_gradients(ofc_net* net, const float* i1, const float* i2, int nb, int h, int w,
                              const float* target, const uint8_t* mask, float* flow, float* grads, double* loss,
                              void* stream, char* err, size_t errlen);

/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8, learning rate lr) on `grads` (NULL: the network's own buffer) */
OFC_API int ofc_net_adam(ofc_net* net, const float* grads, float lr, void* stream, char* err, size_t errlen);

/* The learned proposal in an engine's pair calls (ofc_track_pair, ofc_track_pair_device, ofc_track_pairs) that have
 * no start field: the network's flow, interpolated between the cell centres, starts the fine stage in place of the
 * POC grid. After the fine stage every tile of tile x tile pixels is judged on its pixels inside the ROI and beyond
 * 4 sigma_w + 40 px of the border: it fails when more than max_low_share of them have conf < conf_min. When a tile
 * fails, POC runs, its dense start replaces the network's inside the failed tiles, and the fine stage runs again
 * from that start. params: ofc_net_param_count() floats (host memory); NULL: the POC coarse stage again (the
 * default). Sequence legs and pairs with a start field always use POC. The engine must be idle (OFC_ERR_BUSY). */
OFC_API int ofc_set_coarse_net(ofc_engine* eng, const float* params, size_t n, int tile, double max_low_share,
                               char* err, size_t errlen);

/* Counters of the learned proposal since ofc_set_coarse_net: out[0] pairs, out[1] tiles judged, out[2] tiles that
 * failed, out[3] pairs that fell back to POC. */
OFC_API int ofc_coarse_net_stats(ofc_engine* eng, uint64_t* out);

#ifdef __cplusplus
}
#endif
#endif /* OPTFLOW_CUDA_NET_H */
