// synth.cu -- speckle rendering on the GPU (python/optflow_ref/synth.py:20-190 restated): Gaussian blobs
// evaluated at the inverse-mapped coordinates of ss x ss subsamples per pixel, 0.5 + 0.25 tanh(mean), float64.
#include "common.cuh"
#include "synth_field.cuh"

namespace ofc {

// synth.render (synth.py:150-190) as a gather: blob k adds a_k exp(-d^2 / (2 r_k^2)) to exactly the subsamples
// [i0, i1) x [j0, j1) that the reference's per-blob rectangle covers (half size 5.2 r_k + 2 around the mapped
// centre, computed on the host with the reference's floor/ceil); blobs are binned by the cell of their mapped
// centre, and a cell is at least the largest half size + 1 px wide, so the 3 x 3 cells around a subsample hold
// every blob whose rectangle contains it. d is measured between the subsample's inverse-mapped position and the
// blob's reference centre; the pixel is 0.5 + 0.25 tanh(mean of its ss x ss subsamples), all in float64.
__global__ void k_synth_render(const SynthBlob* __restrict__ blobs, const int* __restrict__ cell_start, int ncx,
                               int ncy, double cell, int w, int h, int ss, const ofc_field* field, double* out) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= w) return;
  double acc = 0;
  for (int si = 0; si < ss; si++)
    for (int sj = 0; sj < ss; sj++) {
      int i = y * ss + si, j = x * ss + sj;
      double xs = x + ((sj + 0.5) / ss - 0.5), ys = y + ((si + 0.5) / ss - 0.5);
      double X = xs, Y = ys;
      if (field) field_inverse(*field, xs, ys, X, Y);
      int cx = (int)floor((xs + cell) / cell), cy = (int)floor((ys + cell) / cell);
      double a = 0;
      for (int cj = max(cy - 1, 0); cj <= min(cy + 1, ncy - 1); cj++)
        for (int ci = max(cx - 1, 0); ci <= min(cx + 1, ncx - 1); ci++) {
          int c = cj * ncx + ci;
          for (int b = cell_start[c]; b < cell_start[c + 1]; b++) {
            const SynthBlob& B = blobs[b];
            if (i < B.i0 || i >= B.i1 || j < B.j0 || j >= B.j1) continue;
            double dx = X - B.cx, dy = Y - B.cy;
            a += B.a * exp(-(dx * dx + dy * dy) / (2 * (B.r * B.r)));
          }
        }
      acc += a;
    }
  out[(size_t)y * w + x] = 0.5 + 0.25 * tanh(acc / (ss * ss));
}

void synth_render_dev(const SynthBlob* blobs, const int* cell_start, int ncx, int ncy, double cell, int w, int h,
                      int ss, const ofc_field* field, double* out, cudaStream_t st) {
  dim3 g(div_up(w, 128), h);
  OFC_LAUNCH(k_synth_render, g, 128, 0, st, blobs, cell_start, ncx, ncy, cell, w, h, ss, field, out);
}

}  // namespace ofc
