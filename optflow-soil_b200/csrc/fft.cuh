// fft.cuh -- arbitrary-length FP32 FFTs staged in shared memory, fused with the Gabor filter bank and the
// cubic B-spline prefilter (the "responses" of the fine stage, python/optflow_ref/phaseflow.py:455-456).
#pragma once
#include "common.cuh"

namespace ofc {

constexpr int FFT_MAXST = 16;
// the padded length of 2048-wide images, whose transforms run on a plan fixed at compile time
constexpr int FFT_FIXED_L = 2112;
// the lengths whose transforms run on plans fixed at compile time (their factor order is the default one: the plan
// table's variants apply to the other lengths): the padded lengths (side + 64) of sides 256, 512, 768, 960, 1024,
// 1536 and 2048
bool fft_fixed_length(int L);
// the Bluestein inner length whose two transforms run on a plan fixed at compile time: that of 604 = 4 151 (the
// padded height of 540-row frames), 1216 = 8 8 19
constexpr int FFT_FIXED_M = 1216;
constexpr int FFT_E = 8;       // complex values per thread (sets the threads of a block)
constexpr int FFT_TMAX = 512;  // threads per block at most

// A 1-D plan of length L: mixed-radix Stockham stages (radix p[i], stride s[i] = product of the radices
// before it) and the twiddle table W[t] = exp(-2 pi i t / L), t < L, rounded from float64.
// A length with a prime factor above 31 is transformed by Bluestein's chirp z-transform (as the reference's Metal
// FFT does, rust/crates/optflow-gpu/src/fft.rs:1-3): M > 0 is then the inner length (a length >= 2L - 1 of
// the radices with butterflies, of fewest stages: fft_work_length), the stages and tw are those of length M, chirp[n] = exp(-i pi n^2 / L) for n < L, and filt is the
// length-M transform of the conjugate chirp (wrapped: index m and M - m for m < L) times 1 / M.
struct FftPlan {
  int L = 0;
  int nst = 0;
  int p[FFT_MAXST] = {};
  int s[FFT_MAXST] = {};
  unsigned magic[FFT_MAXST] = {};
  const float2* tw = nullptr;
  int M = 0;
  const float2* chirp = nullptr;
  const float2* filt = nullptr;
};

// the length the stages of L's plan run on (and the shared-memory buffers are sized for): L, or Bluestein's M
__host__ __device__ inline int fft_work_len(const FftPlan& p) { return p.M ? p.M : p.L; }

// radices with a register-resident butterfly: the lengths transformed directly
bool fft_supported(int L);
// the stages' length of a plan of L (L itself, or Bluestein's inner length); 0 when no plan exists
int fft_work_length(int L);
// whether the column and row passes of a ph x pw padded window fit in shared memory
bool fft_fits(int ph, int pw);
// host: factor L (or Bluestein's M) and fill p/s; the caller sets tw (fft_twiddles(fft_work_length(L))) and, for
// Bluestein, chirp and filt (fft_bluestein_tables: L chirp values, then M filter values)
FftPlan fft_make_plan(int L);
// the plan with a given factor order (0 .. FFT_PLAN_VARIANTS - 1); fft_make_plan(L) takes the plan table's choice
constexpr int FFT_PLAN_VARIANTS = 4;
FftPlan fft_make_plan(int L, int variant);
// the process-wide plan table: the factor order of the runtime plans of length L (0: the default order); plans an
// engine has already built keep theirs
void fft_set_plan_variant(int L, int variant);
int fft_plan_variant(int L);
std::vector<float2> fft_twiddles(int L);
std::vector<float2> fft_bluestein_tables(int L, int M);
// threads of a block that transforms C interleaved lines of length L (multiple of C and of 32)
int fft_threads(int L, int C);

// Separable Gabor tables of one padded size (gabor_bank, phaseflow.py:73-89). Filter k is
//   G_k(x, y) = hp(x, y) ex_k[x] ey_k[y],  hp = 1 - hx[x] hy[y] = omx[x] + hx[x] omy[y]
// with hx = exp(-f^2 s_hp^2 / 2) and omx = 1 - hx = -expm1(-f^2 s_hp^2 / 2) (no cancellation near DC), the
// frequency grids fx, fy = np.fft.fftfreq * 2 pi, and the Gaussian factors ex_k, ey_k of filter k. float64 tables
// (the reference pack) and float32 copies (the responses).
struct GaborTables {
  int F = 0, ph = 0, pw = 0;
  const double *fx = nullptr, *fy = nullptr, *hx = nullptr, *hy = nullptr, *omx = nullptr, *omy = nullptr;
  const double *ex = nullptr, *ey = nullptr;
  const float *hxf = nullptr, *omxf = nullptr, *omyf = nullptr, *exf = nullptr, *eyf = nullptr;
  const float *bxf = nullptr, *byf = nullptr;  // 1 / (4 + 2 cos w) per axis: the B-spline prefilter on the periodic grid
  const float2* yt2 = nullptr;  // per filter k and row y: (omy[y], ey_k[y] by[y]) (float32)
};
// host tables: float64 [fx pw | fy ph | hx pw | hy ph | omx pw | omy ph | ex F*pw | ey F*ph | bx pw | by ph], then
// from gabor_yt2_offset (even) the pairs (omy[y], ey_k[y] by[y]) per filter and row
std::vector<double> gabor_tables_host(int ph, int pw, const ofc_config& c);
size_t gabor_yt2_offset(int ph, int pw, int F);
// binds g to a device copy of the tables: d64 (the host float64 vector) and d32 (its float32 image)
void gabor_bind(GaborTables& g, const double* d64, const float* d32, int ph, int pw, int F);

// forward row transforms of the reflect-padded real image img (W x H) -> out (ph x pw)
void launch_fft_rows_fwd_real(const float* img, int W, int H, const FftPlan& plw, int ph, float2* out,
                              cudaStream_t st);
// column transforms of the responses: forward (in place in T, which then holds the 2-D spectrum), then per
// filter multiply + inverse + B-spline prefilter along y -> U: F planes (ph x pw)
void launch_fft_cols_filters(float2* T, const FftPlan& plh, int pw, const GaborTables& g, float2* U, cudaStream_t st);
// inverse row transforms + B-spline prefilter along x + scale -> responses R in filter pairs, node-major: filter
// 2j + c at node (y, x) at R[((j ph + y) pw + x) 2 + c] (pair j's second filter a copy of filter F - 1 when F is odd);
// R holds resp_values(F, ph * pw) values
void launch_fft_rows_inv_resp(const float2* U, const FftPlan& plw, int ph, int F, float2* R, cudaStream_t st);
inline size_t resp_values(int F, size_t Np) { return (size_t)2 * ((F + 1) / 2) * Np; }

// the reference pack (reference_phase, phaseflow.py:92-112). launch_fft_cols_fwd: forward column transforms of the
// row-transformed T, in place (T then holds the 2-D spectrum S); launch_fft_cols_ref_f32: for filters [k0, k1) the
// 3 planes per filter S G, S G i fx, S G i fy (the factors formed in float64), inverse along y, into U; then the
// inverse row transforms cropped to W x H with, per pixel, (r.re, r.im, gx, gy) and amp formed in float64 and
// stored float32. The transforms are float32, as the reference's Rust port computes them (rustfft f32,
// gabor.rs:230-270).
void launch_fft_cols_fwd(float2* T, const FftPlan& plh, int pw, cudaStream_t st);
void launch_fft_cols_ref_f32(const float2* S, const FftPlan& plh, int pw, const GaborTables& g, int k0, int k1,
                             float2* U, cudaStream_t st);
void launch_fft_rows_inv_ref_f32(const float2* U, const FftPlan& plw, int ph, int k0, int k1, int W, int H,
                                 float4* ref4, float* amp, cudaStream_t st);

// generic complex FFT of C-line batches held in global memory (tests and tools): data (lines x L)
void launch_fft_lines(float2* data, int lines, const FftPlan& pl, bool inverse, cudaStream_t st);

}  // namespace ofc
