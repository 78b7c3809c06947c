// Launch parameters and launchers of the transform kernels (device side in
// kernels.cu).  Every offset and stride is in complex elements of the pass's
// precision; a pass sees its data as lines of N points.
#pragma once
#include <cuda_runtime.h>

#include "engine.cuh"

namespace b2f {

enum Prec : int { PREC_F32 = 0, PREC_F64 = 1, PREC_DF64 = 2 };

// Bytes of one complex value of each precision.
inline size_t complex_bytes(Prec p) { return p == PREC_F32 ? 8 : 16; }

enum PassFlags : uint32_t {
  PF_CONJ_IN = 1u << 0,      // conjugate on load (inverse through the forward kernels)
  PF_CONJ_OUT = 1u << 1,     // conjugate on store
  PF_SCALE = 1u << 2,        // multiply by `scale` on store
  PF_TW_STORE = 1u << 3,     // multiply output k of inner line c by W_M^{c k}
  PF_CFIRST_LOAD = 1u << 4,  // adjacent lines first when loading (column tiles)
  PF_CFIRST_STORE = 1u << 5, // adjacent lines first when storing
  PF_TW_TABLE = 1u << 6,     // stage twiddles from the plan table (else computed)
  PF_STORE_SMEM = 1u << 7,   // register kernel: final store through shared memory, lines first
};

// Where the G lines of one CTA live.  Lines are numbered
// line = (outer * mid_n + mid) * inner_n + inner, and the line at
// (outer, mid, inner) starts at outer*X_outer + mid*X_mid + inner*X_inner
// with its points X_es apart (X = in or out).  A CTA takes G consecutive
// `inner` lines of one (outer, mid) row: adjacent columns when X_inner is 1,
// consecutive contiguous lines when X_inner is the line length.
struct LineIO {
  uint32_t inner_n, mid_n;
  uint32_t tiles;  // ceil(inner_n / G)
  uint32_t tw_div; // inner index / tw_div = the four-step row index
  int64_t in_es, in_inner, in_mid, in_outer;
  int64_t out_es, out_inner, out_mid, out_outer;
};

struct LinesParams {
  const void* in;
  void* out;
  const void* tw;  // stage twiddle table (PF_TW_TABLE)
  uint32_t N, G, LD, flags;
  FastDiv dN, dG;
  LineIO io;
  FastDiv d_tw;         // division by io.tw_div
  uint64_t tw_store_M;
  // PF_TW_STORE from tables (when tws_a is set): W_M^m = tws_a[m / L] *
  // tws_b[m % L], L = d_tws.d (a power of two), both tables built in FP64
  // and rounded once
  const void* tws_a;
  const void* tws_b;
  FastDiv d_tws;
  double scale;
  Schedule sch;
};

// Rader: prime N, convolution of length N-1 through sch (length N-1).
struct RaderParams {
  LinesParams L;  // L.N = p (the line), L.sch = schedule of p - 1
  const uint32_t* perm_in;   // perm_in[q] = g^q mod p, q < p-1
  const uint32_t* perm_out;  // perm_out[n-1] = r with g^-r = n (mod p), 1 <= n < p
  const void* bhat;          // FFT_{p-1}(b) / (p-1), b[q] = W_p^{g^-q}
  FastDiv dP1;               // division by p - 1
};

// Bluestein: N points through a length-M convolution (sch has length M).
struct BluesteinParams {
  LinesParams L;  // L.N = line length, L.sch = schedule of M
  uint32_t M;
  const void* bhat;  // FFT_M(b) / M, b = conjugate chirp, symmetric
  FastDiv dM, dMN;   // division by M and by M - N
  const void* chirp;  // exp(-i pi n^2 / N) for n < N, FP64-built (null: computed in-kernel)
};

// Bluestein over a convolution too long for one CTA: the chirp
// pre-multiply (in layout -> workspace lines of M), the spectrum product
// (in place on the workspace) and the chirp post-multiply (workspace ->
// out layout) run as separate passes around multi-pass FFT_M.
// Elementwise passes of the multi-pass Bluestein (BE_PRE/MID/POST) and
// Rader (BE_RADER_*) routes.
enum BlueElemMode : uint32_t {
  BE_PRE = 0, BE_MID = 1, BE_POST = 2, BE_RADER_PRE = 3, BE_RADER_MID = 4, BE_RADER_POST = 5
};
struct BlueElemParams {
  const void* in;
  void* out;
  const void* bhat;
  uint32_t N, M, mode, flags;
  uint64_t s, nlines;  // axis stride and number of lines (line l = o*s + i)
  double scale;
  const void* chirp;   // exp(-i pi n^2 / N) for n < N, FP64-built (null: computed in-kernel)
  // Rader (N = p prime, M = p - 1): perm_in[q] = g^q, perm_out[n-1] = r with
  // g^-r = n, and two values a line (x[0], X[0]) kept between the passes
  const uint32_t* perm_in;
  const uint32_t* perm_out;
  void* x0;
};

// Generic real transforms (any N0): axis-0 lines expanded to full complex
// lines, transformed by any complex route, then packed (R2C); or the
// Hermitian mirror of the packed half, an inverse complex route, the real
// part (C2R).  Lines are contiguous: real line r at r*N0, packed at r*P,
// complex line at r*N0.
enum RealElemMode : uint32_t { RE_EXPAND = 0, RE_PACK = 1, RE_UNPACK = 2, RE_TAKE_REAL = 3 };
struct RealElemParams {
  const void* in;
  void* out;
  uint32_t N0, P, mode, pad;
  uint64_t nlines;
};

// Real transforms on axis 0 (contiguous lines; batches and the other axes
// are `nlines` lines, real line r at r*N0 floats, packed line at r*(N0/2+1)).
struct RealParams {
  const void* in;
  void* out;
  const void* tw;
  uint32_t N0, h, G, LD, flags;
  uint64_t nlines;
  double scale;
  FastDiv dh, dG, dN0, dP;  // h, G, N0, packed length
  Schedule sch;             // schedule of h (even N0) or N0 (odd N0)
  const void* rtw;          // fixed-length kernels: W_N0^k for k < h (FP64-built)
};

// Small volumes (the crate's SmallVolumePlan, src/runtime/small_volume.rs:
// 1-42, 223-272): every axis of a C2C volume of at most 4096 points in one
// CTA and one HBM pass.  The CTA loads its volume into shared memory, runs
// each axis over all of that axis's lines (gathered into lines of pitch LD,
// transformed by the Stockham engine, scattered back) and stores it.
constexpr int kSmallVolumeMaxRank = 3;
constexpr uint32_t kSmallVolumeMaxPoints = 4096;
struct SmallVolumeParams {
  const void* in;
  void* out;
  const void* tw;  // stage twiddles of every axis (sch[a].st[s].tw_off into it)
  uint32_t rank, V, flags, buf;  // V points per volume, buf = values per work buffer
  uint32_t dims[kSmallVolumeMaxRank], strides[kSmallVolumeMaxRank], LD[kSmallVolumeMaxRank];
  FastDiv dN[kSmallVolumeMaxRank], dS[kSmallVolumeMaxRank];
  uint64_t nvol;
  double scale;
  Schedule sch[kSmallVolumeMaxRank];
};

// Per-precision launchers (kernels.cu).
cudaError_t launch_lines(Prec p, const LinesParams& prm, unsigned grid, unsigned threads,
                         size_t smem, cudaStream_t st);
// Register-resident power-of-two lines: E values per thread, column-major
// (adjacent lines first) or line-major thread order.
// TMA-staged column tiles (tmatile.cu): whether a pass's shape can use
// them, their CTAs per SM, and the launch (false: not launched, the input
// view cannot be a tensor map; *err carries a launch error otherwise).
bool tma_tile_shape_ok(const LinesParams& lp, uint64_t outer_n);
int tma_tile_ctas_per_sm(const LinesParams& lp, unsigned threads);
bool launch_pow2_tma(const LinesParams& lp, uint64_t ntiles, uint64_t outer_n, unsigned threads,
                     unsigned grid, unsigned int* flag, cudaStream_t st, cudaError_t* err);
// Even-length real transforms whose half is a power of two (16..4096),
// f32/f64, on the fixed-length register kernels (regfft_fixed.cuh):
// cudaErrorInvalidValue when no such kernel exists.
cudaError_t launch_real_fixed(Prec p, bool r2c, const RealParams& prm, unsigned grid,
                              unsigned threads, size_t smem, cudaStream_t st);
cudaError_t launch_pow2(Prec p, int E, bool colmajor, const LinesParams& prm, unsigned grid,
                        unsigned threads, size_t smem, cudaStream_t st);
cudaError_t launch_rader(Prec p, const RaderParams& prm, unsigned grid, unsigned threads,
                         size_t smem, cudaStream_t st);
cudaError_t launch_bluestein(Prec p, const BluesteinParams& prm, unsigned grid,
                             unsigned threads, size_t smem, cudaStream_t st);
cudaError_t launch_r2c(Prec p, const RealParams& prm, unsigned grid, unsigned threads,
                       size_t smem, cudaStream_t st);
cudaError_t launch_c2r(Prec p, const RealParams& prm, unsigned grid, unsigned threads,
                       size_t smem, cudaStream_t st);
cudaError_t launch_blue_elem(Prec p, const BlueElemParams& prm, cudaStream_t st);
cudaError_t launch_real_elem(Prec p, const RealElemParams& prm, cudaStream_t st);
cudaError_t launch_small_volume(Prec p, const SmallVolumeParams& prm, unsigned threads,
                                size_t smem, cudaStream_t st);
// out[i] = scale * (conj?) in[i] for n complex values (length-1 transforms).
cudaError_t launch_scale_copy(Prec p, const void* in, void* out, uint64_t n, double scale,
                              bool conj, cudaStream_t st);

// Largest dynamic shared memory a CTA may use on this device.
size_t max_smem_per_block();

// Values per thread per stage the kernels of a precision are built for.
inline uint32_t emax_of(Prec p) { return p == PREC_F32 ? 32u : 16u; }

}  // namespace b2f
