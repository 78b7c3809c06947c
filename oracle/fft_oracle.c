/*
 * FP64 host oracle for the FFT transform path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the parity tests,
 * smoke() and the bench's CPU-baseline leg compare against; the product
 * (wgpufft_b200/) never links, loads or calls it.
 *
 * It restates, in plain C, the reference crate's host math module
 * (src/math/mod.rs of MaximEremenko/wgpuFFT):
 *   - fft_f64 / fft_f64_recursive  (src/math/mod.rs:274-361): mixed-radix
 *     Cooley-Tukey that splits off the smallest prime factor, plain DFT for
 *     primes <= 64 (MAX_DIRECT_PRIME_F64, :294), Bluestein above;
 *   - bluestein_f64                (src/math/mod.rs:366-405);
 *   - reference_c2c_nd_f64         (src/math/mod.rs:214-266): axis-by-axis
 *     lines, axis 0 contiguous, batches as contiguous blocks, scale applied
 *     on the last transformed axis;
 *   - reference_c2c_nd             (src/math/mod.rs:155-208): the f32 plain
 *     DFT, restated bit-for-bit in float for the small known-answer tests;
 *   - reference_r2c_packed_interleaved / reference_c2r_from_packed_interleaved
 *     (src/math/mod.rs:81-153) with packed_coords_for_full_spectrum and
 *     is_self_conjugate_bin (src/math/mod.rs:466-502);
 *   - FftConfig::scale / scale_f64 (src/config.rs:262-286);
 *   - line_base_for_axis / strides_for_shape (src/math/mod.rs:430-516,
 *     src/runtime/nd_wgsl.rs:57-75).
 * The real-transform helpers here run the full spectrum through the FP64
 * path (the reference runs its f32 plain DFT there); the packing and the
 * Hermitian mirror are the reference's.
 *
 * Enumerations follow the reference: direction 0 = Forward, 1 = Inverse;
 * normalization 0 = None, 1 = Forward, 2 = Inverse (default), 3 = Orthogonal.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    double re, im;
} cd;

static const double TAU = 6.283185307179586476925286766559;
static const double PI = 3.1415926535897932384626433832795;

static inline cd cmul(cd a, cd b) {
    cd r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}

#define MAX_DIRECT_PRIME_F64 64

static void fft_f64_impl(const cd *input, cd *output, size_t n, int sign);

/* bluestein_f64, src/math/mod.rs:366-405. */
static void bluestein_f64(const cd *values, cd *out, size_t n, int sign) {
    cd *chirp = (cd *)malloc(sizeof(cd) * n);
    for (size_t k = 0; k < n; ++k) {
        unsigned __int128 sq = (unsigned __int128)k * k % (2 * (unsigned __int128)n);
        double ang = sign * PI * (double)sq / (double)n;
        chirp[k].re = cos(ang);
        chirp[k].im = sin(ang);
    }
    size_t m = 1;
    while (m < 2 * n - 1) m <<= 1;
    cd *a = (cd *)calloc(m, sizeof(cd));
    cd *b = (cd *)calloc(m, sizeof(cd));
    cd *fa = (cd *)malloc(sizeof(cd) * m);
    cd *fb = (cd *)malloc(sizeof(cd) * m);
    for (size_t k = 0; k < n; ++k) {
        a[k] = cmul(values[k], chirp[k]);
        cd c = {chirp[k].re, -chirp[k].im};
        b[k] = c;
        if (k > 0) b[m - k] = c;
    }
    fft_f64_impl(a, fa, m, -1);
    fft_f64_impl(b, fb, m, -1);
    for (size_t k = 0; k < m; ++k) fa[k] = cmul(fa[k], fb[k]);
    fft_f64_impl(fa, a, m, +1);
    for (size_t k = 0; k < n; ++k) {
        cd v = cmul(a[k], chirp[k]);
        out[k].re = v.re / (double)m;
        out[k].im = v.im / (double)m;
    }
    free(chirp);
    free(a);
    free(b);
    free(fa);
    free(fb);
}

/* fft_f64_recursive, src/math/mod.rs:300-361. */
static void fft_f64_recursive(const cd *input, size_t stride, cd *output, size_t n,
                              const cd *roots, size_t root_stride, int sign) {
    size_t p = n;
    for (size_t f = 2; f * f <= n; ++f) {
        if (n % f == 0) {
            p = f;
            break;
        }
    }
    if (p == n && n > MAX_DIRECT_PRIME_F64) {
        cd *values = (cd *)malloc(sizeof(cd) * n);
        for (size_t j = 0; j < n; ++j) values[j] = input[j * stride];
        bluestein_f64(values, output, n, sign);
        free(values);
        return;
    }
    if (p == n) {
        for (size_t k = 0; k < n; ++k) {
            cd sum = {0.0, 0.0};
            for (size_t j = 0; j < n; ++j) {
                cd t = cmul(input[j * stride], roots[(j * k % n) * root_stride]);
                sum.re += t.re;
                sum.im += t.im;
            }
            output[k] = sum;
        }
        return;
    }
    size_t m = n / p;
    for (size_t r = 0; r < p; ++r)
        fft_f64_recursive(input + r * stride, stride * p, output + r * m, m, roots,
                          root_stride * p, sign);
    cd colbuf[64];
    cd *column = p <= 64 ? colbuf : (cd *)malloc(sizeof(cd) * p);
    for (size_t k = 0; k < m; ++k) {
        for (size_t r = 0; r < p; ++r) column[r] = cmul(output[r * m + k], roots[r * k * root_stride]);
        for (size_t s = 0; s < p; ++s) {
            cd sum = {0.0, 0.0};
            for (size_t r = 0; r < p; ++r) {
                cd t = cmul(column[r], roots[(r * s % p) * m * root_stride]);
                sum.re += t.re;
                sum.im += t.im;
            }
            output[k + m * s] = sum;
        }
    }
    if (column != colbuf) free(column);
}

/* fft_f64, src/math/mod.rs:274-292: roots of unity of the full length, then
 * the recursion.  sign = -1 forward, +1 inverse. */
static void fft_f64_impl(const cd *input, cd *output, size_t n, int sign) {
    if (n <= 1) {
        if (n == 1) output[0] = input[0];
        return;
    }
    cd *roots = (cd *)malloc(sizeof(cd) * n);
    for (size_t k = 0; k < n; ++k) {
        double ang = sign * TAU * (double)k / (double)n;
        roots[k].re = cos(ang);
        roots[k].im = sin(ang);
    }
    fft_f64_recursive(input, 1, output, n, roots, 1, sign);
    free(roots);
}

/* Public: unnormalised DFT of one line, interleaved [re, im] doubles. */
void oracle_fft_f64(const double *in, double *out, uint64_t n, int inverse) {
    fft_f64_impl((const cd *)in, (cd *)out, (size_t)n, inverse ? +1 : -1);
}

static int validate_shape(const uint64_t *shape, int rank, const int32_t *axes, int naxes,
                          uint64_t batch) {
    if (rank <= 0 || naxes <= 0 || batch == 0) return -1;
    for (int i = 0; i < rank; ++i)
        if (shape[i] == 0) return -1;
    for (int i = 0; i < naxes; ++i) {
        if (axes[i] < 0 || axes[i] >= rank) return -1;
        for (int j = 0; j < i; ++j)
            if (axes[j] == axes[i]) return -1;
    }
    return 0;
}

/* FftConfig::scale_f64, src/config.rs:276-286. */
double oracle_scale_f64(uint64_t logical_len, int inverse, int normalization) {
    double len = (double)logical_len;
    switch (normalization) {
    case 0: return 1.0;
    case 1: return inverse ? 1.0 : 1.0 / len;
    case 2: return inverse ? 1.0 / len : 1.0;
    case 3: return 1.0 / sqrt(len);
    default: return 1.0;
    }
}

/* FftConfig::scale (f32 arithmetic), src/config.rs:262-274. */
float oracle_scale_f32(uint64_t logical_len, int inverse, int normalization) {
    float len = (float)logical_len;
    switch (normalization) {
    case 0: return 1.0f;
    case 1: return inverse ? 1.0f : 1.0f / len;
    case 2: return inverse ? 1.0f / len : 1.0f;
    case 3: return 1.0f / sqrtf(len);
    default: return 1.0f;
    }
}

/* line_base_for_axis, src/math/mod.rs:504-516. */
static size_t line_base_for_axis(size_t line, int axis, const uint64_t *shape,
                                 const size_t *strides, int rank) {
    size_t base = 0;
    for (int d = 0; d < rank; ++d) {
        if (d == axis) continue;
        size_t coord = line % shape[d];
        line /= shape[d];
        base += coord * strides[d];
    }
    return base;
}

/* reference_c2c_nd_f64, src/math/mod.rs:214-266.  Lines are independent, so
 * they run on OpenMP threads; each line goes through fft_f64. */
int oracle_c2c_nd_f64(const double *in, double *out, const uint64_t *shape, int rank,
                      const int32_t *axes, int naxes, uint64_t batch, int inverse,
                      int normalization) {
    if (validate_shape(shape, rank, axes, naxes, batch)) return -1;
    size_t strides[16];
    if (rank > 16) return -1;
    size_t logical = 1;
    for (int d = 0; d < rank; ++d) {
        strides[d] = logical;
        logical *= shape[d];
    }
    size_t total = logical * batch;
    double final_scale = oracle_scale_f64(logical, inverse, normalization);
    int sign = inverse ? +1 : -1;
    cd *values = (cd *)malloc(sizeof(cd) * total);
    cd *next = (cd *)malloc(sizeof(cd) * total);
    memcpy(values, in, sizeof(cd) * total);
    for (int ai = 0; ai < naxes; ++ai) {
        int axis = axes[ai];
        size_t axis_len = shape[axis];
        size_t stride = strides[axis];
        size_t lines_per_batch = logical / axis_len;
        double scale = (ai + 1 == naxes) ? final_scale : 1.0;
        size_t nlines = lines_per_batch * batch;
#pragma omp parallel
        {
            cd *line_in = (cd *)malloc(sizeof(cd) * axis_len);
            cd *line_out = (cd *)malloc(sizeof(cd) * axis_len);
#pragma omp for schedule(dynamic, 16)
            for (size_t li = 0; li < nlines; ++li) {
                size_t b = li / lines_per_batch, line = li % lines_per_batch;
                size_t base = b * logical + line_base_for_axis(line, axis, shape, strides, rank);
                for (size_t n = 0; n < axis_len; ++n) line_in[n] = values[base + n * stride];
                fft_f64_impl(line_in, line_out, axis_len, sign);
                for (size_t k = 0; k < axis_len; ++k) {
                    next[base + k * stride].re = line_out[k].re * scale;
                    next[base + k * stride].im = line_out[k].im * scale;
                }
            }
            free(line_in);
            free(line_out);
        }
        cd *t = values;
        values = next;
        next = t;
    }
    memcpy(out, values, sizeof(cd) * total);
    free(values);
    free(next);
    return 0;
}

/* reference_c2c_nd, src/math/mod.rs:155-208: the f32 plain DFT, computed
 * in float exactly as the reference writes it (angle, sin_cos, sums and
 * scale all in f32).  O(N^2) per line: known-answer tests only. */
int oracle_c2c_nd_dft_f32(const float *in, float *out, const uint64_t *shape, int rank,
                          const int32_t *axes, int naxes, uint64_t batch, int inverse,
                          int normalization) {
    if (validate_shape(shape, rank, axes, naxes, batch)) return -1;
    size_t strides[16];
    if (rank > 16) return -1;
    size_t logical = 1;
    for (int d = 0; d < rank; ++d) {
        strides[d] = logical;
        logical *= shape[d];
    }
    size_t total = logical * batch;
    float sign = inverse ? 1.0f : -1.0f;
    const float tau = 6.28318530717958647692f;
    float final_scale = oracle_scale_f32(logical, inverse, normalization);
    float *values = (float *)malloc(sizeof(float) * 2 * total);
    float *next = (float *)malloc(sizeof(float) * 2 * total);
    memcpy(values, in, sizeof(float) * 2 * total);
    for (int ai = 0; ai < naxes; ++ai) {
        int axis = axes[ai];
        size_t axis_len = shape[axis];
        float axis_len_f = (float)axis_len;
        size_t stride = strides[axis];
        size_t lines_per_batch = logical / axis_len;
        float scale = (ai + 1 == naxes) ? final_scale : 1.0f;
        for (size_t b = 0; b < batch; ++b) {
            for (size_t line = 0; line < lines_per_batch; ++line) {
                size_t base = b * logical + line_base_for_axis(line, axis, shape, strides, rank);
                for (size_t k = 0; k < axis_len; ++k) {
                    float sre = 0.0f, sim = 0.0f;
                    for (size_t n = 0; n < axis_len; ++n) {
                        float vre = values[2 * (base + n * stride)];
                        float vim = values[2 * (base + n * stride) + 1];
                        float angle = sign * tau * (float)k * (float)n / axis_len_f;
                        float s = sinf(angle), c = cosf(angle);
                        sre += vre * c - vim * s;
                        sim += vre * s + vim * c;
                    }
                    next[2 * (base + k * stride)] = sre * scale;
                    next[2 * (base + k * stride) + 1] = sim * scale;
                }
            }
        }
        float *t = values;
        values = next;
        next = t;
    }
    memcpy(out, values, sizeof(float) * 2 * total);
    free(values);
    free(next);
    return 0;
}

/* packed_coords_for_full_spectrum / is_self_conjugate_bin,
 * src/math/mod.rs:466-502. */
static void coords_from_linear(size_t index, const uint64_t *shape, const size_t *strides,
                               int rank, size_t *coords) {
    for (int d = rank - 1; d >= 0; --d) {
        coords[d] = index / strides[d];
        index %= strides[d];
    }
}

static int is_self_conjugate_bin(const size_t *coords, const uint64_t *shape, int rank) {
    size_t x = coords[0];
    int even_x = shape[0] % 2 == 0;
    if (!(x == 0 || (even_x && x == shape[0] / 2))) return 0;
    for (int d = 1; d < rank; ++d) {
        if (shape[d] % 2 == 0) {
            if (coords[d] != 0 && coords[d] != shape[d] / 2) return 0;
        } else if (coords[d] != 0) {
            return 0;
        }
    }
    return 1;
}

/* reference_r2c_packed_interleaved, src/math/mod.rs:81-113, through the FP64
 * transform: real input -> packed [N0/2+1, N1, ...] interleaved complex. */
int oracle_r2c_packed_f64(const double *real, double *packed, const uint64_t *shape, int rank,
                          uint64_t batch, int normalization) {
    int32_t axes[16];
    if (rank > 16 || rank <= 0) return -1;
    for (int d = 0; d < rank; ++d) axes[d] = d;
    size_t logical = 1;
    for (int d = 0; d < rank; ++d) logical *= shape[d];
    size_t total = logical * batch;
    double *full_in = (double *)calloc(2 * total, sizeof(double));
    double *full = (double *)malloc(sizeof(double) * 2 * total);
    for (size_t i = 0; i < total; ++i) full_in[2 * i] = real[i];
    int rc = oracle_c2c_nd_f64(full_in, full, shape, rank, axes, rank, batch, 0, normalization);
    if (rc) {
        free(full_in);
        free(full);
        return rc;
    }
    uint64_t pshape[16];
    size_t pstrides[16], fstrides[16], coords[16];
    size_t plogical = 1, flogical = 1;
    for (int d = 0; d < rank; ++d) {
        pshape[d] = d == 0 ? shape[0] / 2 + 1 : shape[d];
        pstrides[d] = plogical;
        fstrides[d] = flogical;
        plogical *= pshape[d];
        flogical *= shape[d];
    }
    for (size_t b = 0; b < batch; ++b) {
        for (size_t pi = 0; pi < plogical; ++pi) {
            coords_from_linear(pi, pshape, pstrides, rank, coords);
            size_t fi = 0;
            for (int d = 0; d < rank; ++d) fi += coords[d] * fstrides[d];
            packed[2 * (b * plogical + pi)] = full[2 * (b * flogical + fi)];
            packed[2 * (b * plogical + pi) + 1] = full[2 * (b * flogical + fi) + 1];
        }
    }
    free(full_in);
    free(full);
    return 0;
}

/* reference_c2r_from_packed_interleaved, src/math/mod.rs:115-153, through
 * the FP64 transform: Hermitian mirror of the packed half (conjugate for
 * x >= N0/2+1, imaginary part zeroed on self-conjugate bins), inverse C2C,
 * real part. */
int oracle_c2r_from_packed_f64(const double *packed, double *real, const uint64_t *shape, int rank,
                               uint64_t batch, int normalization) {
    int32_t axes[16];
    if (rank > 16 || rank <= 0) return -1;
    for (int d = 0; d < rank; ++d) axes[d] = d;
    uint64_t pshape[16];
    size_t pstrides[16], fstrides[16], coords[16], pcoords[16];
    size_t plogical = 1, flogical = 1;
    for (int d = 0; d < rank; ++d) {
        pshape[d] = d == 0 ? shape[0] / 2 + 1 : shape[d];
        pstrides[d] = plogical;
        fstrides[d] = flogical;
        plogical *= pshape[d];
        flogical *= shape[d];
    }
    size_t total = flogical * batch;
    double *full = (double *)malloc(sizeof(double) * 2 * total);
    double *inv = (double *)malloc(sizeof(double) * 2 * total);
    for (size_t b = 0; b < batch; ++b) {
        for (size_t fi = 0; fi < flogical; ++fi) {
            coords_from_linear(fi, shape, fstrides, rank, coords);
            size_t x = coords[0];
            int mirrored = x >= pshape[0];
            pcoords[0] = mirrored ? shape[0] - x : x;
            for (int d = 1; d < rank; ++d)
                pcoords[d] = (mirrored && coords[d] != 0) ? shape[d] - coords[d] : coords[d];
            size_t pi = 0;
            for (int d = 0; d < rank; ++d) pi += pcoords[d] * pstrides[d];
            double re = packed[2 * (b * plogical + pi)];
            double im = packed[2 * (b * plogical + pi) + 1];
            if (mirrored) im = -im;
            if (is_self_conjugate_bin(coords, shape, rank)) im = 0.0;
            full[2 * (b * flogical + fi)] = re;
            full[2 * (b * flogical + fi) + 1] = im;
        }
    }
    int rc = oracle_c2c_nd_f64(full, inv, shape, rank, axes, rank, batch, 1, normalization);
    if (!rc)
        for (size_t i = 0; i < total; ++i) real[i] = inv[2 * i];
    free(full);
    free(inv);
    return rc;
}

/* Df64 storage helpers (src/math/double_float.rs:22-33, src/cpu.rs:489-517):
 * each complex value is [re_hi, re_lo, im_hi, im_lo] f32 words with
 * hi = f32(x), lo = f32(x - hi). */
void oracle_df64_split(const double *values, float *words, uint64_t count) {
    for (uint64_t i = 0; i < count; ++i) {
        double v = values[i];
        float hi = (float)v;
        float lo = isfinite(hi) ? (float)(v - (double)hi) : 0.0f;
        words[2 * i] = hi;
        words[2 * i + 1] = lo;
    }
}

void oracle_df64_join(const float *words, double *values, uint64_t count) {
    for (uint64_t i = 0; i < count; ++i) values[i] = (double)words[2 * i] + (double)words[2 * i + 1];
}

/* Integer helpers restating src/runtime/axis_policy.rs:84-160 and
 * src/runtime/mod.rs:30-57 (used to check the planner's decisions). */
int oracle_is_prime(uint64_t n) {
    if (n < 2) return 0;
    if (n % 2 == 0) return n == 2;
    for (uint64_t d = 3; d <= n / d; d += 2)
        if (n % d == 0) return 0;
    return 1;
}

static uint64_t mod_pow(uint64_t base, uint64_t exp, uint64_t modulus) {
    uint64_t result = 1;
    base %= modulus;
    while (exp > 0) {
        if (exp & 1) result = (unsigned __int128)result * base % modulus;
        base = (unsigned __int128)base * base % modulus;
        exp >>= 1;
    }
    return result;
}

uint64_t oracle_primitive_root(uint64_t prime) {
    if (!oracle_is_prime(prime)) return 0;
    if (prime == 2) return 1;
    uint64_t phi = prime - 1, factors[64];
    int nf = 0;
    uint64_t n = phi;
    for (uint64_t d = 2; d <= n / d; d += (d == 2 ? 1 : 2)) {
        if (n % d == 0) {
            factors[nf++] = d;
            while (n % d == 0) n /= d;
        }
    }
    if (n > 1) factors[nf++] = n;
    for (uint64_t root = 2; root < prime; ++root) {
        int ok = 1;
        for (int i = 0; i < nf; ++i)
            if (mod_pow(root, phi / factors[i], prime) == 1) {
                ok = 0;
                break;
            }
        if (ok) return root;
    }
    return 0;
}

/* factor_supported_length, src/runtime/mod.rs:34-57: greedy over
 * 13, 11, 8, 7, 5, 4, 3, 2.  Returns the factor count, or -1 when the length
 * has another prime factor. */
int oracle_factor_supported_length(uint64_t len, uint32_t *factors, int cap) {
    static const uint32_t order[] = {13, 11, 8, 7, 5, 4, 3, 2};
    if (len == 0) return -1;
    int count = 0;
    while (len > 1) {
        int found = 0;
        for (int i = 0; i < 8; ++i) {
            if (len % order[i] == 0) {
                if (count < cap) factors[count] = order[i];
                ++count;
                len /= order[i];
                found = 1;
                break;
            }
        }
        if (!found) return -1;
    }
    return count;
}

/* Rader input order (src/runtime/rader_axis.rs:1291-1304):
 * perm[k] = g^(k+1) mod p for k < p-1, g the smallest primitive root. */
int oracle_rader_permutation(uint64_t p, uint32_t *perm) {
    uint64_t g = oracle_primitive_root(p);
    if (!g) return -1;
    uint64_t v = 1;
    for (uint64_t k = 0; k + 1 < p; ++k) {
        v = v * g % p;
        perm[k] = (uint32_t)v;
    }
    return 0;
}
