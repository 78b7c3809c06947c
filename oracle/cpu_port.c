/*
 * Planned CPU FFT used as the CPU baseline of the benchmark.
 *
 * TEST AND CPU-BASELINE INFRASTRUCTURE ONLY: the product never links or calls it.
 *
 * The reference's CPU backend, CpuFftPlan (src/cpu.rs:52-330), cannot be
 * built here: it sits on the third-party crates rustfft 6.4.1 and realfft
 * 3.5.0 (Cargo.lock), and no Rust toolchain is present.  This file restates
 * its structure in C:
 *   - a plan is made once per line length (CpuFftPlan::c2c, src/cpu.rs:90-118),
 *     holding FP64-generated twiddles rounded once to the working type;
 *   - lines are transformed axis by axis, strided axes gathered into a
 *     contiguous line first (transform_axes / transform_strided,
 *     src/cpu.rs:429-442, 557), lines spread over threads
 *     (for_each_chunk_group, src/cpu.rs:822-842), scale last (scale_all, 801);
 * and uses rustfft's published algorithm family: mixed-radix Stockham for
 * 2/3/4/5/7/11/13-smooth lengths, Bluestein over a power of two otherwise.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#define REAL float
#define SFX f32
#include "cpu_port_impl.h"
#undef REAL
#undef SFX

#define REAL double
#define SFX f64
#include "cpu_port_impl.h"
#undef REAL
#undef SFX

static float scale_f32(uint64_t logical, int inverse, int normalization) {
    float len = (float)logical;
    switch (normalization) {
    case 0: return 1.0f;
    case 1: return inverse ? 1.0f : 1.0f / len;
    case 2: return inverse ? 1.0f / len : 1.0f;
    case 3: return 1.0f / sqrtf(len);
    default: return 1.0f;
    }
}

static size_t line_base(size_t line, int axis, const uint64_t *shape, const size_t *strides,
                        int rank) {
    size_t base = 0;
    for (int d = 0; d < rank; ++d) {
        if (d == axis) continue;
        base += (line % shape[d]) * strides[d];
        line /= shape[d];
    }
    return base;
}

/* C2C f32 over an N-D shape (axis 0 contiguous), in place on `data`. */
int cpu_port_c2c_f32(float *data, const uint64_t *shape, int rank, const int32_t *axes,
                     int naxes, uint64_t batch, int inverse, int normalization, int threads) {
    if (rank <= 0 || rank > 16 || naxes <= 0) return -1;
    size_t strides[16], logical = 1;
    for (int d = 0; d < rank; ++d) {
        strides[d] = logical;
        logical *= shape[d];
    }
    int sign = inverse ? +1 : -1;
    cpx_f32 *v = (cpx_f32 *)data;
    if (threads > 0) omp_set_num_threads(threads);
    for (int ai = 0; ai < naxes; ++ai) {
        int axis = axes[ai];
        size_t len = shape[axis], stride = strides[axis];
        size_t lines = logical / len * batch, per_batch = logical / len;
        lineplan_f32 *plan = lineplan_new_f32(len, sign);
#pragma omp parallel
        {
            cpx_f32 *line = (cpx_f32 *)malloc(sizeof(cpx_f32) * len);
            cpx_f32 *work = (cpx_f32 *)malloc(sizeof(cpx_f32) * len);
#pragma omp for schedule(static)
            for (size_t li = 0; li < lines; ++li) {
                size_t base = (li / per_batch) * logical +
                              line_base(li % per_batch, axis, shape, strides, rank);
                if (stride == 1) {
                    lineplan_exec_f32(plan, v + base, work);
                } else {
                    for (size_t n = 0; n < len; ++n) line[n] = v[base + n * stride];
                    lineplan_exec_f32(plan, line, work);
                    for (size_t n = 0; n < len; ++n) v[base + n * stride] = line[n];
                }
            }
            free(line);
            free(work);
        }
        lineplan_free_f32(plan);
    }
    float s = scale_f32(logical, inverse, normalization);
    if (s != 1.0f) {
        size_t total = logical * batch * 2;
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < total; ++i) data[i] *= s;
    }
    return 0;
}

/* A set of planned lines of mixed lengths, each contiguous in one buffer:
 * the CPU counterpart of the batched mixed-length launch. */
typedef struct {
    uint64_t nlines;
    uint64_t *offsets;  /* complex units */
    uint64_t *lengths;
    uint32_t *plan_of;  /* index into plans */
    lineplan_f32 **plans;
    uint64_t nplans;
    uint64_t max_len;
    int inverse, normalization;
} cpu_lines_f32;

void *cpu_port_lines_new_f32(const uint64_t *offsets, const uint64_t *lengths, uint64_t nlines,
                             int inverse, int normalization) {
    cpu_lines_f32 *s = (cpu_lines_f32 *)calloc(1, sizeof(cpu_lines_f32));
    s->nlines = nlines;
    s->inverse = inverse;
    s->normalization = normalization;
    s->offsets = (uint64_t *)malloc(8 * nlines);
    s->lengths = (uint64_t *)malloc(8 * nlines);
    s->plan_of = (uint32_t *)malloc(4 * nlines);
    memcpy(s->offsets, offsets, 8 * nlines);
    memcpy(s->lengths, lengths, 8 * nlines);
    /* plan cache keyed by length: sort unique lengths */
    uint64_t *uniq = (uint64_t *)malloc(8 * nlines);
    uint64_t nu = 0;
    for (uint64_t i = 0; i < nlines; ++i) {
        uint64_t lo = 0, hi = nu;
        while (lo < hi) {
            uint64_t mid = (lo + hi) / 2;
            if (uniq[mid] < lengths[i]) lo = mid + 1;
            else hi = mid;
        }
        if (lo == nu || uniq[lo] != lengths[i]) {
            memmove(uniq + lo + 1, uniq + lo, 8 * (nu - lo));
            uniq[lo] = lengths[i];
            ++nu;
        }
    }
    s->nplans = nu;
    s->plans = (lineplan_f32 **)malloc(sizeof(void *) * nu);
    int sign = inverse ? +1 : -1;
#pragma omp parallel for schedule(dynamic, 1)
    for (uint64_t u = 0; u < nu; ++u) s->plans[u] = lineplan_new_f32(uniq[u], sign);
    for (uint64_t i = 0; i < nlines; ++i) {
        uint64_t lo = 0, hi = nu;
        while (lo < hi) {
            uint64_t mid = (lo + hi) / 2;
            if (uniq[mid] < lengths[i]) lo = mid + 1;
            else hi = mid;
        }
        s->plan_of[i] = (uint32_t)lo;
        if (lengths[i] > s->max_len) s->max_len = lengths[i];
    }
    free(uniq);
    return s;
}

/* Transforms lines [first, first+count) of the set in place. */
int cpu_port_lines_exec_f32(void *handle, float *data, uint64_t first, uint64_t count,
                            int threads) {
    cpu_lines_f32 *s = (cpu_lines_f32 *)handle;
    cpx_f32 *v = (cpx_f32 *)data;
    if (threads > 0) omp_set_num_threads(threads);
    if (first + count > s->nlines) return -1;
#pragma omp parallel
    {
        cpx_f32 *work = (cpx_f32 *)malloc(sizeof(cpx_f32) * (s->max_len ? s->max_len : 1));
#pragma omp for schedule(dynamic, 1)
        for (uint64_t i = first; i < first + count; ++i) {
            cpx_f32 *line = v + s->offsets[i];
            lineplan_exec_f32(s->plans[s->plan_of[i]], line, work);
            float sc = scale_f32(s->lengths[i], s->inverse, s->normalization);
            if (sc != 1.0f)
                for (uint64_t n = 0; n < s->lengths[i]; ++n) {
                    line[n].re *= sc;
                    line[n].im *= sc;
                }
        }
        free(work);
    }
    return 0;
}

void cpu_port_lines_free_f32(void *handle) {
    cpu_lines_f32 *s = (cpu_lines_f32 *)handle;
    if (!s) return;
    for (uint64_t u = 0; u < s->nplans; ++u) lineplan_free_f32(s->plans[u]);
    free(s->plans);
    free(s->offsets);
    free(s->lengths);
    free(s->plan_of);
    free(s);
}

int cpu_port_max_threads(void) { return omp_get_max_threads(); }

/* f64 line transform (used to cross-check the oracle on long lines). */
int cpu_port_line_f64(double *data, uint64_t n, int inverse) {
    lineplan_f64 *p = lineplan_new_f64(n, inverse ? +1 : -1);
    cpx_f64 *work = (cpx_f64 *)malloc(sizeof(cpx_f64) * n);
    lineplan_exec_f64(p, (cpx_f64 *)data, work);
    free(work);
    lineplan_free_f64(p);
    return 0;
}
