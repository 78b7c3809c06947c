/*
 * Body of the planned CPU FFT, instantiated for float and double by
 * cpu_port.c (REAL, SFX set before inclusion).  TEST AND CPU-BASELINE
 * INFRASTRUCTURE ONLY: see cpu_port.c.
 */
#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define CPX CAT(cpx_, SFX)
#define LPLAN CAT(lineplan_, SFX)

typedef struct {
    REAL re, im;
} CPX;

typedef struct LPLAN {
    size_t n;
    int sign;
    int nstages;
    int radix[64];
    size_t ns[64];      /* sub-length before the stage */
    CPX *tw[64];        /* per stage: tw[k*(R-1) + q-1] = W_{ns*R}^{q k} */
    CPX *roots[64];     /* per stage: W_R^{m}, m < R */
    /* Bluestein */
    int bluestein;
    size_t m;
    CPX *chirp;         /* n entries */
    CPX *bhat;          /* m entries, already divided by m */
    struct LPLAN *inner_f, *inner_i;
} LPLAN;

static void CAT(lineplan_free_, SFX)(LPLAN *p) {
    if (!p) return;
    for (int s = 0; s < p->nstages; ++s) {
        free(p->tw[s]);
        free(p->roots[s]);
    }
    free(p->chirp);
    free(p->bhat);
    CAT(lineplan_free_, SFX)(p->inner_f);
    CAT(lineplan_free_, SFX)(p->inner_i);
    free(p);
}

static void CAT(lineplan_exec_, SFX)(const LPLAN *p, CPX *data, CPX *work);

static LPLAN *CAT(lineplan_new_, SFX)(size_t n, int sign) {
    LPLAN *p = (LPLAN *)calloc(1, sizeof(LPLAN));
    p->n = n;
    p->sign = sign;
    size_t rem = n;
    int ok = 1;
    while (rem > 1) {
        int r = 0;
        if (rem % 4 == 0) r = 4;
        else if (rem % 2 == 0) r = 2;
        else if (rem % 3 == 0) r = 3;
        else if (rem % 5 == 0) r = 5;
        else if (rem % 7 == 0) r = 7;
        else if (rem % 11 == 0) r = 11;
        else if (rem % 13 == 0) r = 13;
        else {
            ok = 0;
            break;
        }
        p->radix[p->nstages++] = r;
        rem /= (size_t)r;
    }
    if (!ok) {
        p->nstages = 0;
        p->bluestein = 1;
        size_t m = 1;
        while (m < 2 * n - 1) m <<= 1;
        p->m = m;
        p->chirp = (CPX *)malloc(sizeof(CPX) * n);
        CPX *b = (CPX *)calloc(m, sizeof(CPX));
        for (size_t k = 0; k < n; ++k) {
            unsigned __int128 sq = (unsigned __int128)k * k % (2 * (unsigned __int128)n);
            double ang = sign * 3.14159265358979323846 * (double)sq / (double)n;
            p->chirp[k].re = (REAL)cos(ang);
            p->chirp[k].im = (REAL)sin(ang);
            b[k].re = (REAL)cos(ang);
            b[k].im = (REAL)-sin(ang);
            if (k) b[m - k] = b[k];
        }
        p->inner_f = CAT(lineplan_new_, SFX)(m, -1);
        p->inner_i = CAT(lineplan_new_, SFX)(m, +1);
        CPX *w = (CPX *)malloc(sizeof(CPX) * m);
        CAT(lineplan_exec_, SFX)(p->inner_f, b, w);
        for (size_t k = 0; k < m; ++k) {
            b[k].re /= (REAL)m;
            b[k].im /= (REAL)m;
        }
        p->bhat = b;
        free(w);
        return p;
    }
    size_t ns = 1;
    for (int s = 0; s < p->nstages; ++s) {
        int r = p->radix[s];
        p->ns[s] = ns;
        p->tw[s] = (CPX *)malloc(sizeof(CPX) * ns * (size_t)(r - 1) + sizeof(CPX));
        for (size_t k = 0; k < ns; ++k)
            for (int q = 1; q < r; ++q) {
                double ang = sign * 6.283185307179586 * (double)(q * k) / (double)(ns * r);
                p->tw[s][k * (r - 1) + q - 1].re = (REAL)cos(ang);
                p->tw[s][k * (r - 1) + q - 1].im = (REAL)sin(ang);
            }
        p->roots[s] = (CPX *)malloc(sizeof(CPX) * r);
        for (int m = 0; m < r; ++m) {
            double ang = sign * 6.283185307179586 * m / r;
            p->roots[s][m].re = (REAL)cos(ang);
            p->roots[s][m].im = (REAL)sin(ang);
        }
        ns *= (size_t)r;
    }
    return p;
}

/* Stockham autosort: ping-pong between data and work; result in data. */
static void CAT(lineplan_exec_, SFX)(const LPLAN *p, CPX *data, CPX *work) {
    size_t n = p->n;
    if (p->bluestein) {
        size_t m = p->m;
        CPX *a = (CPX *)calloc(m, sizeof(CPX));
        CPX *w = (CPX *)malloc(sizeof(CPX) * m);
        for (size_t k = 0; k < n; ++k) {
            CPX x = data[k], c = p->chirp[k];
            a[k].re = x.re * c.re - x.im * c.im;
            a[k].im = x.re * c.im + x.im * c.re;
        }
        CAT(lineplan_exec_, SFX)(p->inner_f, a, w);
        for (size_t k = 0; k < m; ++k) {
            CPX x = a[k], c = p->bhat[k];
            a[k].re = x.re * c.re - x.im * c.im;
            a[k].im = x.re * c.im + x.im * c.re;
        }
        CAT(lineplan_exec_, SFX)(p->inner_i, a, w);
        for (size_t k = 0; k < n; ++k) {
            CPX x = a[k], c = p->chirp[k];
            data[k].re = x.re * c.re - x.im * c.im;
            data[k].im = x.re * c.im + x.im * c.re;
        }
        free(a);
        free(w);
        return;
    }
    CPX *src = data, *dst = work;
    for (int s = 0; s < p->nstages; ++s) {
        int r = p->radix[s];
        size_t ns = p->ns[s];
        size_t stride = n / (size_t)r;
        const CPX *tw = p->tw[s];
        const CPX *rt = p->roots[s];
        for (size_t j = 0; j < stride; ++j) {
            size_t k = j % ns;
            CPX v[13];
            for (int q = 0; q < r; ++q) {
                CPX x = src[j + (size_t)q * stride];
                if (q && ns > 1) {
                    CPX t = tw[k * (r - 1) + q - 1];
                    CPX y = {x.re * t.re - x.im * t.im, x.re * t.im + x.im * t.re};
                    x = y;
                }
                v[q] = x;
            }
            size_t ob = (j - k) * (size_t)r + k;
            if (r == 2) {
                CPX a = v[0], b = v[1];
                dst[ob].re = a.re + b.re;
                dst[ob].im = a.im + b.im;
                dst[ob + ns].re = a.re - b.re;
                dst[ob + ns].im = a.im - b.im;
            } else if (r == 4) {
                CPX a0 = {v[0].re + v[2].re, v[0].im + v[2].im};
                CPX a1 = {v[0].re - v[2].re, v[0].im - v[2].im};
                CPX a2 = {v[1].re + v[3].re, v[1].im + v[3].im};
                CPX a3 = {v[1].re - v[3].re, v[1].im - v[3].im};
                /* multiply a3 by sign*i */
                CPX b3 = {-p->sign * a3.im, p->sign * a3.re};
                dst[ob].re = a0.re + a2.re;
                dst[ob].im = a0.im + a2.im;
                dst[ob + ns].re = a1.re + b3.re;
                dst[ob + ns].im = a1.im + b3.im;
                dst[ob + 2 * ns].re = a0.re - a2.re;
                dst[ob + 2 * ns].im = a0.im - a2.im;
                dst[ob + 3 * ns].re = a1.re - b3.re;
                dst[ob + 3 * ns].im = a1.im - b3.im;
            } else {
                for (int o = 0; o < r; ++o) {
                    REAL sre = 0, sim = 0;
                    for (int q = 0; q < r; ++q) {
                        CPX t = rt[(o * q) % r];
                        sre += v[q].re * t.re - v[q].im * t.im;
                        sim += v[q].re * t.im + v[q].im * t.re;
                    }
                    dst[ob + (size_t)o * ns].re = sre;
                    dst[ob + (size_t)o * ns].im = sim;
                }
            }
        }
        CPX *t = src;
        src = dst;
        dst = t;
    }
    if (src != data) memcpy(data, src, sizeof(CPX) * n);
}

#undef CPX
#undef LPLAN
#undef CAT
#undef CAT_
