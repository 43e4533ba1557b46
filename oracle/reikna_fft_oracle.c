/*
 * CPU oracle: a restatement of reikna's FFT hot path in C (gcc -O3 -fopenmp).
 *
 * TEST INFRASTRUCTURE ONLY.  It is used by tests/ to check the CUDA library, by
 * __graft_entry__.smoke() as the checker, and by bench.py as the timed CPU baseline
 * of the reference algorithm.  Nothing in reikna_b200/ links, loads or calls it.
 *
 * What it restates (file:line inside fjarri/reikna):
 *   rko_radix_array        get_radix_array           reikna/fft/fft.py:24-86
 *   rko_global_radix_info  get_global_radix_info     reikna/fft/fft.py:89-146
 *   rko_kweights           get_kweights              reikna/fft/fft.py:216-236
 *   rko_plan_create        get_fft_kernels / get_fft_1d_kernels / LocalFFTKernel /
 *                          GlobalFFTKernel.create_chain   reikna/fft/fft.py:253-584
 *   run_kernel (body)      fft_local / fft_global    reikna/fft/fft.mako:750-1038
 *                          butterflies fftKernel2..16 fft.mako:48-163, twiddles
 *                          fft.mako:636-649 and 933-947, xweight fft.mako:196-202,
 *                          normalisation fft.mako:747
 * The arithmetic follows reikna's operation order in the working precision (FP32
 * sin/cos of FP32 angles for complex64), so its results carry reikna's rounding
 * behaviour; the data movement through local memory is replaced by plain indexing
 * into the same Stockham positions.
 *
 * Parity is pinned against numpy.fft (which reikna's own tests use as the reference,
 * tests/test_fft/test_fft.py:148-170) and against golden fixtures of reikna's planner
 * functions generated by tests/golden/make_golden.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define RKO_LOCAL 0
#define RKO_GLOBAL 1
#define RKO_MAXK 64
#define MAX_RADIX 16

typedef struct {
    int kind;
    int axis;
    int64_t outer, inner;
    int64_t fft_size, fft_size_real, in_len;
    int reverse_direction, pad_in, takes_kweights, unpad_out, normalize, last_pass, pass_num;
    int nradix;
    int radix[16];
    int radix1, radix2;
    int64_t stride_out, curr_size;
    int kw_index;
} rko_kernel;

typedef struct {
    int ndim;
    int64_t shape[8];
    int nk;
    rko_kernel k[RKO_MAXK];
    int nkw;
    double* kw[8][2]; /* interleaved re/im rows */
} rko_plan;

/* helpers.log2 / min_blocks / bounding_power_of_2 (reikna/helpers.py:92-118) */
static int ilog2(int64_t n) {
    int p = 0;
    while (((int64_t)1 << (p + 1)) <= n) ++p;
    return p;
}
static int64_t min_blocks(int64_t len, int64_t block) { return (len - 1) / block + 1; }
static int64_t bpow2(int64_t n) {
    if (n == 1) return 1;
    return (int64_t)1 << (ilog2(n - 1) + 1);
}

int rko_radix_array(int size, int use_max_radix, int* out) {
    if (size <= 0 || (size & (size - 1))) return -1;
    int n = 0;
    if (use_max_radix) {
        const int radix = size < MAX_RADIX ? size : MAX_RADIX;
        while (size > radix) {
            out[n++] = radix;
            size /= radix;
        }
        out[n++] = size;
        return n;
    }
    switch (size) {
        case 2: out[0] = 2; return 1;
        case 4: out[0] = 4; return 1;
        case 8: out[0] = 8; return 1;
        case 16: out[0] = 8; out[1] = 2; return 2;
        case 32: out[0] = 8; out[1] = 4; return 2;
        case 64: out[0] = 8; out[1] = 8; return 2;
        case 128: out[0] = 8; out[1] = 4; out[2] = 4; return 3;
        case 256: out[0] = 4; out[1] = 4; out[2] = 4; out[3] = 4; return 4;
        case 512: out[0] = 8; out[1] = 8; out[2] = 8; return 3;
        case 1024: out[0] = 16; out[1] = 16; out[2] = 4; return 3;
        case 2048: out[0] = 8; out[1] = 8; out[2] = 8; out[3] = 4; return 4;
    }
    const int lsize = ilog2(size);
    const int ne = (int)min_blocks(lsize, 4);
    for (int i = 0; i < ne - 1; ++i) out[n++] = 16;
    out[n++] = (lsize % 4 == 0) ? 16 : (1 << (lsize % 4));
    return n;
}

int rko_global_radix_info(int64_t size, int* radix, int* radix1, int* radix2) {
    if (size <= 0 || (size & (size - 1))) return -1;
    const int64_t base = size < 128 ? size : 128;
    int n = 0;
    while (size > base) {
        size /= base;
        radix[n++] = (int)base;
    }
    radix[n++] = (int)size;
    for (int i = 0; i < n; ++i) {
        const int r = radix[i];
        if (r <= 8) {
            radix1[i] = r;
            radix2[i] = 1;
        } else {
            int r1 = 2, r2 = r / r1;
            while (r2 > r1) {
                r1 *= 2;
                r2 = r / r1;
            }
            radix1[i] = r1;
            radix2[i] = r2;
        }
    }
    return n;
}

/* plain double-precision FFT used for the Bluestein kernel weights (numpy.fft
 * role in get_kweights); sign = -1 forward, +1 inverse (unnormalised) */
static void dfft(double* re, double* im, int64_t n, int sign) {
    for (int64_t i = 1, j = 0; i < n; ++i) {
        int64_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
    }
    for (int64_t len = 2; len <= n; len <<= 1) {
        for (int64_t k = 0; k < len / 2; ++k) {
            const double a = sign * 2.0 * M_PI * (double)k / (double)len;
            const double wr = cos(a), wi = sin(a);
            for (int64_t i = 0; i < n; i += len) {
                const int64_t u = i + k, v = i + k + len / 2;
                const double xr = re[v] * wr - im[v] * wi, xi = re[v] * wi + im[v] * wr;
                re[v] = re[u] - xr; im[v] = im[u] - xi;
                re[u] += xr; im[u] += xi;
            }
        }
    }
}

/* get_kweights: out[row][2*p] (re), out[row][2*p+1] (im); rows 0 and 1 */
int rko_kweights(int64_t nr, int64_t m, double* out0, double* out1) {
    double *re = (double*)malloc(m * sizeof(double)), *im = (double*)malloc(m * sizeof(double));
    if (!re || !im) return -1;
    for (int row = 0; row < 2; ++row) {
        const double sgn = row == 0 ? 1.0 : -1.0;
        for (int64_t p = 0; p < m; ++p) {
            const int64_t nv = p <= m - nr ? p : m - p; /* [0..M-N] ++ [N-1..1] */
            const double arg = sgn * (M_PI / (double)nr) * ((double)nv * (double)nv);
            re[p] = cos(arg);
            im[p] = sin(arg);
        }
        dfft(re, im, m, row == 0 ? -1 : 1);
        double* o = row == 0 ? out0 : out1;
        const double sc = row == 0 ? 1.0 : (1.0 / (double)m) * (double)m / (double)nr;
        for (int64_t p = 0; p < m; ++p) {
            o[2 * p] = re[p] * sc;
            o[2 * p + 1] = im[p] * sc;
        }
    }
    free(re);
    free(im);
    return 0;
}

static int add_kernel(rko_plan* pl, const rko_kernel* k) {
    if (pl->nk >= RKO_MAXK) return -1;
    pl->k[pl->nk++] = *k;
    return 0;
}

static int add_kw(rko_plan* pl, int64_t nr, int64_t m) {
    if (pl->nkw >= 8) return -1;
    const int idx = pl->nkw++;
    pl->kw[idx][0] = (double*)malloc(2 * m * sizeof(double));
    pl->kw[idx][1] = (double*)malloc(2 * m * sizeof(double));
    if (!pl->kw[idx][0] || !pl->kw[idx][1]) return -1;
    rko_kweights(nr, m, pl->kw[idx][0], pl->kw[idx][1]);
    return idx;
}

/* get_fft_1d_kernels (fft.py:487-529) */
static int fft_1d(rko_plan* pl, int axis, int64_t outer, int64_t n, int64_t inner, int64_t local_limit, int reverse,
                  int64_t nr) {
    rko_kernel k;
    memset(&k, 0, sizeof(k));
    k.axis = axis;
    k.outer = outer;
    k.inner = inner;
    k.fft_size = n;
    k.fft_size_real = nr;
    k.reverse_direction = reverse;
    k.kw_index = -1;
    const int padded = n != nr;
    if (inner == 1 && n / MAX_RADIX <= local_limit) {
        k.kind = RKO_LOCAL;
        k.nradix = rko_radix_array((int)n, 0, k.radix);
        if (n / k.radix[0] > local_limit) k.nradix = rko_radix_array((int)n, 1, k.radix);
        k.pad_in = padded && !reverse;
        k.unpad_out = padded && reverse;
        k.takes_kweights = padded && reverse;
        k.normalize = 1;
        k.last_pass = 1;
        k.in_len = k.pad_in ? nr : n;
        if (k.takes_kweights) k.kw_index = add_kw(pl, nr, n);
        return add_kernel(pl, &k);
    }
    int radix[16], r1[16], r2[16];
    const int np = rko_global_radix_info(n, radix, r1, r2);
    int64_t curr = n, so = 1;
    for (int p = 0; p < np; ++p) {
        rko_kernel g = k;
        g.kind = RKO_GLOBAL;
        g.pass_num = p;
        g.last_pass = p == np - 1;
        g.nradix = 1;
        g.radix[0] = radix[p];
        g.radix1 = r1[p];
        g.radix2 = r2[p];
        g.curr_size = curr;
        g.stride_out = so;
        g.pad_in = padded && p == 0 && !reverse;
        g.takes_kweights = padded && p == 0 && reverse;
        g.unpad_out = padded && g.last_pass && reverse;
        g.normalize = g.last_pass;
        g.in_len = g.pad_in ? nr : n;
        if (g.takes_kweights) g.kw_index = add_kw(pl, nr, n);
        if (add_kernel(pl, &g)) return -1;
        curr /= radix[p];
        so *= radix[p];
    }
    return 0;
}

void rko_plan_destroy(rko_plan* pl) {
    if (!pl) return;
    for (int i = 0; i < pl->nkw; ++i) {
        free(pl->kw[i][0]);
        free(pl->kw[i][1]);
    }
    free(pl);
}

/* get_fft_kernels (fft.py:532-584) with local_kernel_limit (max_total_local_size) */
rko_plan* rko_plan_create(int ndim, const int64_t* shape, int naxes, const int* axes, int64_t local_limit) {
    rko_plan* pl = (rko_plan*)calloc(1, sizeof(rko_plan));
    if (!pl) return NULL;
    pl->ndim = ndim;
    for (int i = 0; i < ndim; ++i) pl->shape[i] = shape[i];
    for (int ai = naxes - 1; ai >= 0; --ai) {
        const int axis = axes[ai];
        int64_t outer = 1, inner = 1;
        for (int i = 0; i < axis; ++i) outer *= shape[i];
        for (int i = axis + 1; i < ndim; ++i) inner *= shape[i];
        const int64_t n = shape[axis];
        if (n == 1) continue;
        const int64_t b = bpow2(n);
        int rc;
        if (b == n) {
            rc = fft_1d(pl, axis, outer, n, inner, local_limit, 0, n);
        } else {
            const int first = pl->nk;
            rc = fft_1d(pl, axis, outer, 2 * b, inner, local_limit, 0, n);
            if (!rc) rc = fft_1d(pl, axis, outer, 2 * b, inner, local_limit, 1, n);
            (void)first;
        }
        if (rc) {
            rko_plan_destroy(pl);
            return NULL;
        }
    }
    return pl;
}

int rko_plan_nkernels(const rko_plan* pl) { return pl->nk; }

/* kernel info: kind, axis, fft_size, fft_size_real, reverse, pad_in, takes_kweights,
 * unpad_out, pass_num, nradix, radix[0..nradix), radix1, radix2 */
int rko_plan_kernel(const rko_plan* pl, int i, int64_t* info) {
    if (i < 0 || i >= pl->nk) return -1;
    const rko_kernel* k = &pl->k[i];
    int n = 0;
    info[n++] = k->kind;
    info[n++] = k->axis;
    info[n++] = k->fft_size;
    info[n++] = k->fft_size_real;
    info[n++] = k->reverse_direction;
    info[n++] = k->pad_in;
    info[n++] = k->takes_kweights;
    info[n++] = k->unpad_out;
    info[n++] = k->pass_num;
    info[n++] = k->nradix;
    for (int r = 0; r < k->nradix; ++r) info[n++] = k->radix[r];
    info[n++] = k->radix1;
    info[n++] = k->radix2;
    return n;
}

#define REAL float
#define SFX(x) x##_f
#define COS cosf
#define SIN sinf
#include "rko_body.h"
#undef REAL
#undef SFX
#undef COS
#undef SIN

#define REAL double
#define SFX(x) x##_d
#define COS cos
#define SIN sin
#include "rko_body.h"
#undef REAL
#undef SFX
#undef COS
#undef SIN

int rko_exec_c64(const rko_plan* pl, const float* in, float* out, int inverse, int nthreads) {
    return exec_f(pl, (const void*)in, (void*)out, inverse, nthreads);
}
int rko_exec_c128(const rko_plan* pl, const double* in, double* out, int inverse, int nthreads) {
    return exec_d(pl, (const void*)in, (void*)out, inverse, nthreads);
}
/* FFT followed by a fused output fftshift (shift[d] per axis) and scale */
int rko_exec_c64_shift(const rko_plan* pl, const float* in, float* out, int inverse, int nthreads, const int* shift,
                       double scale) {
    return exec_ex_f(pl, (const void*)in, (void*)out, inverse, nthreads, shift, scale);
}
int rko_exec_c128_shift(const rko_plan* pl, const double* in, double* out, int inverse, int nthreads,
                        const int* shift, double scale) {
    return exec_ex_d(pl, (const void*)in, (void*)out, inverse, nthreads, shift, scale);
}
