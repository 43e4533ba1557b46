/*
 * Precision-generic body of the CPU oracle (included twice by reikna_fft_oracle.c
 * with REAL = float / double).  TEST INFRASTRUCTURE ONLY: this restates reikna's FFT
 * kernels on the CPU so that the CUDA library can be checked against it; nothing in
 * the product links or calls it.
 */

typedef struct {
    REAL x, y;
} SFX(cx_t);
#define CX SFX(cx_t)

static inline CX SFX(cx)(REAL x, REAL y) {
    CX r;
    r.x = x;
    r.y = y;
    return r;
}
static inline CX SFX(add)(CX a, CX b) { return SFX(cx)(a.x + b.x, a.y + b.y); }
static inline CX SFX(sub)(CX a, CX b) { return SFX(cx)(a.x - b.x, a.y - b.y); }
/* grunnur functions.mul for complex operands */
static inline CX SFX(mul)(CX a, CX b) { return SFX(cx)(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
/* grunnur functions.polar_unit: (cos t, sin t) in the working precision */
static inline CX SFX(polar)(REAL t) { return SFX(cx)(COS(t), SIN(t)); }
/* conj_transp_and_mul (fft.mako:18): (-a.y * b, a.x * b) */
static inline CX SFX(ctm)(CX a, REAL b) { return SFX(cx)(-a.y * b, a.x * b); }

/* fftKernel2S (fft.mako:56-62) */
static inline void SFX(k2s)(CX* d1, CX* d2) {
    CX c = *d1;
    *d1 = SFX(add)(c, *d2);
    *d2 = SFX(sub)(c, *d2);
}
static inline void SFX(swap)(CX* a, CX* b) {
    CX c = *a;
    *a = *b;
    *b = c;
}

/* fftKernel4 (fft.mako:64-72) */
static void SFX(fk4)(CX* a, int dir) {
    SFX(k2s)(a + 0, a + 2);
    SFX(k2s)(a + 1, a + 3);
    SFX(k2s)(a + 0, a + 1);
    a[3] = SFX(ctm)(a[3], (REAL)dir);
    SFX(k2s)(a + 2, a + 3);
    SFX(swap)(a + 1, a + 2);
}
/* fftKernel4s (fft.mako:74-83) */
static void SFX(fk4s)(CX* a0, CX* a1, CX* a2, CX* a3, int dir) {
    SFX(k2s)(a0, a2);
    SFX(k2s)(a1, a3);
    SFX(k2s)(a0, a1);
    *a3 = SFX(ctm)(*a3, (REAL)dir);
    SFX(k2s)(a2, a3);
    SFX(swap)(a1, a2);
}

/* fftKernel8 (fft.mako:91-117) */
static void SFX(fk8)(CX* a, int dir) {
    const REAL s4 = (REAL)0.70710678118654752440;
    const CX w1 = SFX(cx)(s4, s4 * dir);
    const CX w3 = SFX(cx)(-s4, s4 * dir);
    SFX(k2s)(a + 0, a + 4);
    SFX(k2s)(a + 1, a + 5);
    SFX(k2s)(a + 2, a + 6);
    SFX(k2s)(a + 3, a + 7);
    a[5] = SFX(mul)(w1, a[5]);
    a[6] = SFX(ctm)(a[6], (REAL)dir);
    a[7] = SFX(mul)(w3, a[7]);
    SFX(k2s)(a + 0, a + 2);
    SFX(k2s)(a + 1, a + 3);
    SFX(k2s)(a + 4, a + 6);
    SFX(k2s)(a + 5, a + 7);
    a[3] = SFX(ctm)(a[3], (REAL)dir);
    a[7] = SFX(ctm)(a[7], (REAL)dir);
    SFX(k2s)(a + 0, a + 1);
    SFX(k2s)(a + 2, a + 3);
    SFX(k2s)(a + 4, a + 5);
    SFX(k2s)(a + 6, a + 7);
    /* bitreverse8 */
    SFX(swap)(a + 1, a + 4);
    SFX(swap)(a + 3, a + 6);
}

/* fftKernel16 (fft.mako:129-163) */
static void SFX(fk16)(CX* a, int dir) {
    const REAL w0 = (REAL)0.92387953251128675613; /* cos(pi/8) */
    const REAL w1 = (REAL)0.38268343236508977173; /* sin(pi/8) */
    const REAL w2 = (REAL)0.70710678118654752440; /* sin(pi/4) */
    CX t;
    SFX(fk4s)(a + 0, a + 4, a + 8, a + 12, dir);
    SFX(fk4s)(a + 1, a + 5, a + 9, a + 13, dir);
    SFX(fk4s)(a + 2, a + 6, a + 10, a + 14, dir);
    SFX(fk4s)(a + 3, a + 7, a + 11, a + 15, dir);
    t = SFX(cx)(w0, dir * w1);
    a[5] = SFX(mul)(a[5], t);
    t = SFX(cx)(w1, dir * w0);
    a[7] = SFX(mul)(a[7], t);
    t = SFX(cx)(w2, dir * w2);
    a[6] = SFX(mul)(a[6], t);
    a[9] = SFX(mul)(a[9], t);
    a[10] = SFX(ctm)(a[10], (REAL)dir);
    t = SFX(cx)(-w2, dir * w2);
    a[11] = SFX(mul)(a[11], t);
    a[14] = SFX(mul)(a[14], t);
    t = SFX(cx)(w1, dir * w0);
    a[13] = SFX(mul)(a[13], t);
    t = SFX(cx)(-w0, -dir * w1);
    a[15] = SFX(mul)(a[15], t);
    SFX(fk4)(a, dir);
    SFX(fk4)(a + 4, dir);
    SFX(fk4)(a + 8, dir);
    SFX(fk4)(a + 12, dir);
    /* bitreverse4x4 */
    SFX(swap)(a + 1, a + 4);
    SFX(swap)(a + 2, a + 8);
    SFX(swap)(a + 3, a + 12);
    SFX(swap)(a + 6, a + 9);
    SFX(swap)(a + 7, a + 13);
    SFX(swap)(a + 11, a + 14);
}

static void SFX(fk)(CX* a, int r, int dir) {
    switch (r) {
        case 1: break;
        case 2: SFX(k2s)(a, a + 1); break;
        case 4: SFX(fk4)(a, dir); break;
        case 8: SFX(fk8)(a, dir); break;
        case 16: SFX(fk16)(a, dir); break;
        default: abort();
    }
}

/* xweight (fft.mako:196-202): polar_unit(dir * (pi / Nr) * ((pos*pos) mod 2Nr)) */
static inline CX SFX(xweight)(int dir, int64_t pos, int64_t nr) {
    const REAL c = (REAL)(M_PI / (double)nr);
    const int64_t m = (int64_t)(((unsigned __int128)pos * (unsigned __int128)pos) % (unsigned __int128)(2 * nr));
    return SFX(polar)((REAL)dir * c * (REAL)m);
}

/*
 * One kernel of reikna's chain applied to one line (contiguous copy).
 * in: length in_len, out: length out_len.  kw: kernel weights row for this direction.
 */
static void SFX(run_kernel)(const rko_kernel* k, const CX* in, CX* out, CX* work, CX* work2, int dir,
                            const CX* kw) {
    const int64_t n = k->fft_size, nr = k->fft_size_real;
    /* load with pad_in / kweights (fft.mako:206-236, 867-890) */
    for (int64_t p = 0; p < n; ++p) {
        CX v;
        if (k->pad_in) {
            v = p < nr ? in[p] : SFX(cx)(0, 0);
            v = SFX(mul)(v, SFX(xweight)(dir, p, nr));
        } else {
            v = in[p];
        }
        if (k->takes_kweights) v = SFX(mul)(v, kw[p]);
        work[p] = v;
    }
    CX a[128];
    if (k->kind == RKO_LOCAL) {
        /* fft_local (fft.mako:750-814): Stockham stages over radix_arr */
        int64_t P = 1, data_len = n;
        for (int r = 0; r < k->nradix; ++r) {
            const int R = k->radix[r];
            const int last = r == k->nradix - 1;
            for (int64_t b = 0; b < n / R; ++b) {
                for (int m = 0; m < R; ++m) a[m] = work[b + (n / R) * m];
                SFX(fk)(a, R, dir);
                if (!last) {
                    /* insertTwiddleKernel (fft.mako:636-649) */
                    const REAL angf = (REAL)(b / P);
                    for (int kk = 1; kk < R; ++kk) {
                        const REAL c = (REAL)(2.0 * M_PI * kk / (double)data_len);
                        a[kk] = SFX(mul)(a[kk], SFX(polar)(c * angf * (REAL)dir));
                    }
                }
                const int64_t l = b % P, j1 = b / P;
                for (int m = 0; m < R; ++m) work2[l + P * (m + (int64_t)R * j1)] = a[m];
            }
            CX* t = work;
            work = work2;
            work2 = t;
            P *= R;
            data_len /= R;
        }
    } else {
        /* fft_global pass (fft.mako:816-1038) */
        const int R = k->radix[0], r1 = k->radix1, r2 = k->radix2;
        const int64_t so = k->stride_out, cs = k->curr_size;
        for (int64_t i = 0; i < n / R; ++i) {
            CX xin[128];
            for (int m = 0; m < R; ++m) xin[m] = work[i + (n / R) * m];
            CX y[128];
            if (r2 == 1) {
                for (int m = 0; m < R; ++m) a[m] = xin[m];
                SFX(fk)(a, R, dir);
                for (int m = 0; m < R; ++m) y[m] = a[m];
            } else {
                /* radix = r1 * r2: r1-point DFTs over the high digit, twiddle, r2-point DFTs */
                CX z[128];
                for (int t = 0; t < r2; ++t) {
                    for (int j = 0; j < r1; ++j) a[j] = xin[t + r2 * j];
                    SFX(fk)(a, r1, dir);
                    for (int kk = 1; kk < r1; ++kk) {
                        const REAL c = (REAL)(2.0 * M_PI * kk / (double)R);
                        a[kk] = SFX(mul)(a[kk], SFX(polar)(c * (REAL)t * (REAL)dir));
                    }
                    for (int j = 0; j < r1; ++j) z[j * r2 + t] = a[j];
                }
                for (int k1 = 0; k1 < r1; ++k1) {
                    for (int t = 0; t < r2; ++t) a[t] = z[k1 * r2 + t];
                    SFX(fk)(a, r2, dir);
                    for (int k2 = 0; k2 < r2; ++k2) y[k1 + r1 * k2] = a[k2];
                }
            }
            if (!k->last_pass) {
                /* global twiddle (fft.mako:933-947) */
                const REAL ang1 = (REAL)(2.0 * M_PI / (double)cs) * (REAL)(i / so) * (REAL)dir;
                for (int kk = 0; kk < R; ++kk) y[kk] = SFX(mul)(y[kk], SFX(polar)(ang1 * (REAL)kk));
            }
            for (int kk = 0; kk < R; ++kk) work2[(i / so) * R * so + kk * so + (i % so)] = y[kk];
        }
        CX* t = work;
        work = work2;
        work2 = t;
    }
    /* normalisation and store with unpad_out (fft.mako:266-308, 994-1003) */
    const int64_t out_len = k->unpad_out ? nr : n;
    const REAL norm = (dir == 1 && k->normalize) ? (REAL)n : (REAL)1;
    for (int64_t p = 0; p < out_len; ++p) {
        CX v = work[p];
        if (k->unpad_out) v = SFX(mul)(v, SFX(xweight)(-dir, p, nr));
        v.x = v.x / norm;
        v.y = v.y / norm;
        out[p] = v;
    }
}

/* Output transformation of the last store: out[(i + shift) mod n] = scale * A[i]
 * per axis (examples/demo_fftshift_transformation.py:24-71 with mul_const). */
static void SFX(store_shift)(const rko_plan* pl, const CX* A, CX* out, const int* shift, double scale, int nthreads) {
    const int nd = pl->ndim;
    int64_t inner = 1;
    for (int d = 1; d < nd; ++d) inner *= pl->shape[d];
    const REAL s = (REAL)scale;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int64_t i0 = 0; i0 < pl->shape[0]; ++i0) {
        for (int64_t r = 0; r < inner; ++r) {
            int64_t rem = r, dst = 0, mul = 1;
            for (int d = nd - 1; d >= 1; --d) {
                const int64_t n = pl->shape[d];
                int64_t idx = rem % n;
                rem /= n;
                idx = (idx + shift[d]) % n;
                dst += idx * mul;
                mul *= n;
            }
            const int64_t d0 = (i0 + shift[0]) % pl->shape[0];
            CX v = A[i0 * inner + r];
            v.x *= s;
            v.y *= s;
            out[d0 * inner + dst] = v;
        }
    }
}

/* Execute a planned chain on an array (C order, shape[]), in -> out. */
static int SFX(exec_ex)(const rko_plan* pl, const CX* in, CX* out, int inverse, int nthreads, const int* shift,
                        double scale);
static int SFX(exec)(const rko_plan* pl, const CX* in, CX* out, int inverse, int nthreads) {
    return SFX(exec_ex)(pl, in, out, inverse, nthreads, NULL, 1.0);
}
static int SFX(exec_ex)(const rko_plan* pl, const CX* in, CX* out, int inverse, int nthreads, const int* shift,
                        double scale) {
    int64_t total = 1;
    for (int d = 0; d < pl->ndim; ++d) total *= pl->shape[d];
    if (pl->nk == 0) {
        memcpy(out, in, (size_t)total * sizeof(CX));
        return 0;
    }
    /* working arrays large enough for padded intermediates */
    int64_t maxel = total;
    for (int i = 0; i < pl->nk; ++i) {
        const rko_kernel* k = &pl->k[i];
        const int64_t e = k->outer * k->fft_size * k->inner;
        if (e > maxel) maxel = e;
    }
    CX* A = (CX*)malloc((size_t)maxel * sizeof(CX));
    CX* B = (CX*)malloc((size_t)maxel * sizeof(CX));
    if (!A || !B) {
        free(A);
        free(B);
        return -1;
    }
    memcpy(A, in, (size_t)total * sizeof(CX));
    for (int i = 0; i < pl->nk; ++i) {
        const rko_kernel* k = &pl->k[i];
        const int dir = k->reverse_direction ? (1 - inverse * 2) : -(1 - inverse * 2);
        const int64_t in_len = k->in_len;
        const int64_t out_len = k->unpad_out ? k->fft_size_real : k->fft_size;
        const int64_t lines = k->outer * k->inner;
        CX* kw = NULL;
        if (k->takes_kweights) {
            kw = (CX*)malloc((size_t)k->fft_size * sizeof(CX));
            const int row = (1 - dir) / 2;
            for (int64_t p = 0; p < k->fft_size; ++p)
                kw[p] = SFX(cx)((REAL)pl->kw[k->kw_index][row][2 * p], (REAL)pl->kw[k->kw_index][row][2 * p + 1]);
        }
#pragma omp parallel num_threads(nthreads)
        {
            CX* li = (CX*)malloc((size_t)k->fft_size * sizeof(CX));
            CX* lo = (CX*)malloc((size_t)k->fft_size * sizeof(CX));
            CX* w1 = (CX*)malloc((size_t)k->fft_size * sizeof(CX));
            CX* w2 = (CX*)malloc((size_t)k->fft_size * sizeof(CX));
#pragma omp for schedule(static)
            for (int64_t l = 0; l < lines; ++l) {
                const int64_t o = l / k->inner, ii = l % k->inner;
                const CX* src = A + o * in_len * k->inner + ii;
                for (int64_t p = 0; p < in_len; ++p) li[p] = src[p * k->inner];
                for (int64_t p = in_len; p < k->fft_size; ++p) li[p] = SFX(cx)(0, 0);
                SFX(run_kernel)(k, li, lo, w1, w2, dir, kw);
                CX* dst = B + o * out_len * k->inner + ii;
                for (int64_t p = 0; p < out_len; ++p) dst[p * k->inner] = lo[p];
            }
            free(li);
            free(lo);
            free(w1);
            free(w2);
        }
        free(kw);
        CX* t = A;
        A = B;
        B = t;
    }
    if (shift)
        SFX(store_shift)(pl, A, out, shift, scale, nthreads);
    else
        memcpy(out, A, (size_t)total * sizeof(CX));
    free(A);
    free(B);
    return 0;
}

#undef CX
