/*
 * reikna_b200 -- C ABI of the B200 FFT library.
 *
 * This is the drop-in boundary for reikna's FFT hot path.  The Python classes in
 * reikna_b200 (FFT, FFTShift, RFFT, Spectrogram) build an rk_fft_desc from the
 * computation signature and its connected transformations and call these entry
 * points through ctypes; any other host language can bind the same functions.
 *
 * All functions return RK_OK (0) on success or a negative RK_ERR_* code; the
 * message of the last failure on the calling thread is returned by
 * rk_last_error().  No C++ exception crosses this boundary.
 *
 * Reference interfaces replaced (file:line inside fjarri/reikna):
 *   rk_fft_plan_create    FFT.__init__ (reikna/fft/fft.py:630) + Computation.compile
 *                         (reikna/core/computation.py:259) + FFT._build_plan
 *                         (reikna/fft/fft.py:723) + ComputationPlan.finalize
 *                         (reikna/core/computation.py:642)
 *   rk_fft_execute        ComputationCallable.__call__ (reikna/core/computation.py:766)
 *   rk_fft_plan_destroy   Python GC of ComputationCallable / __tempalloc__
 *                         (reikna/core/computation.py:764)
 *   rk_fft_plan_describe  no runtime counterpart; exposes the kernel chain that
 *                         get_fft_kernels (reikna/fft/fft.py:532) would build
 *   rk_fftshift_execute   FFTShift compiled callable (reikna/fft/fftshift.py:65,
 *                         reikna/fft/fftshift.mako:1-84)
 */
#ifndef REIKNA_B200_H
#define REIKNA_B200_H

#ifndef __CUDACC_RTC__
#include <stdint.h>
#endif

#if defined(__GNUC__)
#define RK_API __attribute__((visibility("default")))
#else
#define RK_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define RK_MAXD 8

/* status codes */
#define RK_OK 0
#define RK_ERR_INVALID (-1)     /* bad descriptor or argument (reikna: ValueError) */
#define RK_ERR_UNSUPPORTED (-2) /* valid request this build cannot plan */
#define RK_ERR_CUDA (-3)        /* a CUDA runtime call failed */
#define RK_ERR_NOMEM (-4)       /* device allocation failed */
#define RK_ERR_DEVICE (-5)      /* device-side status word reported an error */

/* element formats of edge arrays */
#define RK_FMT_C64 1   /* complex64  (float2)  */
#define RK_FMT_C128 2  /* complex128 (double2) */
#define RK_FMT_F32 3   /* float32  real */
#define RK_FMT_F64 4   /* float64  real */
#define RK_FMT_F32_PAIR 5 /* two float32 arrays: real part, imaginary part */
#define RK_FMT_F64_PAIR 6 /* two float64 arrays: real part, imaginary part */
#define RK_FMT_I32 7   /* int32 (FFTShift only) */
#define RK_FMT_C64_HALF 8 /* reserved */
#define RK_FMT_CONST 9  /* input only: no array; every element is the edge's additive term
                           (broadcast_const / broadcast_param on the FFT input) */
#define RK_FMT_IGNORE 10 /* output only: no array; the values are dropped (ignore) */
#define RK_FMT_USER 11  /* the element is produced (input) or consumed (output) by device
                           code compiled at run time for this plan (a transformation given as
                           source code): strides must be the C-order strides of the FFT shape
                           (the code receives the flat index), offset 0, no remap; passes that
                           touch such an edge run only with a kernel installed by
                           rk_fft_plan_set_pass_kernel */

/* output post-operations (applied after scale) */
#define RK_POST_NONE 0
#define RK_POST_NORM 1 /* |z|^p, p = post_param; output format must be real (norm_const) */

/* window applied on load along window_axis (spectrogram framing) */
#define RK_WIN_NONE 0
#define RK_WIN_HANN 1 /* 0.5*(1-cos(2*pi*p/(W-1))) for p < W, 1 beyond */

/* plan flags */
#define RK_FLAG_NO_PLANE 1   /* never fuse two axes into one clustered pass */
#define RK_FLAG_NO_BLUE1 2   /* never use the single-pass Bluestein kernel */
#define RK_FLAG_SPLIT_TC 4   /* tensor-core split-precision stages (tf32 hi/lo, FP32
                                accumulate) for 256- and 1024-point contiguous complex64
                                line passes; others run as usual */
#define RK_FLAG_PLANE_WIDE 8 /* plane pass on twice as many CTAs per cluster (tuning) */
#define RK_FLAG_NO_TMA 16    /* never use the persistent TMA-fed line passes */
#define RK_FLAG_PAIR 32      /* two innermost power-of-two axes: row and column passes in one
                                plane-ordered launch instead of the clustered plane pass */
#define RK_FLAG_REAL_POST 64 /* forward transform of the last axis (length L = N/2, a power of two
                                of at most 8192, 4096 for complex128) of a real signal read as
                                interleaved pairs: the single pass stores the real signal's
                                spectrum X[0 .. L) and, when the output edge is L + 1 long, X[L]
                                (examples/demo_specialized_fft.py:175-241 as one pass);
                                rk_fft_execute then rejects inverse = 1 */
#define RK_FLAG_REAL_PRE 128 /* inverse of RK_FLAG_REAL_POST: the input edge holds the L + 1 bins
                                X[0 .. L] of a real signal's spectrum (the imaginary parts of
                                X[0] and X[L] are ignored, as numpy.fft.irfft does), the first
                                load forms the half-length spectrum, and the output holds the
                                2L real samples numpy.fft.irfft gives, as L interleaved pairs
                                (examples/demo_specialized_fft.py:244-331 as one pass);
                                rk_fft_execute then rejects inverse = 0 */
#define RK_FLAG_BATCHABLE 2048 /* plan only passes the persistent batched kernel has tile bodies for
                                (no plane pass, strided fused Bluestein lines of at most 1024
                                points); rk_batch_create members */
#define RK_FLAG_BLUE_PAIR 4096 /* 8192-point complex64 fused Bluestein lines on a two-CTA
                                cluster a line (each CTA one half of the padded spectrum, one
                                exchange through distributed shared memory) instead of one CTA;
                                tuning (about 11% faster below 100 lines, slower from 500) */
#define RK_FLAG_R16 1024      /* 8192-point complex64 fused Bluestein lines with 16 elements a
                                thread on 512 threads instead of 32 on 256 (tuning) */
#define RK_FLAG_NO_HALF 512   /* never run a real signal's last-axis transform as the half-length
                                FFT of its sample pairs (see rk_fft_plan_create) */
#define RK_FLAG_ANTIPERIODIC 256 /* with RK_FLAG_REAL_POST or RK_FLAG_REAL_PRE: the 2L real
                                samples are the first half x[0 .. 2L) of an antiperiodic signal
                                (x[n + 2L] = -x[n]) of length 4L, whose spectrum is the L odd
                                harmonics F[k] = X[2k + 1]; REAL_POST stores F (an output edge
                                of L bins), REAL_PRE reads F and stores x
                                (examples/demo_specialized_fft.py:379-624, APRFFT / IAPRFFT,
                                as one pass each) */

/*
 * One side (input or output) of the FFT as the user sees it after the
 * transformations are folded in.  Element (i_0, ..., i_{nd-1}) of the FFT array
 * lives at   base + offset + sum_d ((i_d + shift_d) mod fft_shape_d) * strides_d
 * (units: elements of the scalar format; complex elements for complex formats).
 * An index with i_d >= shape_d is outside the user array: loads read 0 there
 * (zero padding) and stores drop it (cropping).
 */
typedef struct rk_edge {
    int32_t format;               /* RK_FMT_* */
    int32_t ndim;                 /* must equal the FFT ndim */
    int64_t shape[RK_MAXD];       /* extent of the user array along each FFT axis */
    int64_t strides[RK_MAXD];     /* element strides */
    int64_t offset;               /* first element offset, elements */
    int64_t strides2[RK_MAXD];    /* strides of the imaginary array (PAIR formats) */
    int64_t offset2;
    int32_t shift[RK_MAXD];       /* index remap (fftshift); 0 = identity */
    double scale_re, scale_im;    /* constant complex multiplier */
    int32_t scale_slot;           /* runtime scalar multiplied in, -1 = none */
    int32_t scale_div_slot;       /* runtime scalar divided by, -1 = none */
    int32_t post;                 /* RK_POST_* (output side only) */
    double post_param;
    int32_t window;               /* RK_WIN_* (input side only) */
    int32_t window_axis;
    int64_t window_len;
    int32_t conj;                 /* 1: conjugate the element (after scale) */
    int32_t add_slot;             /* runtime scalar added after the scale, -1 = none */
    double add_re, add_im;        /* constant added after the scale (with add_slot's value):
                                     element = scale * value + add (add_const / add_param,
                                     and the value of an RK_FMT_CONST input) */
    int32_t post_slot;            /* runtime scalar whose real part is the norm order
                                     (norm_param), -1 = post_param */
} rk_edge;

typedef struct rk_fft_desc {
    int32_t dtype;                /* RK_FMT_C64 or RK_FMT_C128: compute precision */
    int32_t ndim;
    int64_t shape[RK_MAXD];       /* FFT array shape */
    int32_t naxes;
    int32_t axes[RK_MAXD];        /* transformed axes, any order, no repeats */
    int32_t flags;                /* RK_FLAG_* */
    rk_edge input;
    rk_edge output;
} rk_fft_desc;

typedef struct rk_fft_plan rk_fft_plan;

/* Initialise an edge to "contiguous array of the FFT shape, identity ops". */
RK_API int rk_edge_init(rk_edge* e, int32_t format, int32_t ndim, const int64_t* shape);

/* Build a plan on the current CUDA device: kernel chain, temporaries, twiddle and
 * Bluestein tables (generated on the device in FP64).  Synchronous. */
RK_API int rk_fft_plan_create(const rk_fft_desc* desc, rk_fft_plan** plan);

/* Run the plan asynchronously on `stream` (a cudaStream_t; NULL = legacy default).
 * outputs/inputs: device pointers of the user arrays (2 for PAIR formats).
 * inverse: 0 forward (exp(-i...)), 1 inverse normalised by 1/N (IFFT(FFT(x)) = x).
 * scalars: n_scalars complex values, as (re, im) pairs of doubles, for the runtime
 * scalar slots referenced by the edges.
 * Output may alias input. */
RK_API int rk_fft_execute(rk_fft_plan* plan, void* const* outputs, int32_t n_outputs,
                   const void* const* inputs, int32_t n_inputs, int32_t inverse,
                   const double* scalars, int32_t n_scalars, void* stream);

RK_API int rk_fft_plan_destroy(rk_fft_plan* plan);

/*
 * Transformations given as source code (reikna's Transformation(parameters, code),
 * reikna/core/transformation.py:42-120, inlined by reikna into the first and last
 * kernel, reikna/core/transformation_modules.py:260-318).  An edge of format
 * RK_FMT_USER is read or written by device functions compiled at run time together
 * with the pass kernel that calls them; the host compiles one kernel per pass that
 * touches such an edge and installs it here.
 *
 * rk_fft_plan_pass_info: info[0..7] = {kind (0 line, 1 plane), L, mode (0 position,
 *   1 lane), variant, complex128 (0/1), threads per CTA, user bits (1: the pass loads
 *   the input edge's user code, 2: it stores through the output edge's), lines per
 *   CTA}; *smem = dynamic shared memory bytes of a CTA.
 * rk_fft_plan_set_pass_kernel: load a cubin `image` (size bytes) holding the
 *   extern "C" kernel `name` with the pass's launch shape and a single
 *   `rk::PassParams` argument, and run pass `index` with it from now on.
 * rk_fft_execute_user: rk_fft_execute plus up to 8 64-bit words per edge handed to
 *   the user code (array pointers and scalar bit patterns, as the host that generated
 *   the code laid them out).
 */
RK_API int rk_fft_plan_pass_info(const rk_fft_plan* plan, int32_t index, int32_t* info, int64_t* smem);
RK_API int rk_fft_plan_set_pass_kernel(rk_fft_plan* plan, int32_t index, const void* image, int64_t size,
                                       const char* name);
RK_API int rk_fft_execute_user(rk_fft_plan* plan, void* const* outputs, int32_t n_outputs, const void* const* inputs,
                               int32_t n_inputs, int32_t inverse, const double* scalars, int32_t n_scalars,
                               const uint64_t* user_in, int32_t n_user_in, const uint64_t* user_out,
                               int32_t n_user_out, void* stream);

/* Device bytes owned by the plan (temporaries + tables). */
RK_API int rk_fft_plan_device_bytes(const rk_fft_plan* plan, int64_t* bytes);

/* Describe the kernel chain as JSON text without touching the GPU (planner only).
 * Writes at most `cap` bytes including the terminating NUL; *needed receives the
 * full length. */
RK_API int rk_fft_plan_describe(const rk_fft_desc* desc, char* buf, int64_t cap, int64_t* needed);

/* Number of kernels rk_fft_execute launches for this plan. */
RK_API int rk_fft_plan_launches(const rk_fft_plan* plan, int32_t* n);

/* Number of the plan's passes that run on the tensor cores (RK_FLAG_SPLIT_TC).  No
 * counterpart in the reference, which has no tensor-core path. */
RK_API int rk_fft_plan_tc_passes(const rk_fft_plan* plan, int32_t* n);

/* Per-pass timing: record a CUDA event pair around every kernel of the next
 * `max_calls` rk_fft_execute calls (0 stops recording and frees the events).
 * rk_fft_profile_read synchronises on the recorded events and returns, per pass,
 * the summed milliseconds over the `*calls` recorded executions. */
RK_API int rk_fft_profile(rk_fft_plan* plan, int32_t max_calls);
RK_API int rk_fft_profile_read(rk_fft_plan* plan, double* ms_per_pass, int32_t n_passes, int32_t* calls);

/*
 * Standalone FFTShift (reikna/fft/fftshift.py:14): out = fftshift(in) over `axes`
 * (inverse = 1: ifftshift).  Any element size in {4, 8, 16} bytes; contiguous
 * C-order arrays.  Output may alias input (in-place swap kernel when every shifted
 * axis is even, otherwise an out-of-place kernel through `scratch`, which must
 * hold the whole array; scratch may be NULL when every axis is even).
 */
RK_API int rk_fftshift_execute(void* out, const void* in, int32_t elem_bytes, int32_t ndim,
                        const int64_t* shape, int32_t naxes, const int32_t* axes,
                        int32_t inverse, void* scratch, void* stream);

/*
 * Batched transpose of a C-order array of `batch` matrices of height x width
 * elements: out[b][w][h] = in[b][h][w]; replaces one kernel call of reikna's
 * Transpose (reikna/algorithms/transpose.py:157-201), which realises any axis
 * permutation as a sequence of such swaps of adjacent axis groups.  elem_bytes in
 * {1, 2, 4, 8, 16}; pointers aligned to the element size; out may not alias in.
 */
RK_API int rk_transpose_execute(void* out, const void* in, int32_t elem_bytes, int64_t batch, int64_t height,
                                int64_t width, void* stream);

/*
 * Real-signal transforms through a half-length complex FFT, the steps the reference
 * runs as separate kernels around its FFT (examples/demo_specialized_fft.py:156-331,
 * demo_specialized_fft.mako:1-62).  A real array of even length N is read by the
 * complex FFT of length half = N / 2 as interleaved (re, im) pairs.
 *   rk_rfft_twiddles: table[k] = exp(-2 pi i k / N), k = 0 .. half (FP64, rounded).
 *   rk_rfft_post: out[b][k], k < half + store_last, from the half-length spectrum
 *                 z[b][0 .. half) (out may not alias z).
 *   rk_irfft_pre: z[b][0 .. half) from the half-spectrum x[b][0 .. half], for the
 *                 inverse half-length FFT; imaginary parts of bins 0 and half ignored.
 * fmt: RK_FMT_C64 or RK_FMT_C128 (the complex type of z, out, x and the table).
 */
RK_API int rk_rfft_twiddles(void* table, int32_t fmt, int64_t half, void* stream);
RK_API int rk_rfft_post(void* out, const void* z, const void* table, int32_t fmt, int64_t half, int64_t batch,
                        int32_t store_last, void* stream);
RK_API int rk_irfft_pre(void* z, const void* x, const void* table, int32_t fmt, int64_t half, int64_t batch,
                        void* stream);

/*
 * Antiperiodic real signals (examples/demo_specialized_fft.py:334-624, APRFFT /
 * IAPRFFT): the first half x[0 .. 2 half) of a signal with x[n + 2 half] = -x[n];
 * its spectrum is the odd harmonics F[k] = X[2k + 1], k < half.  These are the
 * element-wise steps of the multi-kernel route (half lengths the one-pass
 * RK_FLAG_ANTIPERIODIC plans do not cover); the reference reaches the same F through
 * an RFFT, a cumulative sum and a reduction instead.
 *   rk_aprfft_twiddles: table[k] = exp(-i pi (2k + 1) / (2 half)), k < half, then
 *                       table[half + m] = exp(-i pi m / half), m < half.
 *   rk_aprfft_twiddle:  out[b][m] = in[b][m] table[half + m] (inverse: conjugated);
 *                       in place allowed.  Forward: before FFT_half of the pairs;
 *                       inverse: after the inverse FFT_half, giving the pairs.
 *   rk_aprfft_post:     F[b][k] = C[k] (1 - i w_k) + conj(C[half - 1 - k]) (1 + i w_k)
 *                       from C = FFT_half (out may not alias z).
 *   rk_iaprfft_pre:     C[b][k] = (F[k] conj(1 - i w_k) + conj(F[half - 1 - k])
 *                       conj(1 + i w_k)) / 4 for the inverse FFT_half (z may not alias x).
 */
RK_API int rk_aprfft_twiddles(void* table, int32_t fmt, int64_t half, void* stream);
RK_API int rk_aprfft_twiddle(void* out, const void* in, const void* table, int32_t fmt, int64_t half, int64_t batch,
                             int32_t inverse, void* stream);
RK_API int rk_aprfft_post(void* out, const void* z, const void* table, int32_t fmt, int64_t half, int64_t batch,
                          void* stream);
RK_API int rk_iaprfft_pre(void* z, const void* x, const void* table, int32_t fmt, int64_t half, int64_t batch,
                          void* stream);

/*
 * Allocation-free batched 1-D complex64 FFT.  No counterpart in the reference: it
 * exists for callers that cannot allocate device memory when they need a transform
 * (code inside a memory pool or arena that owns the device, loops that must not
 * enter the allocator, hosts that only lend their own buffers).  out/in: contiguous
 * (batch, n) complex64 device arrays (may alias); n a power of two in
 * [4096, 1048576]; batch * n <= 4194304 (the 32 MiB static scratch every device that
 * loads the library holds until exit).  inverse = 1 gives the 1/n-normalised inverse.
 * Calls no allocating routine.  All calls on a device share the scratch: calls that
 * may overlap on the GPU race.  The first call on a device resolves the static
 * arrays and fills its twiddle tables (kernel launches plus a device
 * synchronisation): make it before any stream capture.  Larger sizes are rejected
 * with RK_ERR_INVALID, and so are a stream or arrays that do not belong to the
 * current device (the static arrays used are the current device's).
 */
RK_API int rk_fft1d_c64_noalloc(void* out, const void* in, int64_t n, int64_t batch, int32_t inverse, void* stream);

/*
 * Batched launch: several plans (any lengths, axes, transformations) executed by one
 * persistent kernel launch.  The reference runs each compiled computation as its own
 * chain of kernel launches (ComputationCallable.__call__, reikna/core/computation.py:766);
 * a batch replaces N such calls.  Every pass of every member must be a line pass with
 * a compiled batched variant (complex64; power-of-two lengths up to 8192 along the
 * contiguous axis, 16 to 256 along strided axes; no plane
 * passes: plan the members with RK_FLAG_NO_PLANE), else RK_ERR_UNSUPPORTED.  A plan
 * may appear once per batch.  The batch keeps pointers to the plans: destroy it
 * before them.  Calls of one batch must be stream-ordered (one stream, or ordered by
 * the caller); each call waits for the host staging slot it reuses (4 in flight).
 */
typedef struct rk_batch rk_batch;
RK_API int rk_batch_create(rk_fft_plan* const* plans, int32_t nplans, rk_batch** batch);
/* outputs[i] / inputs[i]: the pointer arrays of member i, as for rk_fft_execute;
 * inverse, scalars, n_scalars: per member, each may be NULL (forward, no scalars). */
RK_API int rk_batch_execute(rk_batch* batch, void* const* const* outputs, const void* const* const* inputs,
                            const int32_t* inverse, const double* const* scalars, const int32_t* n_scalars,
                            void* stream);
RK_API int rk_batch_destroy(rk_batch* batch);
/* tiles (tasks), passes and grid size of the persistent launch */
RK_API int rk_batch_info(const rk_batch* batch, int64_t* ntasks, int32_t* npasses, int32_t* grid);

RK_API const char* rk_last_error(void);

/* Library version string. */
RK_API const char* rk_version(void);

/* Device status word of the current device (nonzero: a kernel gave up a bounded
 * wait, RK_ERR_DEVICE territory).  Synchronises the device; clear = 1 resets it. */
RK_API int rk_device_status(int32_t* status, int32_t clear);

/* Status bits of the device status word. */
#define RK_STATUS_TIMEOUT 1      /* a bounded wait (copy, cluster exchange, batch or pair
                                    dependency) ran out of its limit */
#define RK_STATUS_BAD_VARIANT 2  /* a batched task had no compiled tile body */

/* Limit, in SM clock cycles, of every bounded wait in the library's kernels on the
 * current device (default 2e9, about one second).  No counterpart in the reference
 * (reikna's kernels never wait on each other).  Set / read. */
RK_API int rk_set_wait_limit(int64_t cycles);
RK_API int rk_get_wait_limit(int64_t* cycles);

/* Synchronise `stream` and return RK_ERR_DEVICE (with the word in rk_last_error) if
 * the current device's status word is nonzero; the word is left as it is. */
RK_API int rk_stream_check(void* stream);

/* Self-test of the bounded waits: one persistent-batch task whose dependency can never
 * complete (the pass it waits for has no tiles), run on `stream` and synchronised.
 * The wait gives up after the current wait limit, the task's body is skipped, and the
 * call returns RK_ERR_DEVICE with RK_STATUS_TIMEOUT set in the status word (clear it
 * with rk_device_status(&w, 1) afterwards).  No counterpart in the reference. */
RK_API int rk_selftest_stalled_wait(void* stream);

/* sizeof(rk_edge) and sizeof(rk_fft_desc) as compiled, for binding checks. */
RK_API int rk_abi_sizes(int64_t* edge_bytes, int64_t* desc_bytes);

#ifdef __cplusplus
}
#endif

#endif /* REIKNA_B200_H */
