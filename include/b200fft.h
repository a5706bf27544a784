/*
 * b200fft.h — C ABI of the B200-native ParaFaFT transform backend.
 *
 * These entry points are what a ParaFaFT backend needs from a batched 1D FFT
 * engine: the `Backend` concept of ParaFaFT (backend/fft_backend.hpp:45-196)
 * calls plan creation once per stage, then executes the plans on arbitrary
 * pointers with the same layout ("new-array" execution,
 * backend/fft_backend.hpp:107-111). The C++ class B200Backend<T>
 * (include/fft_backend_b200.hpp) implements that concept on top of this ABI.
 *
 * All transforms are unnormalised; forward uses exp(-2*pi*i*j*k/n), backward
 * exp(+2*pi*i*j*k/n) (backend/fft_backend.hpp:25-28, FFTW sign convention).
 *
 * Every function returns B200FFT_SUCCESS (0) or a negative status; the text of
 * the last failure on the calling thread is available from b200fft_last_error().
 *
 * Execution model. Work is stream-ordered and asynchronous until
 * b200fft_sync(). A handle may hold back two kinds of work so that it can fuse
 * it (results are identical to immediate execution):
 *   - a device-to-device b200fft_memcpy whose destination is then transformed
 *     in place is folded into that transform (the transform reads the copy's
 *     source and writes the destination), which removes the identity copies
 *     that ParaFaFT's single-rank exchange_local issues between stages
 *     (parafaft_common.hpp:467-543);
 *   - consecutive b200fft_exec_c2c calls of one middle-axis stage on
 *     consecutive slices (the leading-dimension loop of
 *     parafaft_c2c.hpp:875-896 / parafaft_r2c.hpp:1224-1244) are merged into
 *     one launch that starts as soon as the last slice of the loop arrives.
 * Held-back work is issued by the next call on the handle that does not extend
 * it and by b200fft_sync()/b200fft_flush(). Create the handle with
 * B200FFT_FLAG_NO_DEFER to issue every call immediately.
 */
#ifndef B200FFT_H
#define B200FFT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define B200FFT_SUCCESS 0
#define B200FFT_ERR_INVALID_ARG (-1)   /* bad handle, pointer, stage, size   */
#define B200FFT_ERR_UNSUPPORTED (-2)   /* length/layout the engine lacks     */
#define B200FFT_ERR_NO_PLAN (-3)       /* exec before the matching plan      */
#define B200FFT_ERR_CUDA (-4)          /* CUDA runtime failure               */
#define B200FFT_ERR_RANGE (-5)         /* size arithmetic would overflow     */
#define B200FFT_ERR_NO_DEVICE (-6)     /* no CUDA device visible             */
#define B200FFT_ERR_DEVICE_STATUS (-7) /* a kernel reported a failure        */

/* ---- enums mirroring parafaft::FFTDirection / FFTPlanFlag --------------- */
/* backend/fft_backend.hpp:25-28 */
#define B200FFT_FORWARD 0
#define B200FFT_BACKWARD 1
/* backend/fft_backend.hpp:39-43 */
#define B200FFT_PLAN_ESTIMATE 0
#define B200FFT_PLAN_MEASURE 1
#define B200FFT_PLAN_PATIENT 2

/* precision of a handle (FloatType of the backend) */
#define B200FFT_F32 0
#define B200FFT_F64 1

/* handle creation flags (bitwise or) */
#define B200FFT_FLAG_NO_DEFER 1u   /* issue every call at once: no fusion   */
#define B200FFT_FLAG_RECORD_ONLY 2u /* plan and account, never touch a GPU  */
#define B200FFT_FLAG_GENERIC_ONLY 4u /* force the runtime-generic kernels    */
/* FP32 C2C plans of length 256, 512 and 1024 use the split-precision
 * tensor-core kernels: radix-16 DFT blocks as FP16 hi+lo matrix products
 * with FP32 accumulation (relative L2 error within twice the plain FP32
 * kernels'). Other plans are unaffected. Also set by B200FFT_SPLIT_TC=1. */
#define B200FFT_FLAG_SPLIT_TC 8u

typedef struct b200fft_handle_s *b200fft_handle;

/* Counters a handle keeps since creation (or the last reset). */
typedef struct b200fft_stats {
  uint64_t kernel_launches;   /* transform kernels launched              */
  uint64_t exec_calls;        /* exec_c2c/r2c/c2r calls received          */
  uint64_t coalesced_calls;   /* exec_c2c calls merged into a prior launch */
  uint64_t memcpy_calls;      /* b200fft_memcpy/memcpy2d calls received   */
  uint64_t fused_copies;      /* memcpy calls folded into a transform     */
  uint64_t copies_issued;     /* cudaMemcpy*Async actually issued         */
  uint64_t bytes_copied;      /* bytes moved by the issued copies         */
  uint64_t bytes_transformed; /* algorithmic bytes read+written by kernels */
} b200fft_stats;

/* One entry of the launch log a handle keeps (see b200fft_get_log). */
typedef struct b200fft_launch_record {
  int kind;          /* 0 c2c, 1 r2c, 2 c2r, 3 copy                         */
  int direction;     /* B200FFT_FORWARD / B200FFT_BACKWARD                   */
  int stage;         /* stage index for c2c, -1 otherwise                    */
  int family;        /* 0 static specialised kernel, 1 runtime generic,
                        2/3 split-precision tensor core (mma.sync / tcgen05),
                        4 TMA-fed specialised column kernel, -1 copy */
  int length;        /* transform length (real length for r2c/c2r)          */
  int fused_copy;    /* 1 when the transform read a held-back copy's source */
  long long transforms; /* 1D transforms in the launch (batch x slabs)      */
  long long slabs;      /* number of coalesced slices                       */
  long long bytes;      /* algorithmic bytes (or copy bytes)                */
  double ms;            /* device time from CUDA events around the launch on
                           the handle's stream when profiling is on, else -1 */
} b200fft_launch_record;

/* ---- library ------------------------------------------------------------ */
/* Text of the last failure on this thread ("" when none). */
const char *b200fft_last_error(void);
/* Library version as 10000*major + 100*minor + patch. */
int b200fft_version(void);
/* Number of usable CUDA devices (0 when none; never fails). */
int b200fft_device_count(void);

/* ---- handles (replaces the backend constructor/destructor,
 *      fft_backend_cufft.hpp:191-237) ------------------------------------- */
/* Backend(num_stages, comm, plan_flag): precision is B200FFT_F32/F64. */
int b200fft_create(int precision, int num_stages, int plan_flag,
                   unsigned flags, b200fft_handle *out);
/* ~Backend(): synchronises the handle's stream, frees plans and tables. */
int b200fft_destroy(b200fft_handle h);
/* Use a caller-owned cudaStream_t instead of the handle's own stream
 * (NULL restores the handle's stream). Held-back work is issued first. */
int b200fft_set_stream(b200fft_handle h, void *cuda_stream);

/* ---- C2C stages (fft_backend_cufft.hpp:292-312 create_stage_plan,
 *      :325-337 execute_stage) ------------------------------------------- */
/* Batched 1D C2C of `length` points; element j of transform b sits at
 * data[b*dist + j*stride] (complex elements). batch/stride/dist are 64-bit:
 * no int narrowing (the cuFFT backend's narrow_plan_arg limit,
 * fft_backend_cufft.hpp:673-689, does not apply). */
int b200fft_plan_c2c(b200fft_handle h, int stage, int length, size_t batch,
                     ptrdiff_t stride, ptrdiff_t dist);
int b200fft_exec_c2c(b200fft_handle h, int stage, int direction, void *data);

/* ---- in-place R2C / C2R (fft_backend_cufft.hpp:360-405, :427-469) ------- */
/* `stride` and `dist` are in real (FloatType) units; the complex side uses
 * stride and dist/2 complex elements, as FFTW's guru64 plans do
 * (fft_backend_fftw.hpp:439-549). */
int b200fft_plan_r2c(b200fft_handle h, int length, size_t batch,
                     ptrdiff_t stride, ptrdiff_t dist);
int b200fft_exec_r2c(b200fft_handle h, void *padded_real);
int b200fft_plan_c2r(b200fft_handle h, int length, size_t batch,
                     ptrdiff_t stride, ptrdiff_t dist);
/* Ignores Im of the DC and Nyquist terms, as FFTW's c2r does. */
int b200fft_exec_c2r(b200fft_handle h, void *padded_real);

/* ---- copies and ordering (fft_backend_cufft.hpp:483-519) ---------------- */
int b200fft_memcpy(b200fft_handle h, void *dst, const void *src, size_t bytes);
int b200fft_memcpy2d(b200fft_handle h, void *dst, size_t dpitch,
                     const void *src, size_t spitch, size_t width,
                     size_t height);
/* Issue held-back work, then block until the handle's stream is idle. */
int b200fft_sync(b200fft_handle h);
/* Issue held-back work without blocking. */
int b200fft_flush(b200fft_handle h);

/* ---- planning with measurement (FFTPlanFlag::Measure / Patient) ---------- */
/* Buffer the next plans may use to time kernel candidates in place (contents
 * are overwritten, as FFTW_MEASURE overwrites its planning array). ParaFaFT
 * passes its scratch buffer to create_*_plan for this (parafaft_c2c.hpp:263-284,
 * parafaft_r2c.hpp:1174-1203); B200Backend forwards it here. bytes = 0 means
 * "large enough for every plan's layout". */
int b200fft_set_work_buffer(b200fft_handle h, void *work, size_t bytes);
/* The kernel a plan uses (kind 0 c2c with `stage`, 1 r2c, 2 c2r). */
int b200fft_plan_describe(b200fft_handle h, int kind, int stage, char *buf,
                          size_t buflen);
/* Plan cache, the analogue of FFTW wisdom (fft_backend_fftw.hpp:666-694):
 * measured choices keyed by GPU model and plan geometry. Import returns the
 * number of entries read (or a negative status). */
int b200fft_export_wisdom(const char *path);
int b200fft_import_wisdom(const char *path);
int b200fft_forget_wisdom(void);

/* ---- device memory for the backend's Buffer/ComplexBuffer types
 *      (replaces cuvector<T>, fft_backend_cufft.hpp:58-121) --------------- */
int b200fft_alloc(size_t bytes, void **ptr);
int b200fft_free(void *ptr);

/* ---- batches of independent grids (no counterpart in the reference: the
 *      batching extension of the backend) ---------------------------------- */
/* A group runs the transforms of many handles (for example one ParaFaFT
 * object per grid) together. Member handles use the group's stream. Between
 * b200fft_group_begin and b200fft_group_end their passes are recorded (after
 * the usual copy fusion and slice coalescing) instead of launched, and
 * b200fft_sync on them returns at once. b200fft_group_end then runs the
 * recording level by level (level d: the d-th recorded pass or copy of every
 * handle): passes with a specialised kernel launch once per (precision, kind,
 * layout, direction, length), one CTA per tile of any handle's pass (a single
 * pass launches its plan's own kernel); the others share one persistent
 * launch whose CTAs take (transform, tile) work items from a device queue.
 * The launches of one level run side by side on several streams, so the
 * handles of a group must not share data. The recorded schedule stays valid
 * for the same buffers: group_replay runs it again, group_capture records it
 * once into a CUDA graph that replay then launches. */
typedef struct b200fft_group_s *b200fft_group;
int b200fft_group_create(b200fft_group *out);
/* Detaches the member handles (they return to their own streams). */
int b200fft_group_destroy(b200fft_group g);
int b200fft_group_add(b200fft_group g, b200fft_handle h);
int b200fft_group_begin(b200fft_group g);
/* Build the schedule from the recording and run it once (asynchronously). */
int b200fft_group_end(b200fft_group g);
/* Record the built schedule into a CUDA graph (replay then launches it). */
int b200fft_group_capture(b200fft_group g);
/* Run the built schedule again on the group's stream. */
int b200fft_group_replay(b200fft_group g);
int b200fft_group_sync(b200fft_group g);
/* Launches, passes and bytes of the last built schedule. */
int b200fft_group_stats(b200fft_group g, b200fft_stats *out);

/* ---- transform without allocation (no counterpart in the reference) ------ */
/* One batched C2C transform of `length` points (element j of transform b at
 * in/out[b*dist + j*stride], in == out allowed) on `cuda_stream` (NULL: the
 * default stream), for callers that cannot allocate device memory where they
 * transform: applications that hand out all device memory from their own pool,
 * and latency-critical loops that must not let cudaMalloc/cudaFree synchronize
 * the device. It needs no handle and calls no allocator: its twiddle table
 * lives in a fixed 128 KiB array inside the library, so `length` must be a
 * power of two from 2 to 4096 (anything else returns B200FFT_ERR_UNSUPPORTED).
 * The first call on a device resolves that array's address; make it before any
 * stream capture. The address is kept for the life of the process, so calls
 * after cudaDeviceReset on that device are not supported. All calls on a
 * device share the array: calls that may run concurrently on the GPU race, so
 * order them on one stream. Columns run on the default tile of the length
 * (no per-stride tile choice, unlike a handle's plan). */
int b200fft_c2c_noalloc(int precision, int direction, int length, size_t batch,
                        ptrdiff_t stride, ptrdiff_t dist, const void *in, void *out,
                        void *cuda_stream);

/* ---- introspection ------------------------------------------------------ */
int b200fft_get_stats(b200fft_handle h, b200fft_stats *out);
int b200fft_reset_stats(b200fft_handle h);
/* Turn per-launch timing on (1) or off (0): each kernel launch and issued
 * copy is bracketed by CUDA events on the handle's stream; b200fft_get_log
 * waits for them and reports the elapsed milliseconds. */
int b200fft_set_profiling(b200fft_handle h, int on);
/* Copy up to `cap` most recent launch records (oldest first); *count gets
 * the number written. The log keeps the last 4096 records. */
int b200fft_get_log(b200fft_handle h, b200fft_launch_record *out, int cap,
                    int *count);
/* Describe the kernel a plan would use: writes a NUL-terminated summary such
 * as "static L=512 col tb=16 nt=256 radices=8x8x8" into buf. Pure host code;
 * works without a GPU. kind: 0 c2c, 1 r2c, 2 c2r. */
int b200fft_describe(int precision, int kind, int length, size_t batch,
                     ptrdiff_t stride, ptrdiff_t dist, char *buf,
                     size_t buflen);
/* 1 when the engine has a kernel for this length and kind, else 0. */
int b200fft_supported(int precision, int kind, int length);

#ifdef __cplusplus
}
#endif

#endif /* B200FFT_H */
