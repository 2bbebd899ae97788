/* C ABI of the B200 batched FFT library (libbfly_b200.so).
 *
 * Plain pointers, sizes and int status codes; no C++ or torch types.  Each entry point
 * replaces one method of the reference's C++ plan API (TruNcat3/ascend-fft,
 * include/butterfly/plan.hpp; implementation src/framework/butterfly.cpp), cited beside it.
 *
 * Status codes (reference docs/reference/api.md:34-50):
 *   context init: 0 ok, -1 runtime, -2 device, -3 stream, -4 configuration, -9 re-init
 *   plan calls:   0 ok, -1 kernel unavailable, -2 prepare, -3 alloc, -4 H2D, -5 launch,
 *                 -6 sync, -7 D2H (measure: acceptance failed), -8 shape/guard
 *   C ABI only:   -10 null handle / argument, -11 buffer too small
 *
 * Layouts: complex data is interleaved fp32 [re, im]; C2C rows are [batch][2n] floats,
 * R2C output / C2R input rows are [batch][n+2] floats (n/2+1 complex bins).
 * Threading: one thread at a time per plan; a context owns one CUDA stream.
 */
#ifndef BFLY_B200_H
#define BFLY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bfly_context bfly_context;
typedef struct bfly_plan bfly_plan;

typedef struct bfly_metric {
    double eta_us;
    double measured_us;
    double max_rel_err;
    int measured_ok;
} bfly_metric;

/* Library version string. */
const char* bfly_version(void);

/* Context lifetime; replaces bfly::Context::Context / ~Context (plan.hpp:62-63). */
int bfly_context_create(bfly_context** out);
void bfly_context_destroy(bfly_context* ctx);

/* Replaces Context::init(profilePath, spacePath, kernelPath) (plan.hpp:68,
 * butterfly.cpp:938-958).  kernel_path "builtin" selects the kernels compiled into this
 * library. */
int bfly_context_init(bfly_context* ctx, const char* profile_path, const char* space_path,
                      const char* kernel_path);
/* Same, overriding the profile's device_index (one process per GPU). */
int bfly_context_init_device(bfly_context* ctx, const char* profile_path,
                             const char* space_path, const char* kernel_path, int device);

/* Replaces Context::enumerate (plan.hpp:75): writes "id\tstate\treason\n" lines into buf
 * (NUL-terminated); *count receives the number of candidates, *needed the bytes required. */
int bfly_context_enumerate(bfly_context* ctx, uint32_t n, uint32_t batch, char* buf,
                           size_t cap, int* count, size_t* needed);

/* Replaces Context::select(n, batch, topK, log) (plan.hpp:78, butterfly.cpp:999-1102):
 * the measuring autotuner.  log may be NULL; otherwise up to log_cap bytes are written. */
int bfly_context_select(bfly_context* ctx, uint32_t n, uint32_t batch, int top_k,
                        bfly_plan** out, char* log, size_t log_cap);

/* Replaces Context::makePlan(candidate) (plan.hpp:82): the candidate is named by the id
 * printed by enumerate. */
int bfly_context_make_plan(bfly_context* ctx, uint32_t n, uint32_t batch,
                           const char* candidate_id, bfly_plan** out);

/* Persist autotuner choices in a JSON file (new; the reference re-measures every select). */
int bfly_context_set_tuning_cache(bfly_context* ctx, const char* path);

/* The context's CUDA stream (cudaStream_t as void*). */
void* bfly_context_stream(bfly_context* ctx);

/* Replaces Plan::~Plan (plan.hpp:28). */
void bfly_plan_destroy(bfly_plan* plan);

/* Candidate id of the plan into buf. */
int bfly_plan_candidate_id(bfly_plan* plan, char* buf, size_t cap);

/* Replaces Plan::prepare(n, batch) (plan.hpp:34, butterfly.cpp:587-658). */
int bfly_plan_prepare(bfly_plan* plan, uint32_t n, uint32_t batch);

/* Replaces Plan::run (plan.hpp:37, butterfly.cpp:723-749): synchronous C2C forward of host
 * buffers [batch][2n], n in [64, 4096]. */
int bfly_plan_run_c2c(bfly_plan* plan, const float* in, float* out, uint32_t n, uint32_t batch);

/* New: many synchronous host-to-host C2C requests in one call.  The reference transforms one
 * request per call (Plan::run, butterfly.cpp:723-749: upload, launch, synchronise, download),
 * so the copies of successive requests never overlap; here every request is validated first
 * (-8 before any allocation or copy, any exec_c2c length, batch*2n fp32 per buffer), then their
 * row chunks flow through an upload stream, the context stream and a download stream.  Pinned
 * host buffers reach the bidirectional PCIe bandwidth. */
typedef struct bfly_host_request {
    const float* in;       /* [batch][2n] fp32, host */
    float* out;            /* [batch][2n] fp32, host */
    uint32_t n;
    uint32_t batch;
    int32_t direction;     /* -1 forward, +1 inverse */
    float scale;
} bfly_host_request;
int bfly_plan_run_c2c_many(bfly_plan* plan, const bfly_host_request* reqs, size_t count);

/* Replaces Plan::runR2C (plan.hpp:40, butterfly.cpp:753-806): [batch][n] -> [batch][n+2],
 * n in [128, 8192]. */
int bfly_plan_run_r2c(bfly_plan* plan, const float* in, float* out, uint32_t n, uint32_t batch);

/* Replaces Plan::runC2R (plan.hpp:43, butterfly.cpp:810-850): [batch][n+2] -> [batch][n]
 * including 1/n, n in [64, 4096]. */
int bfly_plan_run_c2r(bfly_plan* plan, const float* in, float* out, uint32_t n, uint32_t batch);

/* Replaces Plan::measure (plan.hpp:45, butterfly.cpp:852-924). */
int bfly_plan_measure(bfly_plan* plan, uint32_t n, uint32_t batch, bfly_metric* out);

/* New: synchronous inverse C2C (unnormalised inverse times scale), n in [64, 4096].
 * The reference has no public inverse; it is implied by its C2R sign flip
 * (src/ascendc/fft_real.cpp:6-7). */
int bfly_plan_run_c2c_inverse(bfly_plan* plan, const float* in, float* out, uint32_t n,
                              uint32_t batch, float scale);

/* New: synchronous long C2C via four-step, n in [8192, 65536], direction -1 / +1.
 * Replaces the harness-only four-step chain (src/host/fft_check.cpp:289-362, 843-970). */
int bfly_plan_run_c2c_long(bfly_plan* plan, const float* in, float* out, uint32_t n,
                           uint32_t batch, int direction);

/* New asynchronous device-pointer entry points.  Enqueue on `stream` (a cudaStream_t; NULL is
 * the CUDA default stream, bfly_context_stream() the context's) and return without
 * synchronising.  The first call for a length builds
 * its twiddle tables (and the four-step workspace) and synchronises the context stream once;
 * make it before any stream capture. */
/* C2C, power-of-two n in [32, 65536]; n = A*2^k (A in {3, 5, 9, 15}, 2^k >= 16, n <= 12288) by
 * the prime-factor mapping in one kernel; other n = 2^a 3^b 5^c 7^d 11^e 13^f <= 12288 (2..16 included) by
 * mixed-radix Stockham passes in one kernel; any other n in [2, 8192] by Bluestein's algorithm
 * in one kernel (the reference supports powers of two only, docs/reference/support.md:14);
 * direction -1 forward / +1 inverse; output multiplied by scale. */
int bfly_plan_exec_c2c_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t n,
                             uint64_t batch, int direction, float scale, void* stream);
/* New: 2-D C2C over [batch][ny][nx] complex (rows of nx contiguous): nx-point row transforms
 * (any exec_c2c length) into d_out, then ny-point column transforms in place in d_out,
 * ny in [32, 4096]; scale applied once; batch * ny <= 2^32 - 1.  The reference has no 2-D
 * transform (docs/reference/support.md:14; docs/testing.md:20 and :120 plan range-Doppler and
 * 2-D at 256^2..2048^2 and 1024x128). */
int bfly_plan_exec_c2c_2d_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t ny,
                                uint32_t nx, uint64_t batch, int direction, float scale,
                                void* stream);
/* New: 2-D real transforms (numpy.fft.rfft2 / irfft2 layouts): [batch][ny][nx] fp32 <->
 * [batch][ny][nx/2+1] complex64; nx in the R2C / C2R envelope, ny in [32, 4096] (power of two);
 * output times scale.  r2c_2d: R2C rows then column transforms in place in d_out; c2r_2d:
 * inverse column transforms into a plan-owned buffer (d_in unchanged), then C2R rows.  The
 * reference has no 2-D transform (docs/reference/support.md:14). */
int bfly_plan_exec_r2c_2d_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t ny,
                                uint32_t nx, uint64_t batch, float scale, void* stream);
int bfly_plan_exec_c2r_2d_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t ny,
                                uint32_t nx, uint64_t batch, float scale, void* stream);
/* New: C2C along the middle axis of a contiguous [outer][n][inner] complex array (element i
 * of transform (o, c) at (o*n + i)*inner + c): inner == 1 is exec_c2c; inner > 1 needs n in
 * [32, 4096].  d_in == d_out allowed.  The reference supports contiguous rows only
 * (docs/reference/support.md:11 and docs/testing.md:21 list strided layouts as missing). */
int bfly_plan_exec_c2c_axis_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t n,
                                  uint64_t outer, uint64_t inner, int direction, float scale,
                                  void* stream);
/* New: STFT of `signals` contiguous fp32 signals of sig_len samples: frames of n samples (n a
 * power of two in [64, 8192], or even with n/2 13-smooth up to 24576) every `hop`, centred with reflect padding when center != 0
 * (sig_len > n/2; torch.stft's defaults), times d_window (n floats, 8-byte aligned, or NULL), one-sided
 * spectrum of every frame into d_out = [signals][frames][n/2+1] complex;
 * frames = center ? 1 + sig_len/hop : 1 + (sig_len-n)/hop, returned in *frames (may be NULL).
 * The reference measures STFT only as a dense-frame R2C proxy (docs/testing.md:118,
 * config/test_matrix.json); framing, window and overlap run here inside one kernel. */
int bfly_plan_exec_stft_async(bfly_plan* plan, const void* d_sig, void* d_out, uint32_t n,
                              uint64_t signals, uint64_t sig_len, uint32_t hop, int center,
                              const void* d_window, uint64_t* frames, void* stream);
/* New: inverse STFT (torch.istft), n a power of two in [64, 8192] or even with n/2 13-smooth up
 * to 8192: d_spec = [signals][frames][n/2+1] complex64 -> d_out =
 * [signals][out_len] fp32: every frame inverse-transformed (1/n), then overlap-added with the
 * window (d_window, n floats, 8-byte aligned, or NULL) and divided by the overlap-added squared window, from
 * padded position n/2 when center != 0, times scale; hop <= n; samples whose window envelope
 * is zero are written as 0.  The reference has no STFT of its own. */
int bfly_plan_exec_istft_async(bfly_plan* plan, const void* d_spec, void* d_out, uint32_t n,
                               uint64_t signals, uint32_t frames, uint32_t hop, int center,
                               const void* d_window, uint64_t out_len, float scale, void* stream);
/* New: gradients of the two calls above for autograd, one kernel each, n a power of two in
 * [64, 8192] (no counterpart in the reference, which has no STFT or autograd).
 * stft_backward: d_grad_spec = [signals][frames][n/2+1] complex64, the gradient of a real loss
 * with respect to exec_stft's output -> d_grad_sig = [signals][sig_len] fp32, the gradient with
 * respect to its signal (window multiply, overlap-add and, when center != 0, the reflect
 * padding folded back; then sig_len >= n + 2).
 * istft_backward: d_grad_out = [signals][out_len] fp32, the gradient with respect to
 * exec_istft's output -> d_grad_spec = [signals][frames][n/2+1] complex64, the gradient with
 * respect to its spectrum (envelope division, window, one-sided weights and scale included).
 * Arguments as in exec_stft / exec_istft; -8 for shapes they do not serve. */
int bfly_plan_exec_stft_backward_async(bfly_plan* plan, const void* d_grad_spec, void* d_grad_sig, uint32_t n,
                                       uint64_t signals, uint64_t sig_len, uint32_t hop, int center,
                                       const void* d_window, void* stream);
int bfly_plan_exec_istft_backward_async(bfly_plan* plan, const void* d_grad_out, void* d_grad_spec, uint32_t n,
                                        uint64_t signals, uint32_t frames, uint32_t hop, int center,
                                        const void* d_window, uint64_t out_len, float scale, void* stream);
/* R2C [batch][n] -> [batch][n/2+1] complex, n a power of two in [64, 8192], or even with n/2
 * = 2^a 3^b 5^c 7^d 11^e 13^f up to 12288 (mixed-radix passes; the reference supports powers of
 * two only); bins 0 and n/2 scaled by s_edge, the others by s_int (1, 1 for the plain transform). */
int bfly_plan_exec_r2c_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t n,
                             uint64_t batch, float s_edge, float s_int, void* stream);
/* C2R [batch][n/2+1] -> [batch][n], lengths as exec_r2c; input bins scaled by s_edge / s_int,
 * output by out_scale (1/n is numpy.fft.irfft; imaginary parts of bins 0 and n/2 ignored). */
int bfly_plan_exec_c2r_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t n,
                             uint64_t batch, float s_edge, float s_int, float out_scale,
                             void* stream);

/* New: split-BF16 tensor-core C2C on the 5th-generation tensor cores (tcgen05, fp32
 * accumulate in tensor memory): each radix-16 pass is a dense contraction with the DFT-16
 * matrix; operands split into split_terms = 2 (hi+lo, 3 products) or 3 (hi+mid+lo, 6 products)
 * bf16 terms.  n a power of two in 64..4096 (radix-16 passes on the tensor cores, a final
 * radix-2/4/8 pass in fp32 when n is not a power of 16); direction -1 / +1; output times scale; asynchronous on
 * `stream`.  The reference has no counterpart (its Cube-unit probe src/ascendc/cube_probe.cpp
 * never reached a usable matrix unit). */
int bfly_plan_exec_c2c_tc_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t n,
                                uint64_t batch, int direction, float scale, int split_terms,
                                void* stream);
/* Status word of the tensor-core launches on the current device: 0, or 1 when a bounded wait
 * for an MMA ran out (the launch then stopped early); reading clears it. */
int bfly_tc_device_status(unsigned* status);
/* Status word of the single-launch long C2C schedules on the current device: 0, bit 1 when a
 * bounded wait of the cluster kernel (one thread-block cluster per row) ran out, bit 2 when one
 * of the ring kernel (both four-step passes in one launch) did (that launch's output is
 * invalid); reading clears it.  The reference has no counterpart (its long path,
 * src/host/fft_check.cpp:843-970, is a sequence of global-memory passes). */
int bfly_long_device_status(unsigned* status);

/* New: ragged persistent launch.  One kernel launch transforms a set of requests with
 * different lengths (32..4096, powers of two), batch counts and directions; the work list is
 * built once on the device and exec is a single launch that can be captured in a CUDA graph.
 * The ragged object uses the plan's twiddle tables and must be destroyed before the plan.
 * The reference has no counterpart (it launches one kernel per transform,
 * src/framework/butterfly.cpp:743). */
typedef struct bfly_ragged bfly_ragged;
typedef struct bfly_ragged_request {
    const void* d_in;      /* [batch][n] complex64 */
    void* d_out;           /* [batch][n] complex64 */
    uint32_t n;
    int32_t direction;     /* -1 forward, +1 inverse */
    uint64_t batch;
    float scale;
    uint32_t reserved;
} bfly_ragged_request;
int bfly_ragged_create(bfly_plan* plan, const bfly_ragged_request* reqs, size_t count,
                       bfly_ragged** out);
int bfly_ragged_exec_async(bfly_ragged* ragged, void* stream);
/* tiles, resident grid and launch mode: -1 (default) one 4096-point tile per CTA, scheduled by
 * the hardware; 0 persistent CTAs with plain loads; 1, 2 persistent CTAs with bulk-copy staged
 * tiles (every input 16-byte aligned).  BFLY_RAGGED_STAGES=-1/0/1/2 overrides. */
int bfly_ragged_info(bfly_ragged* ragged, uint64_t* tiles, int* grid, int* stages);
/* Status word of the staged launches on the current device: 0, or 1 when a bounded wait for a
 * staged copy ran out (the launch then stopped early); reading clears it. */
int bfly_ragged_device_status(unsigned* status);
/* The same work list built with an explicit launch configuration: mode as above (-1, 0, 1, 2;
 * 1 and 2 need every input 16-byte aligned) and, per length, the register radix of its tiles:
 * bit (log2 n - 5) of radix8 set = 256 threads x 8 values per tile, clear = x 16 (n = 4096 has
 * only the 16-value tiles, so bit 7 must be clear).  bfly_ragged_create uses mode -1 and
 * radix8 = 0x3.  -8 for an invalid request or configuration. */
int bfly_ragged_create_config(bfly_plan* plan, const bfly_ragged_request* reqs, size_t count, int mode,
                              uint32_t radix8, bfly_ragged** out);
/* Autotuned work list (the ragged counterpart of bfly_context_select): builds the default
 * configuration, then measures the other radix of each length present and the other launch
 * modes on these very requests, and returns the fastest.  It runs the list many times: outputs
 * (and the inputs of in-place requests) are overwritten.  With a tuning cache set, the choice
 * for the same lengths, batch counts and input alignment on this GPU is reused without
 * measuring.  log may be NULL.  Returns 0, a bfly_ragged_create code, or -5 when a launch or
 * timing failed. */
int bfly_context_tune_ragged(bfly_context* ctx, bfly_plan* plan, const bfly_ragged_request* reqs, size_t count,
                             bfly_ragged** out, char* log, size_t log_cap);
/* Launch mode and radix mask of a work list. */
int bfly_ragged_config(bfly_ragged* ragged, int* mode, uint32_t* radix8);
void bfly_ragged_destroy(bfly_ragged* ragged);

/* New: long C2C (four-step, n in {8192, 16384, 32768, 65536}) that allocates no device memory,
 * for callers that cannot call cudaMalloc when they need the transform: code running while a
 * CUDA graph is captured, real-time loops that must not allocate after start-up, programs whose
 * GPU memory belongs to another allocator or budget.  No counterpart in the reference.
 * Its workspace is a fixed 32 MiB array in the library's device image (every GPU that loads
 * the library keeps it until exit), so n * batch must be <= 4,194,304 complex values; larger
 * requests return -12 before any GPU work.  No plan or context is needed: it runs on the
 * current device.  The first call on a device looks up the array addresses, loads every kernel
 * variant it can launch, builds its twiddle tables on `stream` and waits for that stream once;
 * make that first call before any stream capture (a first call on a stream that is being
 * captured returns -13 and leaves the capture untouched).  All calls share the one workspace:
 * calls that overlap on the GPU race.
 * Status: 0, -8 shape/direction, -10 null pointer, -12 too large, -13 first call on a capturing
 * stream, -1 runtime, -5 launch. */
int bfly_exec_c2c_long_noalloc(const void* d_in, void* d_out, uint32_t n, uint64_t batch,
                               int direction, float scale, void* stream);

/* Acceptance helpers with the reference's semantics (include/butterfly/reference.hpp:14-60). */
double bfly_max_rel_scaled(const float* got, const float* ref, size_t len);
float bfly_pattern_at(size_t i);
uint32_t bfly_sample_batches(uint32_t batch, uint32_t want, uint32_t* out, uint32_t max_out);

#ifdef __cplusplus
}
#endif

#endif /* BFLY_B200_H */
