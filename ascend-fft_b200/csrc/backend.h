// Device seam of the host runtime.  plan.cpp (Context / Plan / autotuner) is plain C++ and
// reaches the GPU only through these functions; backend_cuda.cu implements them on the CUDA
// runtime and the hand-written sm_100a kernels, and the CPU guard tests link a counting fake
// with failure injection instead (the pattern of the reference's tests/stubs/acl/acl_rt.h:15-53).
// Every function returns 0 on success and a nonzero CUDA-style error otherwise.
#pragma once
#include <cstddef>
#include <cstdint>

namespace bfly {
namespace backend {

// ------------------------------------------------------------------ runtime
int deviceCount(int* count);
int setDevice(int device);
int deviceName(int device, char* buf, size_t cap);
int smCount(int device, int* count);
int streamCreate(void** stream);
int streamDestroy(void* stream);
int alloc(void** ptr, size_t bytes);
int release(void* ptr);
int allocHost(void** ptr, size_t bytes);   // pinned staging buffer
int releaseHost(void* ptr);
int copyH2D(void* dst, const void* src, size_t bytes, void* stream);
int copyD2H(void* dst, const void* src, size_t bytes, void* stream);
int streamSync(void* stream);
// Opt kernel `fn` into `bytes` of dynamic shared memory on the current device (no-op at or below
// the 48 KB default); done once per (device, kernel), thread-safe.
int optInSharedMemory(const void* fn, int bytes);

// Ordering between streams (events without timing).
int eventCreate(void** event);
int eventDestroy(void* event);
int eventRecord(void* event, void* stream);
int streamWaitEvent(void* stream, void* event);   // later work on `stream` waits for `event`
int eventSync(void* event);                       // host waits for `event`
bool isPinnedHost(const void* ptr);               // page-locked (or registered) host memory

// Device-side elapsed time between start() and stop() on one stream (CUDA events).
struct Timer;
int timerCreate(Timer** timer);
int timerStart(Timer* timer, void* stream);
int timerStop(Timer* timer, void* stream, float* ms);   // synchronises the stop event
void timerDestroy(Timer* timer);

// ------------------------------------------------------------------ kernel variants
// kind: which kernel family; n: transform length (real length for R2C/C2R);
// e: complex values per thread (register radix); cta: threads per CTA.
enum Kind : int { kC2C = 0, kR2C = 1, kC2R = 2 };
bool hasVariant(int kind, uint32_t n, int e, int cta);
size_t variantSmemBytes(int kind, uint32_t n, int e, int cta);

// Twiddle tables (float2 entries), all computed in FP64 on the device.
size_t stockhamTwiddleCount(uint32_t n, int e);        // Sched<n,e>::TWSIZE (0 if none)
int buildStockhamTwiddles(void* tw, uint32_t n, int e, void* stream);
// tw[i] = exp(-2*pi*i*(i*stride mod n)/n), i < count
int buildLinearTwiddles(void* tw, int count, long long stride, long long n, void* stream);

int launchC2C(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale,
              const void* tw, int e, int cta, void* stream);
// R2C of real length n: tw = Stockham table of (n/2, e), twr = W_n^k for k = 0..n/2.
int launchR2C(const void* in, void* out, uint32_t n, uint64_t batch, const void* tw,
              const void* twr, int e, int cta, bool weighted, float sEdge, float sInt,
              void* stream);
int launchC2R(const void* in, void* out, uint32_t n, uint64_t batch, const void* tw,
              const void* twr, int e, int cta, float sEdge, float sInt, float outScale,
              void* stream);

// Four-step long C2C, n = n1 * n2.
bool hasLongSplit(uint32_t n1, uint32_t n2);
void longSplit(uint32_t n, uint32_t* n1, uint32_t* n2);   // chosen split (0,0 if none)
int longE();                                                // register radix of both passes
int launchLongA(const void* in, void* out, uint32_t n1, uint32_t n2, uint64_t batch,
                bool inverse, const void* tw1, const void* tlo, const void* thi, void* stream);
int launchLongB(const void* in, void* out, uint32_t n1, uint32_t n2, uint64_t batch,
                bool inverse, float scale, const void* tw2, void* stream);
// Load every pass-A and pass-B variant on the current device and opt each into its shared
// memory, so that later launches neither load device code nor set kernel attributes.
int prepareLongKernels();

// Long C2C as one persistent cooperative launch of the four-step schedule, the intermediate
// kept in a ring of longRingSlots() slots of `slotRows` rows each (L2-resident): `ring` holds
// min(slots, ceil(batch / slotRows)) * slotRows * n complex values, `counters` 2 * slots
// unsigned values (zeroed by the launch on `stream`).  Tables as for the four-step kernels.
bool hasLongRing(uint32_t n);
int longRingSlots();
uint32_t longRingSlotRows(uint32_t n, uint64_t batch, size_t slotBytes);
int launchLongRing(const void* in, void* out, void* ring, uint32_t slotRows, uint32_t n, uint64_t batch,
                   bool inverse, float scale, const void* tw1, const void* tw2, const void* tlo, const void* thi,
                   void* counters, void* stream);
int longRingStatus(unsigned* status, bool clear);   // nonzero *status: a bounded wait ran out

// Single-pass long C2C: one thread-block cluster per row, transpose through distributed
// shared memory (n in 8192..65536; tw1 = Stockham (n/256, 16), tw2 = Stockham (256, 16)).
// `cta` threads per CTA (256, or 512 for n >= 16384) sets the cluster size n / (16 * cta).
// Returns kLongClusterUnaligned (nothing launched) when `in` is not 16-byte aligned, which the
// TMA tensor map needs; callers then use the four-step kernels.
constexpr int kLongClusterUnaligned = 0x4c43;
bool hasLongCluster(uint32_t n, int cta);
int launchLongCluster(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale,
                      const void* tw1, const void* tw2, const void* tlo, const void* thi, int cta, void* stream);
int longClusterStatus(unsigned* status, bool clear);   // device error word of the cluster kernel; 0 on success

// C2C of n = A*B by the prime-factor (Good-Thomas) mapping: A in {3, 5, 9, 15}, B a power of two
// >= 16, n <= kPfaMaxN.  pfaSplit gives (A, B) or false; twB = Stockham table (B, 16), wA =
// W_A^m, m < A (linear table of A entries for length A).
constexpr uint32_t kPfaMaxN = 12288;
bool pfaSplit(uint32_t n, uint32_t* a, uint32_t* b);
int launchPfa(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale, const void* twB,
              const void* wA, void* stream);

// Any-length C2C (Bluestein), n in [2, kBluesteinMaxN], in one kernel per padded length M =
// bluesteinM(n) (power of two >= 2n-1, >= 64).  Tables per n: chirp (n float2), filter (M
// float2), built in FP64 on the device with an M-double2 scratch; tw = Stockham table (M, 16).
constexpr uint32_t kBluesteinMaxN = 8192;
uint32_t bluesteinM(uint32_t n);   // 0 when n is outside [2, kBluesteinMaxN]
int buildBluesteinTables(void* chirp, void* filt, void* scratch, uint32_t n, void* stream);
int launchBluestein(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale,
                    const void* tw, const void* chirp, const void* filt, void* stream);

// Mixed-radix C2C for 13-smooth lengths n = 2^a 3^b 5^c 7^d 11^e 13^f in [2, kMixedMaxN]:
// Stockham passes through shared memory in one kernel, radices 16, 8, 4, 2 and the odd /
// composite radices 3, 5, 7, 9 (3x3), 11, 13, 6, 10, 14 (2 x odd), 12 (4x3), 15 (3x5).  mixedRadix picks the passes: 16s
// for the power-of-two part, then 15s and 9s, then the remaining odd primes, each paired with one
// or two of the leftover factors 2 (6, 10, 14, 12), then 11s and 13s, then the leftover power
// of two.
// ns[p] = product of the radices before pass p; pass p >= 1 reads its twiddles W_(Ns R)^(k r)
// at tw[twoff[p] + (r-1) Ns + k], r < R, k < Ns (twsize entries, built by buildMixedTwiddles).
constexpr uint32_t kMixedMaxN = 12288;
constexpr int kMixedMaxPasses = 16;
struct MixedRadix {
    int n = 0, passes = 0, twsize = 0;
    int radix[kMixedMaxPasses] = {};
    int ns[kMixedMaxPasses] = {};
    int twoff[kMixedMaxPasses] = {};
};
inline bool mixedRadix(uint32_t n, MixedRadix* m) {
    if (n < 2 || n > kMixedMaxN) return false;
    int e[6] = {0, 0, 0, 0, 0, 0};   // exponents of 2, 3, 5, 7, 11, 13
    uint32_t rest = n;
    static constexpr uint32_t kPrime[6] = {2, 3, 5, 7, 11, 13};
    for (int i = 0; i < 6; ++i)
        while (rest % kPrime[i] == 0) {
            rest /= kPrime[i];
            ++e[i];
        }
    if (rest != 1) return false;
    if (!m) return true;
    // k16 passes of radix 16 first; the rest as below.  Every k16 from the most to none is tried
    // and the fewest passes kept (n = 10000: 10^4 rather than 16 5^4).
    auto build = [&](int k16) {
        MixedRadix r;
        r.n = (int)n;
        int f[4] = {e[0] - 4 * k16, e[1], e[2], e[3]};
        auto push = [&](int radix) {
            r.ns[r.passes] = r.passes ? r.ns[r.passes - 1] * r.radix[r.passes - 1] : 1;
            r.twoff[r.passes] = r.twsize;
            if (r.passes) r.twsize += (radix - 1) * r.ns[r.passes];
            r.radix[r.passes++] = radix;
        };
        for (int i = 0; i < k16; ++i) push(16);
        for (; f[1] >= 1 && f[2] >= 1; --f[1], --f[2]) push(15);
        for (; f[1] >= 2; f[1] -= 2) push(9);
        for (; f[3] >= 1; --f[3]) push(f[0] >= 1 ? (--f[0], 14) : 7);
        for (; f[2] >= 1; --f[2]) push(f[0] >= 1 ? (--f[0], 10) : 5);
        for (; f[1] >= 1; --f[1]) push(f[0] >= 2 ? (f[0] -= 2, 12) : f[0] >= 1 ? (--f[0], 6) : 3);
        for (int i = 0; i < e[4]; ++i) push(11);
        for (int i = 0; i < e[5]; ++i) push(13);
        for (; f[0] >= 4; f[0] -= 4) push(16);
        if (f[0] >= 1) push(1 << f[0]);
        return r;
    };
    MixedRadix best = build(e[0] / 4);
    for (int k16 = e[0] / 4 - 1; k16 >= 0; --k16) {
        const MixedRadix r = build(k16);
        if (r.passes < best.passes) best = r;
    }
    *m = best;
    return true;
}
int buildMixedTwiddles(void* tw, const MixedRadix& plan, void* stream);   // FP64 on the device
int launchMixed(const void* in, void* out, const MixedRadix& plan, uint64_t batch, bool inverse, float scale,
                const void* tw, void* stream);
// Real transforms of even n = 2M with the M-point passes `half` (M 13-smooth): R2C / C2R with
// the layouts, split and per-bin weights of launchR2C / launchC2R, and the STFT of launchStft;
// twr = W_n^k, k <= M (linear table of M + 1 entries).
int launchR2CMixed(const void* in, void* out, const MixedRadix& half, uint64_t batch, const void* tw, const void* twr,
                   float sEdge, float sInt, void* stream);
int launchC2RMixed(const void* in, void* out, const MixedRadix& half, uint64_t batch, const void* tw, const void* twr,
                   float sEdge, float sInt, float outScale, void* stream);
int launchStftMixed(const void* sig, void* out, const MixedRadix& half, uint64_t signals, uint32_t framesPerSignal,
                    uint64_t sigLen, uint64_t sigStride, uint32_t hop, bool center, const void* window,
                    const void* tw, const void* twr, void* stream);
// Inverse STFT of even non-power-of-two n <= kIstftMixedMaxN (n/2 13-smooth): the single
// kernel of launchIstft on the mixed-radix passes (arguments as launchIstft).
constexpr uint32_t kIstftMixedMaxN = 8192;
int launchIstftMixed(const void* spec, void* out, const MixedRadix& half, uint64_t signals, uint32_t frames,
                     uint32_t hop, int64_t start, uint64_t outLen, const void* window, const void* tw, const void* twr,
                     float scale, void* stream);

// STFT: `signals` real signals of sigLen samples (signal s at s*sigStride floats), frames of n
// samples every `hop` (centred with reflect padding when `center`), times `window` (n floats,
// or null for none), R2C of each frame into out[s][f][n/2+1].  n a power of two in
// [kStftMinN, kStftMaxN]; tw = Stockham table (n/2, 16), twr = W_n^k, k <= n/2.
constexpr uint32_t kStftMinN = 64, kStftMaxN = 8192;
bool hasStft(uint32_t n);
int launchStft(const void* sig, void* out, uint32_t n, uint64_t signals, uint32_t framesPerSignal,
               uint64_t sigLen, uint64_t sigStride, uint32_t hop, bool center, const void* window,
               const void* tw, const void* twr, void* stream);

// Inverse STFT in one kernel: out[s][i] = y[i + start], y[p] = sum_f w[j] x_f[j] / sum_f w[j]^2
// (j = p - f*hop in [0, n), x_f = scale/n * irfft of spec[s][f], window null = 1), zero past the
// last frame; spec = [signals][frames][n/2+1] float2, hop <= n, tables as for launchStft.
// Work split: signal s, segment c of q frames per CTA, `rows` frames per wave; istftSegments
// picks q for `slots` resident CTAs on the device.
void istftSegments(uint32_t n, int rows, uint32_t frames, uint32_t hop, uint64_t signals, uint64_t slots,
                   uint32_t* q, uint32_t* segs);
int launchIstft(const void* spec, void* out, uint32_t n, uint64_t signals, uint32_t frames, uint32_t hop,
                int64_t start, uint64_t outLen, const void* window, const void* tw, const void* twr, float scale,
                void* stream);
// Adjoints for autograd, power-of-two n in [64, 8192], one kernel each.
// STFT -> signal: gradSpec [signals][frames][n/2+1] -> gradSig [signals][sigLen] (the gradient of
// launchStft's input; centred needs sigLen >= n + 2).
int launchStftAdjoint(const void* gradSpec, void* gradSig, uint32_t n, uint64_t signals, uint32_t frames,
                      uint32_t hop, bool center, uint64_t sigLen, const void* window, const void* tw, const void* twr,
                      void* stream);
// inverse STFT -> spectrum: gradOut [signals][outLen] -> gradSpec [signals][frames][n/2+1] (the
// gradient of launchIstft's input; start and scale as that call's).
int launchIstftAdjoint(const void* gradOut, void* gradSpec, uint32_t n, uint64_t signals, uint32_t frames,
                       uint32_t hop, int64_t start, uint64_t outLen, const void* window, const void* tw,
                       const void* twr, float scale, void* stream);

// Column FFTs: ny-point transforms down the ncols columns of `mats` row-major matrices,
// element (m, i, col) at m*matStride + i*pitch + col (float2 units).  ny in 32..4096;
// tw = Stockham table (ny, 16); in == out allowed.
bool hasCols(uint32_t ny);
int launchCols(const void* in, void* out, uint32_t ny, uint32_t ncols, uint64_t pitch, uint64_t matStride,
               uint64_t mats, bool inverse, float scale, const void* tw, void* stream);

// Ragged persistent launch over a device array of RaggedEntry (ragged.h).
int raggedSmemBytes();
int raggedGrid(int device, int* grid);   // resident CTAs on the whole device
int launchRagged(const void* entries, int count, uint64_t totalTiles, int grid, void* stream);
// TMA-staged variant (inputs 16-byte aligned): `stages` = 1 or 2 staging buffers per CTA.
int raggedStagedGrid(int device, int stages, int* grid);
int launchRaggedStaged(const void* entries, int count, uint64_t totalTiles, int grid, int stages,
                       void* stream);
// One tile per CTA (grid = tiles), hardware-scheduled; tileMap = request index per tile or
// nullptr (binary search).
int launchRaggedFlat(const void* entries, int count, const void* tileMap, uint64_t totalTiles,
                     void* stream);
// Device status word of the staged launches (nonzero: a bounded wait ran out).
int raggedStatus(unsigned* status, bool clear);

// Split-BF16 tensor-core C2C (tcgen05): n a power of two in 64..4096 (radix-16 passes on the
// tensor cores, a final radix-2/4/8 pass in fp32), split = 2 or 3 bf16 terms; tw is the
// Stockham table of (n, 16).
bool hasTensorVariant(uint32_t n, int split);
size_t tensorTableBytes(int split);                            // split DFT-16 operand
int buildTensorTable(void* table, int split, void* stream);    // FP64 on the device
// twTc: twiddles of the tensor-core passes after the first, by operand row (FP64 on the device).
size_t tensorTwiddleCount(uint32_t n);
int buildTensorTwiddles(void* tw, uint32_t n, void* stream);
int launchC2CTensor(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale,
                    const void* tw, const void* twTc, const void* table, int split, void* stream);
int tensorStatus(unsigned* status, bool clear);

}  // namespace backend
}  // namespace bfly
