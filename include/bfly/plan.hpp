// bfly::Context / bfly::Plan for NVIDIA B200 (sm_100a): the C++ host API of the batched
// power-of-two fp32 FFT library.  It keeps the surface of the reference's plan API
// (include/butterfly/plan.hpp:26-91 of TruNcat3/ascend-fft) so code written against it ports
// by changing the configuration files:
//   Context::init(profile, space, kernel)  -> 0 | -1 runtime | -2 device | -3 stream |
//                                             -4 configuration | -9 already initialised
//   Context::enumerate / select / makePlan
//   Plan::prepare / run / runR2C / runC2R / measure with the same status codes:
//     0 ok, -1 kernel not available, -2 prepare, -3 alloc, -4 H2D, -5 launch, -6 sync,
//     -7 D2H (measure: acceptance failure), -8 shape / guard (checked before any allocation)
// Additions for the B200 build: inverse C2C, long C2C (four-step, 8192..65536), and the
// asynchronous device-pointer entry points exec* that never cross the host/device boundary.
#pragma once
#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace bfly {

// ---------------------------------------------------------------- H: hardware profile
struct Hardware {
    std::string gpu;            // e.g. "NVIDIA B200"
    std::string arch;           // "sm_100a"
    int deviceIndex = 0;
    int smCount = 0;
    int smemPerCta = 0;         // opt-in maximum dynamic shared memory per CTA (bytes)
    int smemPerSm = 0;
    int regsPerSm = 0;
    int maxThreadsPerSm = 0;
    long long l2Bytes = 0;
    double hbmGbs = 0;          // measured copy bandwidth, the roofline denominator

    // Throws std::exception for unreadable, malformed or invalid configuration.
    static Hardware load(const std::string& profilePath);
};

// ---------------------------------------------------------------- A: mapping
struct Mapping {
    int ctaThreads = 256;                  // threads per CTA
    std::string localExchange = "shared";  // shared (the only lowering)
    int level = 0;                         // 0 = one GPU (batch sharding lives above the plan)
    bool validate(const Hardware& hw, std::string* why) const;
};

// ---------------------------------------------------------------- P: stage plan
struct StagePlan {
    int radix = 16;                        // complex values per thread = register radix
    bool coefficientResidency = true;      // twiddle tables read through L1
    int fusionLevel = 1;                   // passes per kernel launch granularity (1 = all)
    // Dynamic shared memory of the single-pass kernel for complex length n.
    size_t smemBytes(uint32_t n, int ctaThreads) const;
};

// ---------------------------------------------------------------- L: layout
struct Layout {
    enum Pack : uint8_t { Interleaved = 0, Planar = 1 };
    Pack in = Interleaved;
    Pack out = Interleaved;
    bool contiguous = true;
};

// ---------------------------------------------------------------- F: fusion / schedule
struct Fusion {
    std::string precision = "fp32";        // fp32 | split_bf16
    std::string schedule = "stockham";     // stockham (one pass) | four_step (two passes)
};

// ---------------------------------------------------------------- Q: quality / metric
struct Metric {
    double etaUs = 0.0;       // model estimate (µs)
    double measuredUs = 0.0;  // best device time over the timed launches (µs)
    double maxRelErr = 0.0;   // maxRelScaled against the FP64 acceptance reference
    bool measuredOk = false;
};

enum class State : uint8_t { Infeasible = 0, Unverified = 1, Feasible = 2, Measured = 3 };
const char* toString(State s);

struct Candidate {
    std::string id;
    Mapping a;
    StagePlan p;
    Layout l;
    Fusion f;
    Metric q;
    State state = State::Unverified;
    std::string reason;       // why Infeasible
};

struct DesignSpace {
    std::vector<int> ctaThreads;
    std::vector<int> radices;
    std::vector<int> fusionStages;
    std::vector<int> coeffResidency;
    std::vector<std::string> localExchanges;
    std::vector<std::string> layoutsIn;
    std::vector<std::string> layoutsOut;
    std::vector<std::string> precisions;
    std::vector<std::string> schedules;
    std::string raw;

    // Strict loading; missing or malformed files or axes throw std::exception.
    static DesignSpace load(const std::string& path);
    void applyDefaults();
};

// Enumerate the Cartesian product of the space axes for a C2C transform of length n.
std::vector<Candidate> enumerate(const DesignSpace& sp, const Hardware& hw, uint32_t n,
                                 uint32_t batch);
// Non-infeasible candidates, Measured first, then ascending estimate.
std::vector<const Candidate*> rank(const std::vector<Candidate>& cs);
Metric estimate(const Hardware& hw, const Candidate& c, uint32_t n, uint32_t batch);

class Transform {
public:
    enum Kind : uint8_t { GenTwiddles, GenBitReverse, LaunchKernel, Measure } kind;
    std::string label;
};

class Context;
class Plan;

// One request of a batched host round trip (Plan::runMany): C2C of `batch` rows of length n
// (any execC2C length) from host `in` to host `out`, [batch][2n] interleaved fp32 each.
struct HostRequest {
    const float* in;
    float* out;
    uint32_t n;
    uint32_t batch;
    int direction;   // -1 forward, +1 inverse
    float scale;
};

// One request of a ragged launch: C2C of `batch` rows of length n (32..4096, power of two)
// between device buffers, direction -1 forward / +1 inverse, output times scale.
struct RaggedRequest {
    const void* in;
    void* out;
    uint32_t n;
    uint64_t batch;
    int direction;
    float scale;
};

// How a ragged work list is launched: the launch mode (see Ragged::stages) and, per length,
// the register radix of its tiles -- bit (log2 n - 5) of radix8 set: 256 threads x 8 values
// (2048 points) per tile, else x 16 (4096 points); n = 4096 has only the 16-value tiles, so
// bit 7 must be clear.  The default is the library's measured choice for a typical mix.
struct RaggedConfig {
    int mode = -1;
    uint32_t radix8 = 0x3;   // n = 32 and 64 with 8 values per thread
};

// A device work list for one persistent launch over many requests of different lengths and
// batch counts (built once; exec() is a single kernel launch, capturable in a CUDA graph).
// Must not outlive the Plan that built it (it uses that plan's twiddle tables).
class Ragged {
public:
    ~Ragged();
    int exec(void* stream) const;
    uint64_t tiles() const { return total_; }
    int grid() const { return grid_; }
    size_t requests() const { return count_; }
    // Launch mode: -1 (default) one tile per CTA, scheduled by the hardware; 0 persistent CTAs
    // with plain loads; 1 or 2 persistent CTAs with tiles staged in shared memory by bulk copies
    // (all inputs 16-byte aligned).  The environment variable BFLY_RAGGED_STAGES overrides.
    int stages() const { return stages_; }
    // The launch mode and per-length radices this work list was built with.
    RaggedConfig config() const { return RaggedConfig{stages_, radix8_}; }
    // True when every input is 16-byte aligned (the staged modes need it).
    bool aligned() const { return aligned_; }
    // Device status of staged launches: 0, or 1 when a bounded wait ran out (then cleared).
    static int deviceStatus(unsigned* status);

private:
    friend class Plan;
    Ragged() = default;
    void* entries_ = nullptr;
    void* tileMap_ = nullptr;   // request index per tile (one-tile-per-CTA mode)
    size_t count_ = 0;
    uint64_t total_ = 0;
    int grid_ = 0;
    int stages_ = 0;
    uint32_t radix8_ = 0;
    bool aligned_ = false;
};

class Plan {
public:
    ~Plan();
    const Candidate& candidate() const { return cand_; }
    const std::vector<Transform>& transforms() const { return tf_; }

    // Build (idempotently) the FP64-generated twiddle tables for a C2C of length n.
    int prepare(uint32_t n, uint32_t batch = 0xFFFFFFFFu);
    // Synchronous host-pointer entry points (reference semantics and envelopes):
    //   run     C2C forward, n in [64, 4096], in/out [batch][2n]
    //   runR2C  in [batch][n] real -> out [batch][n+2], n in [128, 8192]
    //   runC2R  in [batch][n+2] -> out [batch][n] real incl. 1/n, n in [64, 4096]
    // batch > 0, non-null pointers, batch*2n <= 2^32-1; otherwise -8 before any allocation.
    int run(const float* in, float* out, uint32_t n, uint32_t batch);
    // Many host-to-host C2C requests in one synchronous call: every request is validated first
    // (-8 before any allocation or copy), then their row chunks flow through an upload stream,
    // the context stream and a download stream, so the copies of different requests overlap
    // each other and the kernels.  Host buffers should be pinned for full PCIe bandwidth.
    int runMany(const HostRequest* reqs, size_t count);
    int runR2C(const float* in, float* out, uint32_t n, uint32_t batch);
    int runC2R(const float* in, float* out, uint32_t n, uint32_t batch);
    int measure(uint32_t n, uint32_t batch, Metric* out);

    // B200 additions (synchronous, host pointers)
    int runInverse(const float* in, float* out, uint32_t n, uint32_t batch, float scale);
    int runLong(const float* in, float* out, uint32_t n, uint32_t batch, int direction);

    // Asynchronous device-pointer entry points: enqueue on `stream` (a cudaStream_t; nullptr is
    // the CUDA default stream, stream() the context stream) and return; no host
    // synchronisation, no host<->device copies.
    //   direction -1 forward, +1 inverse; scale multiplies the output.
    //   n in [32, 16384] single pass, [8192, 65536] four-step (workspace grown on demand);
    //   n = A * 2^k (A in {3, 5, 9, 15}, 2^k >= 16, n <= 12288) by the prime-factor mapping in
    //   one kernel; other n = 2^a 3^b 5^c 7^d 11^e 13^f <= 12288 (2..16 included) by mixed-radix Stockham
    //   passes in one kernel; any other n in [2, 8192] by Bluestein's algorithm in one kernel
    //   (the first call for a length builds its tables).
    int execC2C(const void* dIn, void* dOut, uint32_t n, uint64_t batch, int direction,
                float scale, void* stream);
    // 2-D C2C over [batch][ny][nx] complex, rows of nx contiguous: nx-point row transforms
    // (any execC2C length) into dOut, then ny-point column transforms in place in dOut
    // (ny in [32, 4096]); scale applied once.  batch * ny <= 2^32 - 1.
    int execC2C2D(const void* dIn, void* dOut, uint32_t ny, uint32_t nx, uint64_t batch,
                  int direction, float scale, void* stream);
    // 2-D real transforms over [batch][ny][nx] real <-> [batch][ny][nx/2+1] complex (numpy.fft
    // rfft2 / irfft2 layouts), nx as execR2C / execC2R, ny in [32, 4096] (power of two):
    //   execR2C2D: R2C rows into dOut, column transforms in place; output times scale.
    //   execC2R2D: inverse column transforms of dIn into a plan-owned buffer (dIn is not
    //   modified), then C2R rows; output times scale (1/(ny*nx) = numpy.fft.irfft2).  Imaginary
    //   parts of each row's bins 0 and nx/2 after the column pass are ignored, as in execC2R.
    int execR2C2D(const void* dIn, void* dOut, uint32_t ny, uint32_t nx, uint64_t batch, float scale, void* stream);
    int execC2R2D(const void* dIn, void* dOut, uint32_t ny, uint32_t nx, uint64_t batch, float scale, void* stream);
    // C2C along the middle axis of a contiguous [outer][n][inner] complex array: element i of
    // transform (o, c) at (o*n + i)*inner + c.  inner == 1 is execC2C (n in [32, 65536]);
    // inner > 1 runs the column kernel (n in [32, 4096]).  dIn == dOut allowed.
    int execC2CAxis(const void* dIn, void* dOut, uint32_t n, uint64_t outer, uint64_t inner,
                    int direction, float scale, void* stream);
    // STFT of `signals` contiguous real signals of sigLen fp32 samples: frames of n samples
    // (n a power of two in [64, 8192], or even with n/2 13-smooth) every `hop`, centred with reflect padding when
    // `center` (then sigLen > n/2), times dWindow (n floats, or null), R2C of every frame into
    // dOut = [signals][frames][n/2+1] complex, frames = center ? 1 + sigLen/hop
    // : 1 + (sigLen-n)/hop.  *framesOut receives the frame count (may be null).
    int execStft(const void* dSig, void* dOut, uint32_t n, uint64_t signals, uint64_t sigLen, uint32_t hop,
                 bool center, const void* dWindow, uint64_t* framesOut, void* stream);
    // Inverse STFT (torch.istft): dSpec = [signals][frames][n/2+1] complex -> dOut =
    // [signals][outLen] fp32 in one kernel: every frame inverse-transformed (1/n), windowed and
    // overlap-added, out[i] = sum_f w[j] frame_f[j] / sum_f w[j]^2 at padded position
    // i + (center ? n/2 : 0), times `scale`; hop <= n; n a power of two in [64, 8192] or even
    // with n/2 13-smooth up to 8192.  Samples with a zero window envelope, and those past the
    // last frame, are 0.
    int execIstft(const void* dSpec, void* dOut, uint32_t n, uint64_t signals, uint32_t frames, uint32_t hop,
                  bool center, const void* dWindow, uint64_t outLen, float scale, void* stream);
    // Gradients for autograd, in one kernel each (n a power of two in [64, 8192]):
    // execStftBackward: dGradSpec = dL/d(execStft's output) -> dGradSig = dL/d(its signal),
    // the window multiply, overlap-add and reflect fold of a centred STFT included (centred:
    // sigLen >= n + 2); execIstftBackward: dGradOut = dL/d(execIstft's output) -> dGradSpec =
    // dL/d(its spectrum), the envelope division included.  Arguments mean what they mean in
    // execStft / execIstft; -8 for shapes these kernels do not serve.
    int execStftBackward(const void* dGradSpec, void* dGradSig, uint32_t n, uint64_t signals, uint64_t sigLen,
                         uint32_t hop, bool center, const void* dWindow, void* stream);
    int execIstftBackward(const void* dGradOut, void* dGradSpec, uint32_t n, uint64_t signals, uint32_t frames,
                          uint32_t hop, bool center, const void* dWindow, uint64_t outLen, float scale, void* stream);
    // R2C [batch][n] -> [batch][n/2+1] complex, bins scaled by (sEdge at 0 and n/2, sInt
    // elsewhere); sEdge = sInt = 1 is the plain transform.  n a power of two in [64, 8192]
    // (single-pass team kernels), or even with n/2 = 2^a 3^b 5^c 7^d 11^e 13^f <= 12288
    // (mixed-radix passes of n/2 with the split fused); the same lengths for execC2R.
    int execR2C(const void* dIn, void* dOut, uint32_t n, uint64_t batch, float sEdge,
                float sInt, void* stream);
    // C2R [batch][n/2+1] -> [batch][n]; input bins scaled by sEdge/sInt, output by outScale
    // (1/n = numpy.fft.irfft).
    int execC2R(const void* dIn, void* dOut, uint32_t n, uint64_t batch, float sEdge,
                float sInt, float outScale, void* stream);

    // Split-BF16 tensor-core C2C (5th-generation tensor cores, fp32 accumulate): every radix-16
    // pass is a dense contraction with the DFT-16 matrix, operands split into `splitTerms` = 2
    // (hi+lo, 3 products) or 3 (hi+mid+lo, 6 products) bf16 terms.  n a power of two in
    // 64..4096 (radix-16 passes on the tensor cores, a final radix-2/4/8 pass in fp32).
    int execC2CTensor(const void* dIn, void* dOut, uint32_t n, uint64_t batch, int direction,
                      float scale, int splitTerms, void* stream);
    // Device status of the tensor-core launches: 0, or 1 when a bounded MMA wait ran out.
    static int tensorStatus(unsigned* status);
    static int longStatus(unsigned* status);   // cluster long-C2C kernel, same convention

    // Build a ragged persistent launch over `count` requests; *status receives 0 or a code
    // (-8 invalid request or configuration, -2 table build, -3 alloc, -4 upload, -1 runtime).
    // Without `config` the default applies (BFLY_RAGGED_STAGES=-1/0/1/2 overrides its mode);
    // a staged mode (1, 2) with an input that is not 16-byte aligned is invalid.
    std::unique_ptr<Ragged> makeRagged(const RaggedRequest* reqs, size_t count, int* status,
                                       const RaggedConfig* config = nullptr);
    // Device time of one launch of `rg` (CUDA events on the plan stream around chains of
    // back-to-back launches of ~1 ms, best of 3, after ~3 ms of untimed launches), or a
    // negative code.  Runs the work list:
    // every output -- and an in-place request's input -- is overwritten.
    double timeRagged(const Ragged& rg);

    void* stream() const { return stream_; }

private:
    friend class Context;
    explicit Plan(Candidate c);
    struct Impl;
    bool validShape(uint32_t n, uint32_t batch, int kind) const;
    int prepareC2C(uint32_t n, int e);
    int prepareReal(uint32_t n);
    int prepareLong(uint32_t n);
    int prepareBluestein(uint32_t n);
    int preparePfa(uint32_t n);
    int prepareMixed(uint32_t n);
    int prepareAnyLength(uint32_t n);   // tables of whichever kernel execC2C runs for n (not 2^k >= 32)
    int resolve(int kind, uint32_t n, int* e, int* cta) const;
    int execC2CWith(const void* dIn, void* dOut, uint32_t n, uint64_t batch, int direction,
                    float scale, void* stream, void* work);
    static constexpr int kColsE = 16;   // complex values per thread of the column kernels
    int execCols(const void* dIn, void* dOut, uint32_t n, uint64_t mats, uint32_t cols, uint64_t pitch,
                 bool inverse, float scale, void* stream);
    // Upload / enqueue / download of host buffers, pipelined over row chunks on several
    // streams for large batches.  enqueue(dIn, dOut, firstRow, rows, stream) -> exec status.
    template <class Enqueue>
    int roundTrip(const float* in, size_t inRowBytes, float* out, size_t outRowBytes,
                  uint32_t batch, Enqueue&& enqueue);
    Candidate cand_;
    std::vector<Transform> tf_;
    std::unique_ptr<Impl> impl_;
    void* stream_ = nullptr;   // owned by the Context
};

class Context {
public:
    Context();
    ~Context();

    // Configuration errors return -4; repeated initialisation returns -9.
    // kernelPath: "builtin" (or empty) selects the kernels compiled into this library;
    // any other value must name an existing file (the library itself), else makePlan fails.
    int init(const std::string& profilePath, const std::string& spacePath,
             const std::string& kernelPath);
    // Same, with the profile's device_index replaced by `device` (one process per GPU).
    int init(const std::string& profilePath, const std::string& spacePath,
             const std::string& kernelPath, int device);
    const Hardware& hardware() const { return hw_; }
    const DesignSpace& space() const { return sp_; }
    const std::string& kernelPath() const { return kernelPath_; }

    std::vector<Candidate> enumerate(uint32_t n, uint32_t batch) const;
    // Autotuner: rank by estimate, build and measure candidates until topK pass the FP64
    // acceptance check, keep the fastest.  With a tuning cache set, a cached choice for
    // (gpu, n, batch) is returned without measuring and new choices are persisted.
    std::unique_ptr<Plan> select(uint32_t n, uint32_t batch, int topK = 3,
                                 std::string* log = nullptr);
    std::unique_ptr<Plan> makePlan(const Candidate& c);
    // Autotuner of the ragged launch: build the work list on `plan` with the default
    // configuration, then measure the other register radix of each length present (largest
    // share of points first) and the other launch modes, each timed next to the incumbent
    // (candidate, incumbent, incumbent, candidate) and kept only when the whole list runs >= 1%
    // faster in two such comparisons; returns the fastest.  Executes the list many times
    // (outputs, and in-place inputs, are overwritten).  With a tuning cache set, a cached choice
    // for the same lengths, batch counts and input alignment on this GPU is built without
    // measuring, and new choices are persisted.  *status as Plan::makeRagged, -5 when a launch
    // or a timing fails.
    std::unique_ptr<Ragged> tuneRagged(Plan& plan, const RaggedRequest* reqs, size_t count,
                                       int* status, std::string* log = nullptr);
    // Persist autotuned choices in a JSON file; "" disables.
    void setTuningCache(const std::string& path) { tuningCache_ = path; }
    void* stream() const;

private:
    Hardware hw_;
    DesignSpace sp_;
    std::string kernelPath_;
    std::string tuningCache_;
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

// ---------------------------------------------------------------- acceptance helpers
// FP64 reference transforms used by Plan::measure's acceptance check (outputs rounded to fp32),
// with the semantics of the reference's include/butterfly/reference.hpp.
void refFftF32(const float* in, float* out, uint32_t n);
void refR2CF32(const float* in, float* out, uint32_t n);
void refC2RF32(const float* in, float* out, uint32_t n);
// max|got-ref| / max(1, max|ref|) over float components; non-finite -> infinity.
double maxRelScaled(const float* got, const float* ref, size_t len);
float patternAt(size_t i);
uint32_t sampleBatches(uint32_t batch, uint32_t want, uint32_t* out, uint32_t maxOut);

}  // namespace bfly
