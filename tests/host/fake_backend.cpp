// CPU fake of the device seam (ascend-fft_b200/csrc/backend.h) for host-runtime tests.
// "Device memory" is host memory, copies are memcpy, kernels compute a direct DFT on the
// host, and every call is counted with one-shot failure injection -- the pattern of the
// reference's tests/stubs/acl/acl_rt.h:15-53.  Test infrastructure only.
#include "backend.h"
#include "ragged.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace fake {
int allocations = 0, releases = 0, copies = 0, launches = 0, syncs = 0;
int failAllocation = 0, failCopy = 0, failLaunch = 0, failSync = 0;   // 1-based call index
int streamsCreated = 0, streamsDestroyed = 0;
int deviceCountValue = 1;
bool pageableHost = false;   // report host buffers as pageable (staged round trips)
float timerMs = 0.01f;   // reported time per launch
int timedExtra = 0;       // extra launch-equivalents of time, added by costed fake kernels
int raggedCost16 = 0;     // time of a ragged launch: + this many launches per 16-value request
std::vector<const void*> h2dSources;   // source pointer of every host-to-device copy, in issue order
}  // namespace fake

namespace bfly {
namespace backend {

namespace {
using cd = std::complex<double>;

// direct DFT of one row (sign -1 forward), host reference for the fake kernels
void dft(const float* in, float* out, uint32_t n, int sign, float scale) {
    std::vector<cd> x(n), y(n);
    for (uint32_t i = 0; i < n; ++i) x[i] = cd(in[2 * i], in[2 * i + 1]);
    for (uint32_t k = 0; k < n; ++k) {
        cd acc = 0;
        for (uint32_t j = 0; j < n; ++j) {
            const double a = sign * 2.0 * M_PI * (double)(((uint64_t)j * k) % n) / (double)n;
            acc += x[j] * cd(std::cos(a), std::sin(a));
        }
        y[k] = acc * (double)scale;
    }
    for (uint32_t k = 0; k < n; ++k) {
        out[2 * k] = (float)y[k].real();
        out[2 * k + 1] = (float)y[k].imag();
    }
}

int launch() {
    ++fake::launches;
    return fake::launches == fake::failLaunch ? 1 : 0;
}
bool known(int e, int cta, uint32_t n) {
    if ((e != 8 && e != 16) || n < 2u * (uint32_t)e || (n & (n - 1))) return false;
    const uint32_t T = n / (uint32_t)e;
    return (cta == 128 || cta == 256 || cta == 512 || cta == 1024) && T <= (uint32_t)cta &&
           (cta == 1024) == (T == 1024);
}
}  // namespace

int deviceCount(int* count) { *count = fake::deviceCountValue; return 0; }
int setDevice(int) { return 0; }
int deviceName(int, char* buf, size_t cap) { std::strncpy(buf, "fake", cap); return 0; }
int smCount(int, int* count) { *count = 148; return 0; }
int streamCreate(void** s) { ++fake::streamsCreated; *s = reinterpret_cast<void*>(0x1); return 0; }
int streamDestroy(void*) { ++fake::streamsDestroyed; return 0; }
int eventCreate(void** e) { *e = reinterpret_cast<void*>(0x2); return 0; }
int eventDestroy(void*) { return 0; }
int eventRecord(void*, void*) { return 0; }
int streamWaitEvent(void*, void*) { return 0; }
int eventSync(void*) { return 0; }
bool isPinnedHost(const void*) { return !fake::pageableHost; }
int alloc(void** p, size_t bytes) {
    ++fake::allocations;
    if (fake::allocations == fake::failAllocation) { *p = nullptr; return 2; }
    *p = std::malloc(bytes ? bytes : 1);
    return *p ? 0 : 2;
}
int release(void* p) { ++fake::releases; std::free(p); return 0; }
int allocHost(void** p, size_t bytes) { *p = std::malloc(bytes); return *p ? 0 : 2; }
int releaseHost(void* p) { std::free(p); return 0; }
static int copyBytes(void* dst, const void* src, size_t bytes) {
    ++fake::copies;
    if (fake::copies == fake::failCopy || !dst || !src) return 1;
    std::memcpy(dst, src, bytes);
    return 0;
}
int copyH2D(void* dst, const void* src, size_t bytes, void*) {
    fake::h2dSources.push_back(src);
    return copyBytes(dst, src, bytes);
}
int copyD2H(void* dst, const void* src, size_t bytes, void*) { return copyBytes(dst, src, bytes); }
int streamSync(void*) {
    ++fake::syncs;
    return fake::syncs == fake::failSync ? 1 : 0;
}

// Elapsed time: timerMs per kernel launched between start and stop (at least one).
struct Timer { int launchesAtStart; };
int timerCreate(Timer** t) { *t = new Timer{0}; return 0; }
int timerStart(Timer* t, void*) { t->launchesAtStart = fake::launches + fake::timedExtra; return 0; }
int timerStop(Timer* t, void*, float* ms) {
    const int k = fake::launches + fake::timedExtra - t->launchesAtStart;
    *ms = fake::timerMs * (float)(k > 1 ? k : 1);
    return 0;
}
void timerDestroy(Timer* t) { delete t; }

bool hasVariant(int kind, uint32_t n, int e, int cta) {
    if (kind == kC2C) return n >= 32 && n <= 16384 && known(e, cta, n);
    return n >= 64 && n <= 8192 && known(e, cta, n / 2);
}
size_t variantSmemBytes(int, uint32_t n, int, int) { return (size_t)n * 9; }

size_t stockhamTwiddleCount(uint32_t n, int) { return n; }
int buildStockhamTwiddles(void* tw, uint32_t n, int, void*) {
    std::memset(tw, 0, (size_t)n * 8);
    return launch();
}
int buildLinearTwiddles(void* tw, int count, long long, long long, void*) {
    std::memset(tw, 0, (size_t)count * 8);
    return launch();
}

int launchC2C(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale,
              const void*, int, int, void*) {
    if (int r = launch()) return r;
    for (uint64_t b = 0; b < batch; ++b)
        dft((const float*)in + b * 2 * n, (float*)out + b * 2 * n, n, inverse ? 1 : -1, scale);
    return 0;
}
int launchR2C(const void*, void*, uint32_t, uint64_t, const void*, const void*, int, int, bool,
              float, float, void*) {
    return launch();
}
// Direct inverse real DFT (numpy.fft.irfft semantics: imaginary parts of bins 0 and n/2 ignored).
static void c2rDirect(const void* in, void* out, uint32_t n, uint64_t batch, float sEdge, float sInt,
                      float outScale) {
    const uint32_t m = n / 2;
    for (uint64_t b = 0; b < batch; ++b) {
        const float* X = (const float*)in + b * 2 * (m + 1);
        float* x = (float*)out + b * n;
        for (uint32_t j = 0; j < n; ++j) {
            double acc = sEdge * (X[0] + ((j & 1) ? -X[2 * m] : X[2 * m]));
            for (uint32_t k = 1; k < m; ++k) {
                const double a = 2 * M_PI * (double)(((uint64_t)j * k) % n) / n;
                acc += 2.0 * sInt * (X[2 * k] * std::cos(a) - X[2 * k + 1] * std::sin(a));
            }
            x[j] = (float)(acc * outScale);
        }
    }
}

int launchC2R(const void* in, void* out, uint32_t n, uint64_t batch, const void*, const void*, int, int,
              float sEdge, float sInt, float outScale, void*) {
    if (int r = launch()) return r;
    c2rDirect(in, out, n, batch, sEdge, sInt, outScale);
    return 0;
}

bool hasLongSplit(uint32_t n1, uint32_t n2) { return n1 >= 32 && n1 <= 256 && n2 == 256; }
void longSplit(uint32_t n, uint32_t* n1, uint32_t* n2) {
    *n1 = *n2 = 0;
    if (n >= 8192 && n <= 65536 && !(n & (n - 1))) { *n2 = 256; *n1 = n / 256; }
}
int longE() { return 16; }
int launchLongA(const void* in, void* out, uint32_t n1, uint32_t n2, uint64_t batch, bool,
                const void*, const void*, const void*, void*) {
    if (int r = launch()) return r;
    std::memcpy(out, in, (size_t)n1 * n2 * batch * 8);
    return 0;
}
int launchLongB(const void* in, void* out, uint32_t n1, uint32_t n2, uint64_t batch, bool inverse,
                float scale, const void*, void*) {
    if (int r = launch()) return r;
    const uint32_t n = n1 * n2;
    for (uint64_t b = 0; b < batch; ++b)
        dft((const float*)in + b * 2 * n, (float*)out + b * 2 * n, n, inverse ? 1 : -1, scale);
    return 0;
}

bool pfaSplit(uint32_t n, uint32_t* a, uint32_t* b) {
    *a = *b = 0;
    for (uint32_t A : {3u, 5u, 9u, 15u})
        if (n % A == 0 && n / A >= 16 && !((n / A) & (n / A - 1)) && n <= kPfaMaxN) {
            *a = A;
            *b = n / A;
        }
    return *a != 0;
}
int launchPfa(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale, const void*,
              const void*, void*) {
    uint32_t a = 0, b = 0;
    if (!pfaSplit(n, &a, &b)) return 1;
    if (int r = launch()) return r;
    for (uint64_t r = 0; r < batch; ++r)
        dft((const float*)in + r * 2 * n, (float*)out + r * 2 * n, n, inverse ? 1 : -1, scale);
    return 0;
}

uint32_t bluesteinM(uint32_t n) {
    if (n < 2 || n > kBluesteinMaxN) return 0;
    uint32_t m = 64;
    while (m < 2 * n - 1) m <<= 1;
    return m;
}
int buildBluesteinTables(void*, void*, void*, uint32_t n, void*) { return bluesteinM(n) ? launch() : 1; }
int launchBluestein(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale,
                    const void*, const void*, const void*, void*) {
    if (!bluesteinM(n)) return 1;
    if (int r = launch()) return r;
    for (uint64_t b = 0; b < batch; ++b)
        dft((const float*)in + b * 2 * n, (float*)out + b * 2 * n, n, inverse ? 1 : -1, scale);
    return 0;
}

int buildMixedTwiddles(void*, const MixedRadix& plan, void*) { return plan.passes > 0 ? launch() : 1; }
int launchMixed(const void* in, void* out, const MixedRadix& plan, uint64_t batch, bool inverse, float scale,
                const void*, void*) {
    if (!mixedRadix((uint32_t)plan.n, nullptr)) return 1;
    if (int r = launch()) return r;
    const uint32_t n = (uint32_t)plan.n;
    for (uint64_t b = 0; b < batch; ++b)
        dft((const float*)in + b * 2 * n, (float*)out + b * 2 * n, n, inverse ? 1 : -1, scale);
    return 0;
}

// Real transforms of even n = 2M by direct DFTs (bins 0..M; weights as launchR2C / launchC2R).
int launchR2CMixed(const void* in, void* out, const MixedRadix& half, uint64_t batch, const void*, const void*,
                   float sEdge, float sInt, void*) {
    if (!mixedRadix((uint32_t)half.n, nullptr)) return 1;
    if (int r = launch()) return r;
    const uint32_t m = (uint32_t)half.n, n = 2 * m;
    std::vector<float> z(2 * n), spec(2 * n);
    for (uint64_t b = 0; b < batch; ++b) {
        const float* x = (const float*)in + b * n;
        for (uint32_t j = 0; j < n; ++j) {
            z[2 * j] = x[j];
            z[2 * j + 1] = 0.f;
        }
        dft(z.data(), spec.data(), n, -1, 1.f);
        float* o = (float*)out + b * 2 * (m + 1);
        for (uint32_t k = 0; k <= m; ++k) {
            const float w = (k == 0 || k == m) ? sEdge : sInt;
            o[2 * k] = spec[2 * k] * w;
            o[2 * k + 1] = spec[2 * k + 1] * w;
        }
    }
    return 0;
}
int launchC2RMixed(const void* in, void* out, const MixedRadix& half, uint64_t batch, const void*, const void*,
                   float sEdge, float sInt, float outScale, void*) {
    if (!mixedRadix((uint32_t)half.n, nullptr)) return 1;
    if (int r = launch()) return r;
    c2rDirect(in, out, 2 * (uint32_t)half.n, batch, sEdge, sInt, outScale);
    return 0;
}
int launchStftMixed(const void* sig, void* out, const MixedRadix& half, uint64_t signals, uint32_t framesPerSignal,
                    uint64_t sigLen, uint64_t sigStride, uint32_t hop, bool center, const void* window, const void*,
                    const void*, void*) {
    if (!mixedRadix((uint32_t)half.n, nullptr)) return 1;
    if (int r = launch()) return r;
    const uint32_t m = (uint32_t)half.n, n = 2 * m;
    const float* x = (const float*)sig;
    const float* w = (const float*)window;
    std::vector<float> frame(2 * n), spec(2 * n);
    for (uint64_t s = 0; s < signals; ++s)
        for (uint32_t f = 0; f < framesPerSignal; ++f) {
            const long long start = (long long)f * hop - (center ? m : 0);
            for (uint32_t j = 0; j < n; ++j) {
                long long i = start + j;
                if (i < 0) i = -i;
                if (i >= (long long)sigLen) i = 2 * ((long long)sigLen - 1) - i;
                frame[2 * j] = x[s * sigStride + i] * (w ? w[j] : 1.f);
                frame[2 * j + 1] = 0.f;
            }
            dft(frame.data(), spec.data(), n, -1, 1.f);
            std::memcpy((float*)out + 2 * ((s * framesPerSignal + f) * (m + 1)), spec.data(), (m + 1) * 8);
        }
    return 0;
}

bool hasStft(uint32_t n) { return n >= kStftMinN && n <= kStftMaxN && !(n & (n - 1)); }
int launchStft(const void* sig, void* out, uint32_t n, uint64_t signals, uint32_t framesPerSignal,
               uint64_t sigLen, uint64_t sigStride, uint32_t hop, bool center, const void* window,
               const void*, const void*, void*) {
    if (!hasStft(n)) return 1;
    if (int r = launch()) return r;
    const float* x = (const float*)sig;
    const float* w = (const float*)window;
    std::vector<float> frame(2 * n), spec(2 * n);
    for (uint64_t s = 0; s < signals; ++s)
        for (uint32_t f = 0; f < framesPerSignal; ++f) {
            const long long start = (long long)f * hop - (center ? n / 2 : 0);
            for (uint32_t j = 0; j < n; ++j) {
                long long i = start + j;
                if (i < 0) i = -i;
                if (i >= (long long)sigLen) i = 2 * ((long long)sigLen - 1) - i;
                frame[2 * j] = x[s * sigStride + i] * (w ? w[j] : 1.f);
                frame[2 * j + 1] = 0.f;
            }
            dft(frame.data(), spec.data(), n, -1, 1.f);
            float* o = (float*)out + 2 * ((s * framesPerSignal + f) * (n / 2 + 1));
            std::memcpy(o, spec.data(), (n / 2 + 1) * 8);
        }
    return 0;
}

void istftSegments(uint32_t n, int rows, uint32_t frames, uint32_t hop, uint64_t signals, uint64_t slots,
                   uint32_t* q, uint32_t* segs) {
    *q = frames;
    *segs = 1;
    (void)n, (void)rows, (void)hop, (void)signals, (void)slots;
}

// C2R of every frame (scale/n), windowed overlap-add, division by the squared-window envelope.
static void istftDirect(const void* spec, void* out, uint32_t n, uint64_t signals, uint32_t frames, uint32_t hop,
                        int64_t start, uint64_t outLen, const void* window, float scale);
int launchIstftMixed(const void* spec, void* out, const MixedRadix& half, uint64_t signals, uint32_t frames,
                     uint32_t hop, int64_t start, uint64_t outLen, const void* window, const void*, const void*,
                     float scale, void*) {
    const uint32_t n = 2 * (uint32_t)half.n;
    if (!mixedRadix((uint32_t)half.n, nullptr) || n > kIstftMixedMaxN || hop == 0 || hop > n || frames == 0) return 1;
    if (int r = launch()) return r;
    istftDirect(spec, out, n, signals, frames, hop, start, outLen, window, scale);
    return 0;
}
int launchIstft(const void* spec, void* out, uint32_t n, uint64_t signals, uint32_t frames, uint32_t hop,
                int64_t start, uint64_t outLen, const void* window, const void*, const void*, float scale, void*) {
    if (!hasStft(n) || hop == 0 || hop > n || frames == 0) return 1;
    if (int r = launch()) return r;
    istftDirect(spec, out, n, signals, frames, hop, start, outLen, window, scale);
    return 0;
}
// Adjoints by their definitions (direct sums; the device kernels are checked against torch).
int launchStftAdjoint(const void* gradSpec, void* gradSig, uint32_t n, uint64_t signals, uint32_t frames,
                      uint32_t hop, bool center, uint64_t sigLen, const void* window, const void*, const void*,
                      void*) {
    if (!hasStft(n) || hop == 0 || hop > n || frames == 0 || (center && sigLen < (uint64_t)n + 2)) return 1;
    if (int r = launch()) return r;
    const float* w = (const float*)window;
    std::vector<float> fr((size_t)frames * n);
    for (uint64_t s = 0; s < signals; ++s) {
        c2rDirect((const float*)gradSpec + s * frames * (n + 2), fr.data(), n, frames, 1.f, 0.5f, 1.f);
        float* g = (float*)gradSig + s * sigLen;
        for (uint64_t i = 0; i < sigLen; ++i) g[i] = 0.f;
        for (uint32_t f = 0; f < frames; ++f)
            for (uint32_t j = 0; j < n; ++j) {
                long long i = (long long)f * hop + j - (center ? n / 2 : 0);
                if (i < 0) i = -i;
                if (i >= (long long)sigLen) i = 2 * ((long long)sigLen - 1) - i;
                g[i] += (w ? w[j] : 1.f) * fr[(size_t)f * n + j];
            }
    }
    return 0;
}
int launchIstftAdjoint(const void* gradOut, void* gradSpec, uint32_t n, uint64_t signals, uint32_t frames,
                       uint32_t hop, int64_t start, uint64_t outLen, const void* window, const void*, const void*,
                       float scale, void*) {
    if (!hasStft(n) || hop == 0 || hop > n || frames == 0) return 1;
    if (int r = launch()) return r;
    const float* w = (const float*)window;
    const float c = scale / (float)n;
    std::vector<float> frame(2 * n), spec(2 * n);
    for (uint64_t s = 0; s < signals; ++s)
        for (uint32_t f = 0; f < frames; ++f) {
            for (uint32_t j = 0; j < n; ++j) {
                const long long p = (long long)f * hop + j, i = p - start;
                double env = 0;
                for (uint32_t g = 0; g < frames; ++g) {
                    const long long jj = p - (long long)g * hop;
                    if (jj >= 0 && jj < (long long)n) env += (w ? w[jj] : 1.0) * (w ? w[jj] : 1.0);
                }
                const float h = (i >= 0 && i < (long long)outLen && env > 0)
                                    ? (float)(((const float*)gradOut)[s * outLen + i] / env) : 0.f;
                frame[2 * j] = h * (w ? w[j] : 1.f);
                frame[2 * j + 1] = 0.f;
            }
            dft(frame.data(), spec.data(), n, -1, 1.f);
            float* o = (float*)gradSpec + 2 * ((s * frames + f) * (n / 2 + 1));
            for (uint32_t k = 0; k <= n / 2; ++k) {
                const float wt = (k == 0 || k == n / 2) ? c : 2.f * c;
                o[2 * k] = spec[2 * k] * wt;
                o[2 * k + 1] = spec[2 * k + 1] * wt;
            }
        }
    return 0;
}

static void istftDirect(const void* spec, void* out, uint32_t n, uint64_t signals, uint32_t frames, uint32_t hop,
                        int64_t start, uint64_t outLen, const void* window, float scale) {
    const float* w = (const float*)window;
    std::vector<float> fr((size_t)frames * n);
    for (uint64_t s = 0; s < signals; ++s) {
        c2rDirect((const float*)spec + s * frames * (n + 2), fr.data(), n, frames, 1.f, 1.f, scale / n);
        for (uint64_t i = 0; i < outLen; ++i) {
            const long long p = (long long)i + start;
            double acc = 0, env = 0;
            for (uint32_t f = 0; f < frames; ++f) {
                const long long j = p - (long long)f * hop;
                if (j < 0 || j >= (long long)n) continue;
                const double wj = w ? w[j] : 1.0;
                acc += wj * fr[(size_t)f * n + j];
                env += wj * wj;
            }
            ((float*)out)[s * outLen + i] = env > 0 ? (float)(acc / env) : 0.f;
        }
    }
}

bool hasCols(uint32_t ny) { return ny >= 32 && ny <= 4096 && !(ny & (ny - 1)); }
int launchCols(const void* in, void* out, uint32_t ny, uint32_t ncols, uint64_t pitch, uint64_t matStride,
               uint64_t mats, bool inverse, float scale, const void*, void*) {
    if (!hasCols(ny) || ncols == 0 || mats == 0) return 1;
    if (int r = launch()) return r;
    std::vector<float> col(2 * ny), res(2 * ny);   // gather a column, transform, scatter (in == out allowed)
    for (uint64_t m = 0; m < mats; ++m)
        for (uint32_t c = 0; c < ncols; ++c) {
            const float* src = (const float*)in + 2 * (m * matStride + c);
            float* dst = (float*)out + 2 * (m * matStride + c);
            for (uint32_t i = 0; i < ny; ++i) {
                col[2 * i] = src[2 * i * pitch];
                col[2 * i + 1] = src[2 * i * pitch + 1];
            }
            dft(col.data(), res.data(), ny, inverse ? 1 : -1, scale);
            for (uint32_t i = 0; i < ny; ++i) {
                dst[2 * i * pitch] = res[2 * i];
                dst[2 * i * pitch + 1] = res[2 * i + 1];
            }
        }
    return 0;
}

bool hasLongCluster(uint32_t n, int cta) {
    return (n == 8192 && cta == 256) || ((n == 16384 || n == 32768 || n == 65536) && (cta == 256 || cta == 512));
}
int launchLongCluster(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale,
                      const void*, const void*, const void*, const void*, int cta, void*) {
    if (!hasLongCluster(n, cta)) return 1;
    if (reinterpret_cast<uintptr_t>(in) % 16 != 0) return kLongClusterUnaligned;
    if (int r = launch()) return r;
    for (uint64_t b = 0; b < batch; ++b)
        dft((const float*)in + b * 2 * n, (float*)out + b * 2 * n, n, inverse ? 1 : -1, scale);
    return 0;
}

int longClusterStatus(unsigned* status, bool) { *status = 0; return 0; }

bool hasLongRing(uint32_t n) { return n == 8192 || n == 16384 || n == 32768 || n == 65536; }
int longRingSlots() { return 4; }
uint32_t longRingSlotRows(uint32_t n, uint64_t batch, size_t slotBytes) {
    uint64_t rows = slotBytes / ((uint64_t)n * 8);
    if (rows < 1) rows = 1;
    if (rows > batch) rows = batch;
    return (uint32_t)rows;
}
int launchLongRing(const void* in, void* out, void*, uint32_t, uint32_t n, uint64_t batch, bool inverse, float scale,
                   const void*, const void*, const void*, const void*, void*, void*) {
    if (int r = launch()) return r;
    for (uint64_t b = 0; b < batch; ++b)
        dft((const float*)in + b * 2 * n, (float*)out + b * 2 * n, n, inverse ? 1 : -1, scale);
    return 0;
}
int longRingStatus(unsigned* status, bool) { *status = 0; return 0; }

int raggedSmemBytes() { return 34816; }
int raggedGrid(int, int* grid) { *grid = 148 * 2; return 0; }
int launchRagged(const void* entries, int count, uint64_t, int, void*) {
    if (int r = launch()) return r;
    const RaggedEntry* es = static_cast<const RaggedEntry*>(entries);
    for (int i = 0; i < count; ++i) {
        if (es[i].e == 16) fake::timedExtra += fake::raggedCost16;
        const uint32_t n = 1u << es[i].logn;
        for (uint64_t b = 0; b < es[i].batch; ++b)
            dft((const float*)es[i].in + b * 2 * n, (float*)es[i].out + b * 2 * n, n, es[i].direction,
                es[i].scale);
    }
    return 0;
}

int raggedStagedGrid(int, int stages, int* grid) { *grid = 148 * (stages == 1 ? 3 : 2); return 0; }
int launchRaggedStaged(const void* entries, int count, uint64_t tiles, int grid, int, void* s) {
    return launchRagged(entries, count, tiles, grid, s);
}
int raggedStatus(unsigned* status, bool) { *status = 0; return 0; }
int launchRaggedFlat(const void* entries, int count, const void*, uint64_t tiles, void* s) {
    return launchRagged(entries, count, tiles, 0, s);
}

bool hasTensorVariant(uint32_t n, int split) {
    return n >= 64 && n <= 4096 && !(n & (n - 1)) && (split == 2 || split == 3);
}
size_t tensorTableBytes(int split) { return (size_t)split * 2048; }
int buildTensorTable(void*, int, void*) { return launch(); }
size_t tensorTwiddleCount(uint32_t n) { return n >= 256 ? (n >= 4096 ? 2 : 1) * n : 0; }
int buildTensorTwiddles(void*, uint32_t, void*) { return launch(); }
int launchC2CTensor(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale,
                    const void* tw, const void*, const void*, int, void* s) {
    return launchC2C(in, out, n, batch, inverse, scale, tw, 16, 256, s);
}
int tensorStatus(unsigned* status, bool) { *status = 0; return 0; }

}  // namespace backend
}  // namespace bfly
