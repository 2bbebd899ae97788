// CUDA implementation of the device seam (backend.h): runtime calls, CUDA-event timing,
// kernel-variant resolution and launches of the hand-written sm_100a kernels.
#include "backend.h"
#include "fft_kernels.cuh"
#include "launch.cuh"
#include "registry.cuh"

#include <atomic>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

namespace bfly {
namespace backend {

using dev::Entry;

static cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }
static int rc(cudaError_t e) { return e == cudaSuccess ? 0 : (int)e; }

int deviceCount(int* count) { return rc(cudaGetDeviceCount(count)); }
int setDevice(int device) {
    if (int e = rc(cudaSetDevice(device))) return e;
    return rc(cudaFree(nullptr));   // force context creation
}
int deviceName(int device, char* buf, size_t cap) {
    cudaDeviceProp p;
    if (int e = rc(cudaGetDeviceProperties(&p, device))) return e;
    std::strncpy(buf, p.name, cap ? cap - 1 : 0);
    if (cap) buf[cap - 1] = 0;
    return 0;
}
int smCount(int device, int* count) {
    return rc(cudaDeviceGetAttribute(count, cudaDevAttrMultiProcessorCount, device));
}
int streamCreate(void** stream) {
    cudaStream_t s = nullptr;
    int e = rc(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    *stream = s;
    return e;
}
int streamDestroy(void* stream) { return rc(cudaStreamDestroy(S(stream))); }
int alloc(void** ptr, size_t bytes) { return rc(cudaMalloc(ptr, bytes)); }
int release(void* ptr) { return rc(cudaFree(ptr)); }
int allocHost(void** ptr, size_t bytes) { return rc(cudaMallocHost(ptr, bytes)); }
int releaseHost(void* ptr) { return rc(cudaFreeHost(ptr)); }
int copyH2D(void* dst, const void* src, size_t bytes, void* stream) {
    return rc(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, S(stream)));
}
int copyD2H(void* dst, const void* src, size_t bytes, void* stream) {
    return rc(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, S(stream)));
}
int streamSync(void* stream) { return rc(cudaStreamSynchronize(S(stream))); }
int eventCreate(void** event) {
    cudaEvent_t e = nullptr;
    const int r = rc(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    *event = e;
    return r;
}
int eventDestroy(void* event) { return rc(cudaEventDestroy(static_cast<cudaEvent_t>(event))); }
int eventRecord(void* event, void* stream) { return rc(cudaEventRecord(static_cast<cudaEvent_t>(event), S(stream))); }
int eventSync(void* event) { return rc(cudaEventSynchronize(static_cast<cudaEvent_t>(event))); }
bool isPinnedHost(const void* ptr) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();   // an unknown pointer is ordinary pageable memory
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}
int streamWaitEvent(void* stream, void* event) {
    return rc(cudaStreamWaitEvent(S(stream), static_cast<cudaEvent_t>(event), 0));
}

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
};
int timerCreate(Timer** timer) {
    Timer* t = new Timer;
    if (int e = rc(cudaEventCreate(&t->a))) { delete t; return e; }
    if (int e = rc(cudaEventCreate(&t->b))) { cudaEventDestroy(t->a); delete t; return e; }
    *timer = t;
    return 0;
}
int timerStart(Timer* t, void* stream) { return rc(cudaEventRecord(t->a, S(stream))); }
int timerStop(Timer* t, void* stream, float* ms) {
    if (int e = rc(cudaEventRecord(t->b, S(stream)))) return e;
    if (int e = rc(cudaEventSynchronize(t->b))) return e;
    return rc(cudaEventElapsedTime(ms, t->a, t->b));
}
void timerDestroy(Timer* t) {
    if (!t) return;
    cudaEventDestroy(t->a);
    cudaEventDestroy(t->b);
    delete t;
}

// ------------------------------------------------------------------ variants
static const Entry* findEntry(int kind, uint32_t n, int e, int cta, int flag) {
    switch (kind) {
        case kC2C: return flag ? dev::findC2CInv(n, e, cta) : dev::findC2CFwd(n, e, cta);
        case kR2C: return dev::findR2C(n, e, cta, flag != 0);
        case kC2R: return dev::findC2R(n, e, cta);
        default: return nullptr;
    }
}

bool hasVariant(int kind, uint32_t n, int e, int cta) {
    return findEntry(kind, n, e, cta, 0) != nullptr;
}
size_t variantSmemBytes(int kind, uint32_t n, int e, int cta) {
    const Entry* x = findEntry(kind, n, e, cta, 0);
    return x ? (size_t)x->smem : 0;
}

// Raise the dynamic shared-memory limit once per kernel that needs more than 48 KB.
int optInSharedMemory(const void* fn, int bytes) {
    if (bytes <= 48 * 1024) return 0;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return (int)cudaErrorInvalidDevice;
    static std::mutex mu;
    static std::vector<std::pair<int, const void*>> done;
    std::lock_guard<std::mutex> lock(mu);
    for (const auto& d : done)
        if (d.first == device && d.second == fn) return 0;
    const int e = rc(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    if (!e) done.push_back({device, fn});
    return e;
}

static int prepareEntry(const Entry* x) { return optInSharedMemory(x->fn, x->smem); }

static unsigned gridFor(uint64_t batch, int rows) {
    return (unsigned)((batch + (uint64_t)rows - 1) / (uint64_t)rows);
}

size_t stockhamTwiddleCount(uint32_t n, int e) {
    dev::KTw fn;
    int count = 0;
    return dev::findTw(n, e, &fn, &count) ? (size_t)count : 0;
}

int buildStockhamTwiddles(void* tw, uint32_t n, int e, void* stream) {
    dev::KTw fn;
    int count = 0;
    if (!dev::findTw(n, e, &fn, &count)) return (int)cudaErrorInvalidValue;
    if (count == 0) return 0;
    fn<<<(count + 255) / 256, 256, 0, S(stream)>>>(static_cast<float2*>(tw));
    return rc(cudaGetLastError());
}

int buildLinearTwiddles(void* tw, int count, long long stride, long long n, void* stream) {
    if (count <= 0) return 0;
    dev::k_tw_linear<<<(count + 255) / 256, 256, 0, S(stream)>>>(static_cast<float2*>(tw), count,
                                                                   stride, n);
    return rc(cudaGetLastError());
}

int launchC2C(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale,
              const void* tw, int e, int cta, void* stream) {
    const Entry* x = findEntry(kC2C, n, e, cta, inverse ? 1 : 0);
    if (!x) return (int)cudaErrorInvalidDeviceFunction;
    if (int err = prepareEntry(x)) return err;
    return rc(launchPdl(x->fn, gridFor(batch, x->rows), x->cta, x->smem, S(stream), static_cast<const float2*>(in),
                        static_cast<float2*>(out), static_cast<const float2*>(tw), batch, scale));
}

int launchR2C(const void* in, void* out, uint32_t n, uint64_t batch, const void* tw,
              const void* twr, int e, int cta, bool weighted, float sEdge, float sInt,
              void* stream) {
    const Entry* x = findEntry(kR2C, n, e, cta, weighted ? 1 : 0);
    if (!x) return (int)cudaErrorInvalidDeviceFunction;
    if (int err = prepareEntry(x)) return err;
    return rc(launchPdl(x->fn, gridFor(batch, x->rows), x->cta, x->smem, S(stream), static_cast<const float2*>(in),
                        static_cast<float2*>(out), static_cast<const float2*>(tw), static_cast<const float2*>(twr),
                        batch, sEdge, sInt));
}

int launchC2R(const void* in, void* out, uint32_t n, uint64_t batch, const void* tw,
              const void* twr, int e, int cta, float sEdge, float sInt, float outScale,
              void* stream) {
    const Entry* x = findEntry(kC2R, n, e, cta, 0);
    if (!x) return (int)cudaErrorInvalidDeviceFunction;
    if (int err = prepareEntry(x)) return err;
    return rc(launchPdl(x->fn, gridFor(batch, x->rows), x->cta, x->smem, S(stream), static_cast<const float2*>(in),
                        static_cast<float2*>(out), static_cast<const float2*>(tw), static_cast<const float2*>(twr),
                        batch, sEdge, sInt, outScale));
}

// ------------------------------------------------------------------ four-step
bool hasLongSplit(uint32_t n1, uint32_t n2) {
    return dev::findLongA(n1, false) && dev::findLongB(n2, false);
}
void longSplit(uint32_t n, uint32_t* n1, uint32_t* n2) {
    *n1 = *n2 = 0;
    if (n < 8192 || n > 65536 || (n & (n - 1))) return;
    *n2 = 256;
    *n1 = n / 256;
}
int longE() { return 16; }

static int ilog2u(uint32_t v) {
    int l = 0;
    while ((1u << l) < v) ++l;
    return l;
}

int launchLongA(const void* in, void* out, uint32_t n1, uint32_t n2, uint64_t batch,
                bool inverse, const void* tw1, const void* tlo, const void* thi, void* stream) {
    const Entry* x = dev::findLongA(n1, inverse);
    if (!x || n2 % (uint32_t)x->rows) return (int)cudaErrorInvalidDeviceFunction;
    const uint64_t perRow = n2 / (uint32_t)x->rows;
    if (batch == 0 || batch > 0x7fffffffull / perRow) return (int)cudaErrorInvalidValue;
    if (int err = prepareEntry(x)) return err;
    auto fn = reinterpret_cast<dev::KLongA>(const_cast<void*>(x->fn));
    const uint64_t grid = batch * perRow;
    fn<<<(unsigned)grid, x->cta, x->smem, S(stream)>>>(
        static_cast<const float2*>(in), static_cast<float2*>(out), static_cast<const float2*>(tw1),
        static_cast<const float2*>(tlo), static_cast<const float2*>(thi), batch, ilog2u(n2));
    return rc(cudaGetLastError());
}

int prepareLongKernels() {
    for (uint32_t n1 = 32; n1 <= 256; n1 *= 2)
        for (int inv = 0; inv < 2; ++inv) {
            const Entry* xs[2] = {dev::findLongA(n1, inv != 0), n1 == 256 ? dev::findLongB(256, inv != 0) : nullptr};
            for (const Entry* x : xs) {
                if (!x) continue;
                cudaFuncAttributes attr;
                if (int err = rc(cudaFuncGetAttributes(&attr, x->fn))) return err;   // loads the kernel
                if (int err = prepareEntry(x)) return err;
            }
        }
    return 0;
}

bool hasCols(uint32_t ny) { return dev::findCols(ny, false) != nullptr; }

int launchCols(const void* in, void* out, uint32_t ny, uint32_t ncols, uint64_t pitch, uint64_t matStride,
               uint64_t mats, bool inverse, float scale, const void* tw, void* stream) {
    const Entry* x = dev::findCols(ny, inverse);
    if (!x || ncols == 0 || mats == 0) return (int)cudaErrorInvalidValue;
    const uint32_t colBlocks = (ncols + (uint32_t)x->rows - 1) / (uint32_t)x->rows;
    const uint64_t grid = mats * colBlocks;
    if (grid > 0x7fffffffull) return (int)cudaErrorInvalidValue;
    if (int err = prepareEntry(x)) return err;
    auto fn = reinterpret_cast<dev::KCols>(const_cast<void*>(x->fn));
    fn<<<(unsigned)grid, x->cta, x->smem, S(stream)>>>(static_cast<const float2*>(in), static_cast<float2*>(out),
                                                      static_cast<const float2*>(tw), ncols, pitch, matStride,
                                                      colBlocks, scale);
    return rc(cudaGetLastError());
}

int launchLongB(const void* in, void* out, uint32_t n1, uint32_t n2, uint64_t batch,
                bool inverse, float scale, const void* tw2, void* stream) {
    const Entry* x = dev::findLongB(n2, inverse);
    if (!x || n1 % (uint32_t)x->rows) return (int)cudaErrorInvalidDeviceFunction;
    const uint64_t perRow = n1 / (uint32_t)x->rows;
    if (batch == 0 || batch > 0x7fffffffull / perRow) return (int)cudaErrorInvalidValue;
    if (int err = prepareEntry(x)) return err;
    auto fn = reinterpret_cast<dev::KLongB>(const_cast<void*>(x->fn));
    const uint64_t grid = batch * perRow;
    fn<<<(unsigned)grid, x->cta, x->smem, S(stream)>>>(
        static_cast<const float2*>(in), static_cast<float2*>(out), static_cast<const float2*>(tw2),
        batch, ilog2u(n1), scale);
    return rc(cudaGetLastError());
}

}  // namespace backend
}  // namespace bfly
