// Long C2C (four-step, n = 8192..65536) that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the moment they need a transform: code that runs
// while a CUDA graph is being captured (an allocation would break the capture), real-time
// loops that must not allocate after start-up so their latency stays bounded, and programs
// whose GPU memory is owned by another allocator or budget, where a stray cudaMalloc could
// fail or push past the budget.  The regular entry points grow a plan-owned workspace and
// twiddle tables with cudaMalloc on first use; this one instead keeps its workspace and
// tables in fixed arrays that live in this library's device image.
//
// Limits and behaviour:
//  * the workspace holds at most kScratchElems = 4,194,304 complex values (32 MiB), so
//    n * batch must not exceed it (for example 65536 x 64 or 8192 x 512); larger requests
//    are rejected with status -12 before any GPU work;
//  * every GPU that loads this library keeps the 32 MiB array (plus 18 KB of tables)
//    until the process exits;
//  * the first call on a device looks up the arrays' device addresses, loads every kernel
//    variant it can launch, builds the twiddle tables on the caller's stream and waits for
//    that stream once; make that first call before any stream capture (a first call on a
//    stream that is being captured returns -13 and leaves the capture untouched);
//  * all calls share one workspace: calls whose executions overlap on the GPU (different
//    streams, or different host threads) race and corrupt each other's results.  Nothing in
//    the workspace needs to start at zero: the column pass writes every value the row pass
//    reads.
#include "backend.h"
#include "fft_kernels.cuh"

#include <cuda_runtime.h>

#include <mutex>

namespace bfly {
namespace noalloc {

constexpr unsigned long long kScratchElems = 4194304ull;   // 32 MiB of complex64

// Twiddle tables for every supported length, laid out back to back:
//   Stockham tables of the column lengths n1 = 32, 64, 128, 256 and of the row length 256,
//   then for each n in 8192..65536 the two-level W_n tables lo (256) and hi (n/256).
constexpr int kTw1[4] = {0, 16, 64, 176};                // Sched<n1,16>::TWSIZE prefix sums
constexpr int kTw2 = 416;                                 // Sched<256,16> (240 entries)
constexpr int kLo[4] = {656, 912, 1168, 1424};
constexpr int kHi[4] = {1680, 1712, 1776, 1904};
constexpr int kTableElems = 2160;
static_assert(dev::Sched<32, 16>::TWSIZE == 16 && dev::Sched<64, 16>::TWSIZE == 48 &&
              dev::Sched<128, 16>::TWSIZE == 112 && dev::Sched<256, 16>::TWSIZE == 240,
              "table layout out of date");

static __device__ __align__(256) float2 g_scratch[kScratchElems];
static __device__ __align__(256) float2 g_tables[kTableElems];

struct DeviceState {
    bool ready = false;
    float2* scratch = nullptr;
    float2* tables = nullptr;
};
static std::mutex g_mutex;
static DeviceState g_state[64];

// Set-up on the current device: symbol addresses (host code must not use the array names as
// addresses), every four-step kernel variant this entry point can launch loaded and opted into
// its shared memory (so no later call loads device code or changes a kernel attribute), and the
// FP64-built twiddle tables, built on `stream` and waited for once.  A stream that is being
// captured is refused before anything touches it (-13): the table builds and the wait would
// land in, and break, the caller's capture.
static int setup(cudaStream_t stream, DeviceState* st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess) {
        cudaGetLastError();
        return -13;
    }
    if (cs != cudaStreamCaptureStatusNone) return -13;
    void* scratch = nullptr;
    void* tables = nullptr;
    if (cudaGetSymbolAddress(&scratch, g_scratch) != cudaSuccess) return -1;
    if (cudaGetSymbolAddress(&tables, g_tables) != cudaSuccess) return -1;
    if (bfly::backend::prepareLongKernels()) return -1;
    float2* t = static_cast<float2*>(tables);
    dev::k_tw_stockham<32, 16><<<1, 256, 0, stream>>>(t + kTw1[0]);
    dev::k_tw_stockham<64, 16><<<1, 256, 0, stream>>>(t + kTw1[1]);
    dev::k_tw_stockham<128, 16><<<1, 256, 0, stream>>>(t + kTw1[2]);
    dev::k_tw_stockham<256, 16><<<1, 256, 0, stream>>>(t + kTw1[3]);
    dev::k_tw_stockham<256, 16><<<1, 256, 0, stream>>>(t + kTw2);
    for (int i = 0; i < 4; ++i) {
        const long long n = 8192ll << i;
        dev::k_tw_linear<<<1, 256, 0, stream>>>(t + kLo[i], 256, 1, n);
        dev::k_tw_linear<<<1, 256, 0, stream>>>(t + kHi[i], (int)(n / 256), 256, n);
    }
    if (cudaGetLastError() != cudaSuccess) return -1;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return -1;
    st->scratch = static_cast<float2*>(scratch);
    st->tables = t;
    st->ready = true;
    return 0;
}

}  // namespace noalloc
}  // namespace bfly

extern "C" int bfly_exec_c2c_long_noalloc(const void* d_in, void* d_out, uint32_t n, uint64_t batch,
                                          int direction, float scale, void* stream) {
    using namespace bfly::noalloc;
    if (!d_in || !d_out) return -10;
    if (n < 8192 || n > 65536 || (n & (n - 1)) || batch == 0 || (direction != -1 && direction != 1))
        return -8;
    if (batch > kScratchElems / n) return -12;   // n >= 8192 here; the product could wrap
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) return -1;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DeviceState st;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (!g_state[device].ready) {
            if (int r = setup(s, &g_state[device])) return r;
        }
        st = g_state[device];
    }
    int li = 0;
    while ((8192u << li) < n) ++li;
    const uint32_t n1 = n / 256, n2 = 256;
    const float2* tw1 = st.tables + kTw1[li];
    const bool inv = direction > 0;
    if (bfly::backend::launchLongA(d_in, st.scratch, n1, n2, batch, inv, tw1, st.tables + kLo[li],
                                   st.tables + kHi[li], stream))
        return -5;
    if (bfly::backend::launchLongB(st.scratch, d_out, n1, n2, batch, inv, scale, st.tables + kTw2, stream))
        return -5;
    return 0;
}
