// Ragged persistent launch: a work list of C2C requests with different lengths (32..4096),
// batch counts and directions, processed by one grid of persistent CTAs.  Every tile is
// 256 threads x 16 values = 4096 complex points (rows of one request), so tiles cost the same
// and a static stride over the tile space balances the grid; no atomics and no waits.
// Inverse requests run the forward kernel on conj(x) and conjugate the result
// (IDFT(x) = conj(DFT(conj x))), so one code path per length serves both directions.
#include "fft_kernels.cuh"
#include "ragged.h"

namespace bfly {
namespace dev {

template <int N>
__device__ __forceinline__ void ragged_tile(const RaggedEntry& r, uint64_t tileInReq, float2* smem) {
    constexpr int E = kRaggedE;
    constexpr int T = N / E;
    constexpr int ROWS = kRaggedThreads / T;
    constexpr int S = smem_stride<N, E, false>();
    using TM = Team<N, E, false, (T > 32)>;
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const uint64_t row = tileInReq * ROWS + rl;
    const bool ok = row < r.batch;
    const float2* src = static_cast<const float2*>(r.in) + row * N;
    float2* dst = static_cast<float2*>(r.out) + row * N;
    const float sgn = r.direction > 0 ? -1.f : 1.f;   // conjugation for the inverse
    const float sc = r.scale;
    float2 v[E];
    TM::run(v, smem + rl * S, static_cast<const float2*>(r.tw), t, [&](int i) {
        if (!ok) return make_float2(0.f, 0.f);
        const float2 x = ld_stream(src + i);
        return make_float2(x.x, sgn * x.y);
    });
    if (ok)
        TM::for_each_out(v, t, [&](int i, float2 x) { st_stream(dst + i, make_float2(x.x * sc, sgn * sc * x.y)); });
}

__global__ void __launch_bounds__(kRaggedThreads)
k_ragged(const RaggedEntry* __restrict__ reqs, int nreq, uint64_t totalTiles) {
    extern __shared__ float2 smem[];
    for (uint64_t tile = blockIdx.x; tile < totalTiles; tile += gridDim.x) {
        int lo = 0, hi = nreq - 1;   // last request whose first tile is <= tile
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (reqs[mid].tile0 <= tile) lo = mid;
            else hi = mid - 1;
        }
        const RaggedEntry r = reqs[lo];
        const uint64_t local = tile - r.tile0;
        switch (r.logn) {
            case 5: ragged_tile<32>(r, local, smem); break;
            case 6: ragged_tile<64>(r, local, smem); break;
            case 7: ragged_tile<128>(r, local, smem); break;
            case 8: ragged_tile<256>(r, local, smem); break;
            case 9: ragged_tile<512>(r, local, smem); break;
            case 10: ragged_tile<1024>(r, local, smem); break;
            case 11: ragged_tile<2048>(r, local, smem); break;
            case 12: ragged_tile<4096>(r, local, smem); break;
            default: break;
        }
        __syncthreads();   // the next tile reuses the exchange buffers
    }
}

}  // namespace dev

namespace backend {

template <int N>
static constexpr int raggedSmem() {
    return (kRaggedThreads / (N / kRaggedE)) * dev::smem_stride<N, kRaggedE, false>() * 8;
}

static constexpr int maxi(int a, int b) { return a > b ? a : b; }

int raggedSmemBytes() {
    return maxi(maxi(maxi(raggedSmem<32>(), raggedSmem<64>()), maxi(raggedSmem<128>(), raggedSmem<256>())),
                maxi(maxi(raggedSmem<512>(), raggedSmem<1024>()), maxi(raggedSmem<2048>(), raggedSmem<4096>())));
}

int raggedGrid(int device, int* grid) {
    const int smem = raggedSmemBytes();
    int perSm = 0, sms = 0;
    cudaError_t e = cudaFuncSetAttribute(dev::k_ragged, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, dev::k_ragged, kRaggedThreads, smem);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return (int)e;
    *grid = sms * (perSm > 0 ? perSm : 1);
    return 0;
}

int launchRagged(const void* entries, int count, uint64_t totalTiles, int grid, void* stream) {
    if (count <= 0 || totalTiles == 0) return 0;
    const unsigned g = (unsigned)((uint64_t)grid < totalTiles ? (uint64_t)grid : totalTiles);
    dev::k_ragged<<<g, kRaggedThreads, raggedSmemBytes(), reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const RaggedEntry*>(entries), count, totalTiles);
    return (int)cudaGetLastError();
}

}  // namespace backend
}  // namespace bfly
