// Ragged persistent launch: a work list of C2C requests with different lengths (32..4096),
// batch counts and directions, processed by one grid of persistent CTAs.  Every tile is
// 256 threads x E values (rows of one request; E = 8 or 16, chosen per request in the work
// list), so tiles cost about the same and a static stride over the tile space balances the
// grid; no atomics and no waits.
// Inverse requests run the forward kernel on conj(x) and conjugate the result
// (IDFT(x) = conj(DFT(conj x))), so one code path per length serves both directions.
#include "backend.h"
#include "fft_kernels.cuh"
#include "launch.cuh"
#include "ragged.h"
#include "tma.cuh"

namespace bfly {
namespace dev {

// Nonzero after a staged launch gave up on a bounded wait (read and cleared by the host).
__device__ unsigned int g_ragged_status;

// Every (length, radix) variant of the work list, as case labels of a switch on
// logn * 32 + e; CALL(N, E) is the body for one variant.
#define BFLY_RAGGED_CASES(CALL)                                                              \
    case 5 * 32 + 8: CALL(32, 8); break;      case 5 * 32 + 16: CALL(32, 16); break;         \
    case 6 * 32 + 8: CALL(64, 8); break;      case 6 * 32 + 16: CALL(64, 16); break;         \
    case 7 * 32 + 8: CALL(128, 8); break;     case 7 * 32 + 16: CALL(128, 16); break;        \
    case 8 * 32 + 8: CALL(256, 8); break;     case 8 * 32 + 16: CALL(256, 16); break;        \
    case 9 * 32 + 8: CALL(512, 8); break;     case 9 * 32 + 16: CALL(512, 16); break;        \
    case 10 * 32 + 8: CALL(1024, 8); break;   case 10 * 32 + 16: CALL(1024, 16); break;      \
    case 11 * 32 + 8: CALL(2048, 8); break;   case 11 * 32 + 16: CALL(2048, 16); break;      \
    case 12 * 32 + 16: CALL(4096, 16); break;                                                \
    default: break;

template <int N, int E>
__device__ __forceinline__ void ragged_tile(const RaggedEntry& r, uint64_t tileInReq, float2* smem) {
    static_assert(raggedVariant(ilog2c(N), E), "no such ragged variant");
    constexpr int T = N / E;
    constexpr int ROWS = kRaggedThreads / T;
    constexpr int S = smem_stride<N, E, false>();
    using TM = Team<N, E, false, sync_kind(T, kRaggedThreads)>;
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const uint64_t row = tileInReq * ROWS + rl;
    const bool ok = row < r.batch;
    const float2* src = static_cast<const float2*>(r.in) + row * N;
    float2* dst = static_cast<float2*>(r.out) + row * N;
    const float sgn = r.direction > 0 ? -1.f : 1.f;   // conjugation for the inverse
    const float sc = r.scale;
    float2 v[E];
    TM::run(v, smem + rl * S, static_cast<const float2*>(r.tw), t, rl, [&](int i) {
        if (!ok) return make_float2(0.f, 0.f);
        const float2 x = ld_stream(src + i);
        return make_float2(x.x, sgn * x.y);
    });
    pdl_trigger();
    if (ok)
        TM::for_each_out(v, t, [&](int i, float2 x) { st_stream(dst + i, make_float2(x.x * sc, sgn * sc * x.y)); });
}

__device__ __forceinline__ int find_request_plain(const RaggedEntry* __restrict__ reqs, int nreq, uint64_t tile) {
    int lo = 0, hi = nreq - 1;   // last request whose first tile is <= tile
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (reqs[mid].tile0 <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(kRaggedThreads, 4)
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
#define BFLY_TILE(NN, EE) ragged_tile<NN, EE>(r, local, smem)
        switch (r.logn * 32 + r.e) { BFLY_RAGGED_CASES(BFLY_TILE) }
#undef BFLY_TILE
        __syncthreads();   // the next tile reuses the exchange buffers
    }
}

// One tile per CTA over the same work list: the hardware CTA scheduler balances the tiles
// (no persistent loop); grid = number of tiles.
// `tileMap` (request index of every tile, built with the work list) replaces the binary search
// when present; every thread reads it directly, so no barrier precedes the first data load.
__global__ void __launch_bounds__(kRaggedThreads, 4)
k_ragged_flat(const RaggedEntry* __restrict__ reqs, int nreq, const uint32_t* __restrict__ tileMap,
              uint64_t tileBase) {
    extern __shared__ float2 smem[];
    pdl_wait();
    const uint64_t tile = tileBase + blockIdx.x;
    const int q = tileMap ? (int)__ldg(tileMap + tile) : find_request_plain(reqs, nreq, tile);
    const RaggedEntry r = reqs[q];
    const uint64_t local = tile - r.tile0;
#define BFLY_TILE(NN, EE) ragged_tile<NN, EE>(r, local, smem)
    switch (r.logn * 32 + r.e) { BFLY_RAGGED_CASES(BFLY_TILE) }
#undef BFLY_TILE
}

// ------------------------------------------------------------------ TMA-staged variant
// Same work list and tiles; a tile's input rows are contiguous in global memory, so one bulk
// copy (cp.async.bulk, completing on an mbarrier) stages them in shared memory.  Thread 0
// issues the copy of the CTA's tile i + STAGES as soon as every thread has moved tile i from
// its stage into registers, so HBM reads of later tiles overlap the passes of the current one.
// Inputs must be 16-byte aligned (checked on the host).
constexpr int kStageBytes = kRaggedThreads * 16 * 8;   // largest tile: 4096 complex values

__device__ __forceinline__ int find_request(const RaggedEntry* __restrict__ reqs, int nreq, uint64_t tile) {
    int lo = 0, hi = nreq - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (reqs[mid].tile0 <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Thread 0: stage tile `tile` into `stage` (request index recorded in *slot).
__device__ __forceinline__ void issue_tile(const RaggedEntry* __restrict__ reqs, int nreq, uint64_t tile,
                                           float2* stage, uint64_t* bar, int* slot) {
    const int q = find_request(reqs, nreq, tile);
    *slot = q;
    const RaggedEntry& r = reqs[q];
    const uint64_t local = tile - r.tile0;
    const uint64_t first = local * r.rowsPerTile;
    const uint64_t rows = (r.batch - first) < r.rowsPerTile ? (r.batch - first) : r.rowsPerTile;
    const uint32_t n = 1u << r.logn;
    const uint32_t bytes = (uint32_t)(rows * n * 8u);
    mbar_arrive_expect_tx(bar, bytes);
    bulk_load(stage, static_cast<const float2*>(r.in) + first * n, bytes, bar);
}

template <int N, int E>
__device__ __forceinline__ void ragged_tile_staged(const RaggedEntry& r, uint64_t tileInReq, const float2* stage,
                                                   float2* xbuf, const RaggedEntry* __restrict__ reqs, int nreq,
                                                   uint64_t next, uint64_t totalTiles, float2* nextStage,
                                                   uint64_t* bar, int* slot) {
    constexpr int T = N / E;
    constexpr int ROWS = kRaggedThreads / T;
    constexpr int S = smem_stride<N, E, false>();
    using TM = Team<N, E, false, sync_kind(T, kRaggedThreads)>;
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const uint64_t row = tileInReq * ROWS + rl;
    const bool ok = row < r.batch;
    const float2* src = stage + rl * N;
    float2* dst = static_cast<float2*>(r.out) + row * N;
    const float sgn = r.direction > 0 ? -1.f : 1.f;
    const float sc = r.scale;
    float2 v[E];
    TM::load_first(v, t, [&](int i) {
        const float2 x = src[i];
        return make_float2(x.x, sgn * x.y);
    });
    __syncthreads();   // every thread has consumed this stage
    if (threadIdx.x == 0 && next < totalTiles) {
        fence_proxy_async_smem();
        issue_tile(reqs, nreq, next, nextStage, bar, slot);
    }
    TM::template passes<0>(v, xbuf + rl * S, static_cast<const float2*>(r.tw), t, rl);
    pdl_trigger();
    if (ok)
        TM::for_each_out(v, t, [&](int i, float2 x) { st_stream(dst + i, make_float2(x.x * sc, sgn * sc * x.y)); });
}

template <int STAGES>
__global__ void __launch_bounds__(kRaggedThreads, STAGES == 1 ? 3 : 2)
k_ragged_tma(const RaggedEntry* __restrict__ reqs, int nreq, uint64_t totalTiles, int xbufBytes) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float2* xbuf = reinterpret_cast<float2*>(smem_raw + STAGES * kStageBytes);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + STAGES * kStageBytes + xbufBytes);
    int* slot = reinterpret_cast<int*>(bar + STAGES);
    auto stage = [&](int s) { return reinterpret_cast<float2*>(smem_raw + s * kStageBytes); };
    const uint64_t grid = gridDim.x;
    uint32_t issued[STAGES], consumed[STAGES];
    for (int s = 0; s < STAGES; ++s) issued[s] = consumed[s] = 0;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&bar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int s = 0; s < STAGES; ++s) {
            const uint64_t tile = blockIdx.x + (uint64_t)s * grid;
            if (tile < totalTiles) {
                issue_tile(reqs, nreq, tile, stage(s), &bar[s], &slot[s]);
                ++issued[s];
            }
        }
    __syncthreads();
    uint32_t k = 0;
    for (uint64_t tile = blockIdx.x; tile < totalTiles; tile += grid, ++k) {
        const int s = (int)(k % STAGES);
        const bool ready = mbar_wait_bounded(&bar[s], consumed[s] & 1u);
        if (__syncthreads_or(!ready)) {
            // a copy never completed: record it, give copies in flight a bounded chance, leave
            if (threadIdx.x == 0) {
                atomicOr(&g_ragged_status, 1u);
                for (int q = 0; q < STAGES; ++q)
                    if (issued[q] > consumed[q]) mbar_wait_bounded(&bar[q], consumed[q] & 1u);
            }
            return;
        }
        ++consumed[s];
        const RaggedEntry r = reqs[slot[s]];
        const uint64_t local = tile - r.tile0;
        const uint64_t next = tile + (uint64_t)STAGES * grid;
        if (threadIdx.x == 0 && next < totalTiles) ++issued[s];
#define BFLY_STAGED(NN, EE) \
    ragged_tile_staged<NN, EE>(r, local, stage(s), xbuf, reqs, nreq, next, totalTiles, stage(s), &bar[s], &slot[s])
        switch (r.logn * 32 + r.e) { BFLY_RAGGED_CASES(BFLY_STAGED) }
#undef BFLY_STAGED
        __syncthreads();   // the next tile reuses the exchange buffers
    }
}

}  // namespace dev

namespace backend {

template <int N, int E>
static constexpr int raggedSmem() {
    return (kRaggedThreads / (N / E)) * dev::smem_stride<N, E, false>() * 8;
}

static constexpr int maxi(int a, int b) { return a > b ? a : b; }

template <int N>
static constexpr int raggedSmemBoth() {
    return maxi(raggedSmem<N, 8>(), raggedSmem<N, 16>());
}

// Exchange buffer of the largest variant (every kernel serves every variant).
int raggedSmemBytes() {
    return maxi(maxi(maxi(raggedSmemBoth<32>(), raggedSmemBoth<64>()), maxi(raggedSmemBoth<128>(), raggedSmemBoth<256>())),
                maxi(maxi(raggedSmemBoth<512>(), raggedSmemBoth<1024>()),
                     maxi(raggedSmemBoth<2048>(), raggedSmem<4096, 16>())));
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

static int stagedSmem(int stages) {
    const int xbuf = (raggedSmemBytes() + 127) & ~127;
    return stages * dev::kStageBytes + xbuf + stages * 8 + stages * 4;
}

int raggedStagedGrid(int device, int stages, int* grid) {
    const int smem = stagedSmem(stages);
    const void* fn = stages == 1 ? (const void*)dev::k_ragged_tma<1> : (const void*)dev::k_ragged_tma<2>;
    int perSm = 0, sms = 0;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fn, kRaggedThreads, smem);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return (int)e;
    *grid = sms * (perSm > 0 ? perSm : 1);
    return 0;
}

int launchRaggedStaged(const void* entries, int count, uint64_t totalTiles, int grid, int stages, void* stream) {
    if (count <= 0 || totalTiles == 0) return 0;
    const unsigned g = (unsigned)((uint64_t)grid < totalTiles ? (uint64_t)grid : totalTiles);
    const int xbuf = (raggedSmemBytes() + 127) & ~127;
    const auto* es = static_cast<const RaggedEntry*>(entries);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (stages == 1)
        dev::k_ragged_tma<1><<<g, kRaggedThreads, stagedSmem(1), st>>>(es, count, totalTiles, xbuf);
    else
        dev::k_ragged_tma<2><<<g, kRaggedThreads, stagedSmem(2), st>>>(es, count, totalTiles, xbuf);
    return (int)cudaGetLastError();
}

int launchRaggedFlat(const void* entries, int count, const void* tileMap, uint64_t totalTiles, void* stream) {
    if (count <= 0 || totalTiles == 0) return 0;
    if (int e = optInSharedMemory((const void*)dev::k_ragged_flat, raggedSmemBytes())) return e;
    const auto* es = static_cast<const RaggedEntry*>(entries);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    for (uint64_t base = 0; base < totalTiles; base += 0x7fffffffull) {
        const uint64_t cnt = totalTiles - base < 0x7fffffffull ? totalTiles - base : 0x7fffffffull;
        const uint32_t* map = static_cast<const uint32_t*>(tileMap);
        if (cudaError_t e = launchPdl((const void*)dev::k_ragged_flat, (unsigned)cnt, kRaggedThreads,
                                      raggedSmemBytes(), st, es, count, map, base))
            return (int)e;
    }
    return (int)cudaGetLastError();
}

int raggedStatus(unsigned* status, bool clear) {
    if (cudaMemcpyFromSymbol(status, dev::g_ragged_status, sizeof(unsigned)) != cudaSuccess) return 1;
    if (clear && *status) {
        const unsigned zero = 0;
        if (cudaMemcpyToSymbol(dev::g_ragged_status, &zero, sizeof(unsigned)) != cudaSuccess) return 1;
    }
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
