// Long C2C (n = N1 * 256 = 8192 .. 65536) as ONE persistent launch of the four-step schedule
// whose intermediate stays in L2.
//
// The two passes of the four-step (k_long_a: N1-point column FFTs times W_n^(n2*k1); k_long_b:
// 256-point row FFTs and the transposed store) run as work items of one grid.  Rows are taken
// in chunks of `slotRows`; a chunk's intermediate goes to one of kRingSlots slots of a ring
// (a few MB per slot), small enough to stay in the 126 MB L2 between the two passes, so each
// element crosses HBM once in each direction (16 bytes) instead of twice.
//
// Items (each 256 threads on 4096 values, N1/16 per row and pass) are ordered in stages
//   A(0) | A(1) | A(2) B(0) | A(3) B(1) | ... | A(k-1) B(k-3) | B(k-2) | B(k-1)
// (stage s: pass A of chunk s, then pass B of chunk s - kRingLag) and CTA g runs positions g,
// g + grid, g + 2 grid, ...  A pass-B item of chunk c waits until every pass-A item of chunk c
// has finished (counter aDone[c mod kRingSlots]); a pass-A item of chunk c waits until every
// pass-B item of chunk c - kRingSlots, the previous user of its slot, has finished
// (bDone[c mod kRingSlots]).  The lag keeps a chunk's pass A a stage or more ahead of its pass
// B, so those waits seldom hold anyone up.  Every item an item waits for sits at an earlier
// position, and the grid is launched cooperatively (all CTAs resident), so the lowest
// unfinished position can always run: the schedule cannot deadlock.  The waits are bounded all the same: one that runs out sets
// g_ring_status and every CTA stops waiting and leaves.
//
// Ordering: a finishing item's threads write the slot, bar.sync, then one thread adds to the
// counter with a gpu-scope release reduction; a waiting item's thread acquires the counter and
// bar.syncs before any thread reads.  Slot data are written and read at L2 (st/ld .cg), never
// through L1, which could hold a line of the slot's previous chunk.
#include <cuda_runtime.h>

#include <atomic>

#include "backend.h"
#include "fft_kernels.cuh"
#include "tma.cuh"

namespace bfly {
namespace dev {

__device__ unsigned int g_ring_status;   // nonzero: a bounded wait of k_long_ring ran out

constexpr int kRingThreads = 256;
constexpr int kRingSlots = 4;   // slots of the ring
constexpr int kRingLag = 2;     // stages between a chunk's pass A and its pass B (< kRingSlots)

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Thread 0 waits until *ctr >= target (bounded in time); the result is shared with the CTA.
__device__ __forceinline__ bool ring_wait(const unsigned* ctr, unsigned target) {
    __shared__ int okShared;
    if (threadIdx.x == 0) {
        bool ok = true;
        if (ld_acquire_gpu(ctr) < target) {
            const uint64_t t0 = global_timer_ns();
            for (uint32_t i = 0;; ++i) {
                if (ld_acquire_gpu(ctr) >= target) break;
                if (*(volatile unsigned*)&g_ring_status || global_timer_ns() - t0 > kWaitNs || i >= kWaitIters) {
                    ok = false;
                    break;
                }
                __nanosleep(64);
            }
        }
        if (!ok) atomicOr(&g_ring_status, 1u);
        okShared = ok;
    }
    __syncthreads();
    return okShared != 0;
}

// The CTA's slot writes (or reads) of this item are done: bar.sync makes them visible to thread
// 0, whose gpu-scope release increment (cumulative) publishes them with the count.
__device__ __forceinline__ void ring_signal(unsigned* ctr) {
    __syncthreads();
    if (threadIdx.x == 0) asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(ctr) : "memory");
}

template <int N1, bool INV>
struct Ring {
    static constexpr int N2 = 256, E = 16, N = N1 * N2;
    static constexpr int IPR = N1 / E;                // items per row, each pass
    static constexpr int TA = N1 / E, CA = kRingThreads / TA;   // pass A: threads per column, columns
    static constexpr int SA = smem_stride<N1, E, true>();
    static constexpr int TB = N2 / E, RB = kRingThreads / TB;   // pass B: threads per row, rows (16)
    static constexpr int SB = smem_stride<N2, E, false>();
    static constexpr int SMEM_A = CA * SA * 8, SMEM_B = RB * SB * 8;
    static constexpr int SMEM = SMEM_A > SMEM_B ? SMEM_A : SMEM_B;
    static_assert(CA * TA == kRingThreads && RB * TB == kRingThreads, "item shape");
    static_assert(IPR == N2 / CA && IPR == N1 / RB, "both passes cut a row into N1/16 items");

    // pass A: columns [colBlock*CA, +CA) of row `src` -> slot row `dst`
    static __device__ __forceinline__ void itemA(const float2* __restrict__ src, float2* __restrict__ dst,
                                                 int colBlock, float2* smem, const float2* __restrict__ tw1,
                                                 const float2* __restrict__ tlo, const float2* __restrict__ thi) {
        using TM = Team<N1, E, INV, kSyncBlock>;
        const int c = threadIdx.x % CA;
        const int t = threadIdx.x / CA;
        const uint32_t n2 = (uint32_t)colBlock * CA + c;
        float2 v[E];
        TM::run(v, smem + c * SA, tw1, t, 0, [&](int i) { return ld_stream(src + n2 + ((size_t)i << 8)); });
        TM::for_each_out(v, t, [&](int k1, float2 x) {
            const uint32_t m = n2 * (uint32_t)k1;
            const float2 w = cmul<false>(__ldg(thi + (m >> 8)), __ldg(tlo + (m & 255u)));
            __stcg(dst + n2 + ((size_t)k1 << 8), cmul<INV>(x, w));
        });
    }

    // pass B: rows k1 in [rowBlock*RB, +RB) of slot row `src` -> X[k1 + N1*k2] of `dst`
    static __device__ __forceinline__ void itemB(const float2* __restrict__ src, float2* __restrict__ dst,
                                                 int rowBlock, float2* smem, const float2* __restrict__ tw2,
                                                 float scale) {
        using TM = Team<N2, E, INV, sync_kind(TB, kRingThreads)>;
        const int rl = threadIdx.x / TB;
        const int t = threadIdx.x - rl * TB;
        const int k1_0 = rowBlock * RB;
        const float2* s = src + (size_t)(k1_0 + rl) * N2;
        float2* sm = smem + rl * SB;
        float2 v[E];
        TM::run(v, sm, tw2, t, rl, [&](int i) { return __ldcg(s + i); });
        __syncthreads();
        TM::for_each_out(v, t, [&](int i, float2 x) { sm[spad(i)] = x; });
        __syncthreads();
        float2* d = dst + k1_0;
        for (int idx = threadIdx.x; idx < RB * N2; idx += kRingThreads) {
            const int c = idx % RB;
            const int k2 = idx / RB;
            st_stream(d + c + (size_t)k2 * N1, cscale(smem[c * SB + spad(k2)], scale));
        }
    }
};

template <int N1, bool INV>
__global__ void __launch_bounds__(kRingThreads, 3)
k_long_ring(const float2* __restrict__ in, float2* __restrict__ out, float2* __restrict__ ring,
            const float2* __restrict__ tw1, const float2* __restrict__ tw2, const float2* __restrict__ tlo,
            const float2* __restrict__ thi, unsigned* __restrict__ ctr, uint64_t batch, uint32_t slotRows,
            float scale) {
    using R = Ring<N1, INV>;
    extern __shared__ float2 smem_ring[];
    unsigned* aDone = ctr;
    unsigned* bDone = ctr + kRingSlots;
    const uint64_t chunks = (batch + slotRows - 1) / slotRows;
    const uint64_t per = (uint64_t)slotRows * R::IPR;   // items per chunk and pass
    const uint64_t total = 2 * chunks * per;
    // stages 0 .. chunks + lag - 1; stage s holds A(s) when s < chunks and B(s - lag) when
    // s >= lag; items before stage s: per * (min(s, chunks) + max(0, s - lag))
    const uint64_t lag = kRingLag < chunks ? kRingLag : chunks;
#pragma unroll 1
    for (uint64_t pos = blockIdx.x; pos < total; pos += gridDim.x) {
        // position -> (pass, chunk, item within the chunk)
        bool passB;
        uint64_t chunk, local;
        const uint64_t q = pos / per, r = pos % per;   // q-th block of `per` items
        if (q < lag) {                                  // stages 0 .. lag-1: A only
            passB = false;
            chunk = q;
        } else if (q < lag + 2 * (chunks - lag)) {      // stages lag .. chunks-1: A then B
            const uint64_t t = q - lag;
            passB = (t & 1) != 0;
            chunk = passB ? t / 2 : lag + t / 2;
        } else {                                        // stages chunks .. chunks+lag-1: B only
            passB = true;
            chunk = chunks - lag + (q - lag - 2 * (chunks - lag));
        }
        local = r;
        const int slot = (int)(chunk % kRingSlots);
        const unsigned round = (unsigned)(chunk / kRingSlots);
        const uint64_t rowInChunk = local / R::IPR;
        const int part = (int)(local % R::IPR);
        const uint64_t row = chunk * slotRows + rowInChunk;
        float2* slotRow = ring + ((size_t)slot * slotRows + rowInChunk) * R::N;
        if (!passB) {
            if (!ring_wait(&bDone[slot], round * (unsigned)per)) return;
            if (row < batch) R::itemA(in + row * R::N, slotRow, part, smem_ring, tw1, tlo, thi);
            ring_signal(&aDone[slot]);
        } else {
            if (!ring_wait(&aDone[slot], (round + 1) * (unsigned)per)) return;
            if (row < batch) R::itemB(slotRow, out + row * R::N, part, smem_ring, tw2, scale);
            ring_signal(&bDone[slot]);
        }
    }
}

}  // namespace dev

namespace backend {

namespace {

template <int N1, bool INV>
int launchRing(const void* in, void* out, void* ring, uint32_t slotRows, uint64_t batch, float scale,
               const void* tw1, const void* tw2, const void* tlo, const void* thi, void* ctr, void* stream) {
    using R = dev::Ring<N1, INV>;
    const void* fn = (const void*)dev::k_long_ring<N1, INV>;
    static std::atomic<int> residentOn[64];
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) return (int)cudaErrorInvalidDevice;
    int resident = residentOn[device].load();
    if (!resident) {
        int sms = 0, perSm = 0;
        if (int e = optInSharedMemory(fn, R::SMEM)) return e;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, dev::k_long_ring<N1, INV>, dev::kRingThreads,
                                                          R::SMEM) != cudaSuccess || perSm < 1)
            return (int)cudaErrorInvalidConfiguration;
        resident = sms * perSm;
        residentOn[device].store(resident);
    }
    const uint64_t chunks = (batch + slotRows - 1) / slotRows;
    const uint64_t total = 2 * chunks * (uint64_t)slotRows * R::IPR;
    // per-slot item counters: position counts must stay below 2^32 (ring_wait compares u32)
    if ((chunks / dev::kRingSlots + 2) * (uint64_t)slotRows * R::IPR > 0xFFFFFFFFull) return (int)cudaErrorInvalidValue;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(ctr, 0, 2 * dev::kRingSlots * sizeof(unsigned), s) != cudaSuccess) return (int)cudaGetLastError();
    const unsigned grid = (unsigned)(total < (uint64_t)resident ? total : (uint64_t)resident);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(dev::kRingThreads);
    cfg.dynamicSmemBytes = R::SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;   // every CTA resident: the item waits always end
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return (int)cudaLaunchKernelEx(&cfg, dev::k_long_ring<N1, INV>, static_cast<const float2*>(in),
                                   static_cast<float2*>(out), static_cast<float2*>(ring),
                                   static_cast<const float2*>(tw1), static_cast<const float2*>(tw2),
                                   static_cast<const float2*>(tlo), static_cast<const float2*>(thi),
                                   static_cast<unsigned*>(ctr), batch, slotRows, scale);
}

}  // namespace

bool hasLongRing(uint32_t n) { return n == 8192 || n == 16384 || n == 32768 || n == 65536; }

int longRingSlots() { return dev::kRingSlots; }

uint32_t longRingSlotRows(uint32_t n, uint64_t batch, size_t slotBytes) {
    uint64_t rows = slotBytes / ((uint64_t)n * 8);
    if (rows < 1) rows = 1;
    if (rows > batch) rows = batch;
    return (uint32_t)rows;
}

int launchLongRing(const void* in, void* out, void* ring, uint32_t slotRows, uint32_t n, uint64_t batch,
                   bool inverse, float scale, const void* tw1, const void* tw2, const void* tlo, const void* thi,
                   void* counters, void* stream) {
    if (!hasLongRing(n) || slotRows == 0 || batch == 0) return (int)cudaErrorInvalidValue;
#define BFLY_RING(N1)                                                                                    \
    return inverse ? launchRing<N1, true>(in, out, ring, slotRows, batch, scale, tw1, tw2, tlo, thi, counters, \
                                          stream)                                                         \
                   : launchRing<N1, false>(in, out, ring, slotRows, batch, scale, tw1, tw2, tlo, thi, counters, stream)
    switch (n) {
        case 8192: BFLY_RING(32);
        case 16384: BFLY_RING(64);
        case 32768: BFLY_RING(128);
        case 65536: BFLY_RING(256);
        default: return (int)cudaErrorInvalidValue;
    }
#undef BFLY_RING
}

int longRingStatus(unsigned* status, bool clear) {
    if (cudaMemcpyFromSymbol(status, dev::g_ring_status, sizeof(unsigned)) != cudaSuccess) return 1;
    if (clear && *status) {
        const unsigned zero = 0;
        if (cudaMemcpyToSymbol(dev::g_ring_status, &zero, sizeof(unsigned)) != cudaSuccess) return 1;
    }
    return 0;
}

}  // namespace backend
}  // namespace bfly
