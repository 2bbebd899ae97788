// Long C2C (n = N1 * 256 = 8192 .. 65536) in one HBM pass: one thread-block cluster per row.
//
// The row is the N1 x 256 matrix x[256*n1 + n2] of the four-step decomposition
//   X[k1 + N1*k2] = sum_n2 W_256^(n2*k2) * W_n^(n2*k1) * sum_n1 W_N1^(n1*k1) x[256*n1 + n2].
// CTA `rank` of a C-CTA cluster owns columns n2 in [rank*COLS, (rank+1)*COLS) for step 1 and
// rows k1 in [rank*ROWS2, (rank+1)*ROWS2) for step 2.  The clusters are persistent: cluster `c`
// transforms rows c, c + clusters, ...
//   step 1: the CTA's N1 x COLS column slice arrives by a 2-D TMA tensor copy issued one row
//      ahead; the N1-point column FFTs run in place in the stage (columns across lanes:
//      conflict-free without padding); each value is multiplied by W_n^(n2*k1) (two-level
//      tables built in FP64) and sent with st.async to the CTA owning row k1, completing bytes
//      on that CTA's mbarrier -- the four-step transpose never touches HBM and the sender never
//      waits;
//   step 2: the ROWS2 x 256 receive buffer holds this CTA's rows; the 256-point row FFTs run in
//      place (rows across lanes) and X[k1 + N1*k2] is stored straight from registers: lanes
//      hold consecutive k1, so every warp store covers whole 128-byte lines.
// Software pipeline: iteration j runs step 1 of row j+1 (and sends it) before step 2 of row j,
// with two receive buffers, so the data a CTA waits for was sent one iteration earlier and the
// cluster barrier (per row: arrive after a receive buffer has been read, wait before the sends
// that reuse it) only waits on work one iteration old.
// Every mbarrier wait is bounded; a wait that runs out sets g_long_status and the CTA stops
// waiting and issuing copies but keeps the barrier schedule, so no peer is left waiting.
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include "backend.h"
#include "fft_kernels.cuh"
#include "tma.cuh"

namespace bfly {
namespace dev {

__device__ unsigned int g_long_status;

template <int N1, int C>
struct LongCluster {
    static constexpr int N2 = 256, E = 16, N = N1 * N2;
    static constexpr int NT = N / (C * E);      // threads per CTA
    static constexpr int COLS = N2 / C;         // step-1 columns per CTA
    static constexpr int T1 = N1 / E;           // threads per column
    static constexpr int ROWS2 = N1 / C;        // step-2 rows per CTA
    static constexpr int T2 = N2 / E;           // threads per row
    static constexpr int S2 = N2 + 1;           // receive row stride (odd: rows across lanes hit distinct banks)
    static constexpr uint32_t STAGE_BYTES = (uint32_t)N1 * COLS * 8;
    static constexpr uint32_t RECV_BYTES = (uint32_t)ROWS2 * N2 * 8;   // arriving per row
    static constexpr uint32_t RECV_ALLOC = ((uint32_t)ROWS2 * S2 * 8 + 127u) / 128u * 128u;
    static constexpr uint32_t BAR_OFF = STAGE_BYTES + 2 * RECV_ALLOC;
    static constexpr uint32_t SMEM = BAR_OFF + 64 + 1024;   // + slack to align the base to 1024
    static_assert(COLS * T1 == NT && ROWS2 * T2 == NT, "inconsistent cluster shape");
    static_assert(COLS >= 2 && (COLS * 8) % 16 == 0, "TMA box inner extent must be a multiple of 16 bytes");
    static_assert(2 * COLS <= 256 && N1 <= 256, "TMA box dimensions are at most 256 elements");
    static_assert(STAGE_BYTES % 1024 == 0, "the stage stays 1024-byte aligned");
    static_assert(RECV_BYTES < (1u << 20), "mbarrier transaction limit");
};

template <int N1, int C, bool INV>
__global__ void __launch_bounds__(LongCluster<N1, C>::NT, LongCluster<N1, C>::NT <= 256 ? 2 : 1)
k_long_cluster(const __grid_constant__ CUtensorMap tin, float2* __restrict__ out, const float2* __restrict__ tw1,
               const float2* __restrict__ tw2, const float2* __restrict__ tlo, const float2* __restrict__ thi,
               uint64_t batch, float scale) {
    using L = LongCluster<N1, C>;
    using TA = Team<N1, L::E, INV, kSyncBlock, L::COLS>;   // step 1, element i of a column at i*COLS
    using TB = Team<L::N2, L::E, INV, kSyncBlock, 1>;      // step 2, element i of a row at i
    extern __shared__ unsigned char smem_lc[];
    const uint32_t raw = smem_addr(smem_lc);
    unsigned char* base = smem_lc + (((raw + 1023u) & ~1023u) - raw);
    float2* const stage = reinterpret_cast<float2*>(base);
    float2* const recv0 = reinterpret_cast<float2*>(base + L::STAGE_BYTES);
    uint64_t* const bars = reinterpret_cast<uint64_t*>(base + L::BAR_OFF);   // stage, receive 0, receive 1

    const int tid = threadIdx.x;
    const uint32_t rank = cluster_ctarank();
    const uint64_t cid = blockIdx.x / C, clusters = gridDim.x / C;
    const uint64_t rows = cid < batch ? (batch - cid + clusters - 1) / clusters : 0;
    const int x0 = (int)(rank * L::COLS * 2);   // box origin in floats: rank*COLS*8 bytes, 16-byte multiple
    bool ok = true;
    uint64_t issued = 0, consumed = 0;          // stage copies issued / waited for (thread 0)

    const int c = tid % L::COLS, t1 = tid / L::COLS;     // step-1 column and thread-in-column
    const int r = tid % L::ROWS2, t2 = tid / L::ROWS2;   // step-2 row and thread-in-row
    const uint32_t n2 = rank * L::COLS + c;
    auto recv = [&](uint64_t j) { return recv0 + (j & 1) * (L::RECV_ALLOC / 8); };

    auto issue = [&](uint64_t j) {   // thread 0: row j's slice into the stage
        mbar_arrive_expect_tx(&bars[0], L::STAGE_BYTES);
        tensor_load_2d(stage, &tin, x0, (int)((cid + j * clusters) * N1), &bars[0]);
    };
    // step 1 of row j into v; refills the stage with row j + 1
    auto step1 = [&](uint64_t j, float2 (&v)[L::E]) {
        if (ok) ok = mbar_wait_bounded(&bars[0], (uint32_t)j & 1u);
        if (ok && tid == 0) consumed = j + 1;
        float2* col = stage + c;
        TA::load_first(v, t1, [&](int i) { return col[i * L::COLS]; });
        __syncthreads();
        TA::template passes<0>(v, col, tw1, t1, 0);
        fence_proxy_async_smem();   // this thread's exchange writes precede the TMA refill
        __syncthreads();            // the stage is free
        if (tid == 0 && ok && issued < rows) issue(issued++);
        TA::for_each_slot(v, t1, [&](int k1, float2& x) {
            const uint32_t m = n2 * (uint32_t)k1;   // < n
            x = cmul<INV>(x, cmul<false>(__ldg(thi + (m >> 8)), __ldg(tlo + (m & 255u))));
        });
    };
    // send row j's step-1 values to their owners' receive buffer j&1
    auto send = [&](uint64_t j, float2 (&v)[L::E]) {
        const uint32_t rbase = smem_addr(recv(j) + n2);
        const uint32_t rbar = smem_addr(&bars[1 + (j & 1)]);
        TA::for_each_out(v, t1, [&](int k1, float2 x) {
            const uint32_t owner = (uint32_t)k1 / L::ROWS2;
            const uint32_t off = ((uint32_t)k1 % L::ROWS2) * L::S2 * 8u;
            st_async_f2(cluster_map(rbase + off, owner), x, cluster_map(rbar, owner));
        });
    };

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&bars[2], 1);
        fence_mbar_init();
        if (rows > 0) issue(issued++);
        if (rows > 0) mbar_arrive_expect_tx(&bars[1], L::RECV_BYTES);
        if (rows > 1) mbar_arrive_expect_tx(&bars[2], L::RECV_BYTES);
    }
    __syncthreads();
    cluster_arrive();
    cluster_wait();     // every CTA of the cluster runs and has initialised its barriers
    float2 v[L::E];
    if (rows > 0) {
        step1(0, v);
        send(0, v);
    }
    cluster_arrive();   // receive buffer 1 has never been used
    for (uint64_t j = 0; j < rows; ++j) {
        if (j + 1 < rows) step1(j + 1, v);
        cluster_wait();  // every CTA has read receive buffer (j+1)&1 (row j-1)
        if (j + 1 < rows) send(j + 1, v);
        if (ok) ok = mbar_wait_cluster_bounded(&bars[1 + (j & 1)], (uint32_t)(j >> 1) & 1u);
        float2* row = recv(j) + r * L::S2;
        TB::load_first(v, t2, [&](int i) { return row[i]; });
        __syncthreads();
        TB::template passes<0>(v, row, tw2, t2, 0);
        if (tid == 0 && ok && j + 2 < rows) mbar_arrive_expect_tx(&bars[1 + (j & 1)], L::RECV_BYTES);
        cluster_arrive();   // this thread is done with receive buffer j&1
        float2* dst = out + (cid + j * clusters) * (uint64_t)L::N + rank * L::ROWS2 + r;
        TB::for_each_out(v, t2, [&](int k2, float2 x) { st_stream(dst + (size_t)k2 * N1, cscale(x, scale)); });
    }
    cluster_wait();   // pairs the last arrive: no CTA leaves while a peer may still write to it
    if (!ok) atomicOr(&g_long_status, 1u);
    if (tid == 0)     // after a failed wait: let every copy this CTA issued land before leaving
        for (uint64_t j = consumed; j < issued; ++j) mbar_wait_bounded(&bars[0], (uint32_t)j & 1u);
}

}  // namespace dev

namespace backend {

namespace {

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    return fn;
}

constexpr int kMaxDevices = 64;

template <int N1, int C, bool INV>
int launchCluster(const void* in, void* out, uint64_t batch, float scale, const void* tw1, const void* tw2,
                  const void* tlo, const void* thi, void* stream) {
    using L = dev::LongCluster<N1, C>;
    auto* kern = dev::k_long_cluster<N1, C, INV>;
    static std::atomic<int> maxClusters[kMaxDevices];   // 0 = not yet configured on that device
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
        return (int)cudaErrorInvalidDevice;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(L::NT);
    cfg.dynamicSmemBytes = L::SMEM;
    cfg.stream = reinterpret_cast<cudaStream_t>(stream);
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int mc = maxClusters[device].load();
    if (mc == 0) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM) != cudaSuccess)
            return 1;
        if (C > 8 && cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
            return 1;
        cfg.gridDim = dim3(C);
        if (cudaOccupancyMaxActiveClusters(&mc, kern, &cfg) != cudaSuccess || mc <= 0) return 1;
        maxClusters[device].store(mc);
    }
    if (batch == 0) return 0;
    if (batch * N1 > 0x7fffffffull) return (int)cudaErrorInvalidValue;   // box row coordinate is an int
    EncodeTiled encode = encoder();
    if (!encode) return 1;
    CUtensorMap tm;
    const cuuint64_t gdim[2] = {2ull * L::N2, batch * (uint64_t)N1};   // floats per matrix row, matrix rows
    const cuuint64_t gstride[1] = {2ull * L::N2 * 4};
    const cuuint32_t box[2] = {2u * L::COLS, (cuuint32_t)N1};
    const cuuint32_t estride[2] = {1, 1};
    if (encode(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(in), gdim, gstride, box, estride,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return 1;
    const uint64_t clusters = batch < (uint64_t)mc ? batch : (uint64_t)mc;
    cfg.gridDim = dim3((unsigned)(clusters * C));
    return (int)cudaLaunchKernelEx(&cfg, kern, tm, static_cast<float2*>(out), static_cast<const float2*>(tw1),
                                   static_cast<const float2*>(tw2), static_cast<const float2*>(tlo),
                                   static_cast<const float2*>(thi), batch, scale);
}

}  // namespace

// (n, threads per CTA) -> cluster size: C = n / (16 * cta).
bool hasLongCluster(uint32_t n, int cta) {
    switch (n) {
        case 8192: return cta == 256;
        case 16384:
        case 32768:
        case 65536: return cta == 256 || cta == 512;
        default: return false;
    }
}

int launchLongCluster(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale,
                      const void* tw1, const void* tw2, const void* tlo, const void* thi, int cta, void* stream) {
    if (!hasLongCluster(n, cta)) return (int)cudaErrorInvalidValue;
    if (reinterpret_cast<uintptr_t>(in) % 16 != 0) return kLongClusterUnaligned;   // tensor-map base rule
#define BFLY_LC(N1, C)                                                                              \
    return inverse ? launchCluster<N1, C, true>(in, out, batch, scale, tw1, tw2, tlo, thi, stream) \
                   : launchCluster<N1, C, false>(in, out, batch, scale, tw1, tw2, tlo, thi, stream)
    switch (n * 2 + (cta == 512)) {
        case 2 * 8192: BFLY_LC(32, 2);
        case 2 * 16384: BFLY_LC(64, 4);
        case 2 * 16384 + 1: BFLY_LC(64, 2);
        case 2 * 32768: BFLY_LC(128, 8);
        case 2 * 32768 + 1: BFLY_LC(128, 4);
        case 2 * 65536: BFLY_LC(256, 16);
        case 2 * 65536 + 1: BFLY_LC(256, 8);
        default: return (int)cudaErrorInvalidValue;
    }
#undef BFLY_LC
}

int longClusterStatus(unsigned* status, bool clear) {
    if (cudaMemcpyFromSymbol(status, dev::g_long_status, sizeof(unsigned)) != cudaSuccess) return 1;
    if (clear && *status) {
        const unsigned zero = 0;
        if (cudaMemcpyToSymbol(dev::g_long_status, &zero, sizeof(unsigned)) != cudaSuccess) return 1;
    }
    return 0;
}

}  // namespace backend
}  // namespace bfly
