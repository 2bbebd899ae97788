// Split-BF16 tensor-core C2C for power-of-two lengths 64..4096: every radix-16 pass is a dense
// complex contraction on the 5th-generation tensor cores; lengths that are not powers of 16 end
// with one radix-2/4/8 pass on the CUDA cores in fp32 (64 = 16 x 4, 128 = 16 x 8,
// 512 = 16 x 16 x 2, 1024 = 16 x 16 x 4, 2048 = 16 x 16 x 8).
//
// Pass structure (Stockham, as in fft_core.cuh, one butterfly per thread): thread t owns
// butterfly j of its row and holds the 16 (twiddled, fp32) inputs x_0..x_15.  As reals they form
// row t of an A operand (M = 128 butterflies per tile, K = 32: Re x_0..15, Im x_0..15).  The
// 32 x 32 real matrix of DFT-16 is the B operand (K-major, N = 32 outputs: Re y_0..15,
// Im y_0..15).  Both are split into bf16 terms, a = a_hi + a_lo (+ a_mid for three terms), and
// D = sum over term pairs A_s * B_t accumulates in fp32 in tensor memory (two terms: 3 products
// hi*hi + hi*lo + lo*hi; three terms: 6 products down to 2^-24).  tcgen05.ld returns D's row
// t -- the 16 outputs of butterfly t -- to thread t, which writes them to the Stockham
// positions of the next pass (or, after the last pass, to global memory).
// Twiddles between passes stay fp32 (the Stockham tables of the CUDA-core path, E = 16).
// Inverse transforms use IDFT(x) = conj(DFT(conj x)).
#include <atomic>

#include "backend.h"
#include "fft_kernels.cuh"
#include "registry.cuh"
#include "tcgen05.cuh"

#include <cuda_bf16.h>

namespace bfly {
namespace dev {

__device__ unsigned int g_tc_status;   // nonzero: a bounded wait for an MMA ran out

constexpr int kTcThreads = 256;
constexpr int kTileBytes = 128 * 32 * 2;   // one A tile: 128 rows x 32 bf16
constexpr int kBBytes = 32 * 32 * 2;       // one B term: 32 rows x 32 bf16

// Byte offset of element (row, k) in a no-swizzle K-major operand with K = 32: 8-row x 8-element
// core matrices of 128 bytes, LBO = 128 (next 8 k), SBO = 512 (next 8 rows).
__host__ __device__ constexpr uint32_t kmajor_offset(int row, int k) {
    return (uint32_t)((row >> 3) * 512 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(a)) |
           ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(b)) << 16);
}

// Split v into SPLIT bf16-representable terms (returned as floats, largest first).
template <int SPLIT>
__device__ __forceinline__ void split_terms(float v, float (&t)[SPLIT]) {
    float r = v;
#pragma unroll
    for (int s = 0; s < SPLIT; ++s) {
        t[s] = __bfloat162float(__float2bfloat16_rn(r));
        r = r - t[s];
    }
}

// Split a pair of values into SPLIT packed bf16x2 terms (one conversion per term for both).
template <int SPLIT>
__device__ __forceinline__ void split_pair(float a, float b, uint32_t (&t)[SPLIT]) {
    float ra = a, rb = b;
#pragma unroll
    for (int s = 0; s < SPLIT; ++s) {
        const __nv_bfloat162 h = __float22bfloat162_rn(make_float2(ra, rb));
        t[s] = *reinterpret_cast<const uint32_t*>(&h);
        ra = ra - __low2float(h);
        rb = rb - __high2float(h);
    }
}

// The SPLIT bf16 terms of the 32 x 32 real DFT-16 matrix in the K-major canonical layout
// (SPLIT x 2048 bytes), computed once in FP64: row n = output (Re y_0..15, Im y_0..15), column
// k = input (Re x_0..15, Im x_0..15):
//   Re y_n = sum_k c_nk Re x_k + s_nk Im x_k,  Im y_n = sum_k -s_nk Re x_k + c_nk Im x_k,
//   c_nk = cos(2 pi n k / 16), s_nk = sin(2 pi n k / 16)
template <int SPLIT>
__global__ void k_tc_dft_table(unsigned char* __restrict__ table) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 32 * 32) return;
    const int n = e >> 5, k = e & 31;
    double sn, cs;
    sincospi((double)(((n & 15) * (k & 15)) & 15) / 8.0, &sn, &cs);   // multiples of pi/8
    const float v = (float)((n < 16) ? (k < 16 ? cs : sn) : (k < 16 ? -sn : cs));
    float parts[SPLIT];
    split_terms<SPLIT>(v, parts);
#pragma unroll
    for (int s = 0; s < SPLIT; ++s)
        *reinterpret_cast<__nv_bfloat16*>(table + s * kBBytes + kmajor_offset(n, k)) = __float2bfloat16_rn(parts[s]);
}

template <int N, int SPLIT>
__global__ void __launch_bounds__(kTcThreads, SPLIT == 2 ? 3 : 2)
k_c2c_tc(const float2* __restrict__ in, float2* __restrict__ out, const float2* __restrict__ tw,
         const unsigned char* __restrict__ dftTable, uint64_t batch, int direction, float scale) {
    constexpr int E = 16;
    using Sd = Sched<N, E>;
    constexpr int T = N / E;                      // radix-16 butterflies per row = threads per row
    constexpr int ROWS = kTcThreads / T;
    static_assert(ROWS * T == kTcThreads, "rows fill the CTA");
    constexpr int S = smem_stride<N, E, false>();
    constexpr int P = Sd::P;
    constexpr int RL = Sd::radix(P - 1);          // last radix: 16, or 2/4/8 on the CUDA cores
    constexpr int PT = RL == 16 ? P : P - 1;      // passes on the tensor cores
    static_assert(PT >= 1, "at least one radix-16 pass");
    constexpr int NPROD = SPLIT == 2 ? 3 : 6;

    extern __shared__ __align__(1024) unsigned char smem_tc[];
    unsigned char* aBase = smem_tc;                                   // [SPLIT][2 tiles][8 KB]
    unsigned char* bBase = smem_tc + SPLIT * 2 * kTileBytes;          // [SPLIT][2 KB]
    float2* xbuf = reinterpret_cast<float2*>(bBase + SPLIT * kBBytes);
    uint64_t* bar = reinterpret_cast<uint64_t*>(xbuf + ROWS * S);
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(bar + 1);

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    if (warp == 0) {
        tmem_alloc(tmemSlot, 64);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    // the DFT operand terms, built once per plan (k_tc_dft_table), copied into shared memory
    for (int i = tid; i < SPLIT * kBBytes / 16; i += kTcThreads)
        reinterpret_cast<uint4*>(bBase)[i] = __ldg(reinterpret_cast<const uint4*>(dftTable) + i);
    fence_proxy_async_smem();
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tmem = *tmemSlot;

    const int rl = tid / T;
    const int j = tid - rl * T;
    const float sgn = direction > 0 ? -1.f : 1.f;
    const int tile = tid >> 7, m = tid & 127;
    float2* xr = xbuf + rl * S;
    constexpr uint32_t idesc = umma_idesc_bf16(128, 32);
    const uint64_t groups = (batch + ROWS - 1) / ROWS;
    bool failed = false;
    uint32_t phase = 0;
#pragma unroll 1
    for (uint64_t grp = blockIdx.x; grp < groups && !failed; grp += gridDim.x) {
        const uint64_t row = grp * ROWS + rl;
        const bool ok = row < batch;
        const float2* src = in + row * N;
        float2* dst = out + row * N;
        float2 v[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            float2 x = ok ? ld_stream(src + j + r * (N / 16)) : make_float2(0.f, 0.f);
            v[r] = make_float2(x.x, sgn * x.y);
        }
#pragma unroll 1
        for (int p = 0; p < PT; ++p) {
            const int Ns = Sd::ns(p);
            if (p > 0) {
                const float2* twp = tw + Sd::twoff(p);
                const int k = j & (Ns - 1);
#pragma unroll
                for (int r = 1; r < 16; ++r) v[r] = cmul<false>(v[r], __ldg(twp + (r - 1) * Ns + k));
            }
            // A terms of this butterfly: row m of tile `tile`, K chunks (Re 0-7, Re 8-15, Im 0-7, Im 8-15)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                uint32_t q[4][SPLIT];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int r = (c & 1) * 8 + 2 * e;
                    if (c < 2) split_pair<SPLIT>(v[r].x, v[r + 1].x, q[e]);
                    else split_pair<SPLIT>(v[r].y, v[r + 1].y, q[e]);
                }
#pragma unroll
                for (int s = 0; s < SPLIT; ++s)
                    *reinterpret_cast<uint4*>(aBase + (s * 2 + tile) * kTileBytes + kmajor_offset(m, c * 8)) =
                        make_uint4(q[0][s], q[1][s], q[2][s], q[3][s]);
            }
            fence_proxy_async_smem();
            tc_fence_before_sync();
            __syncthreads();
            if (tid == 0) {
                tc_fence_after_sync();
                // products (A term, B term), smallest first
                constexpr int pa[6] = {2, 1, 0, 1, 0, 0};
                constexpr int pb[6] = {0, 1, 2, 0, 1, 0};
                constexpr int pa2[3] = {1, 0, 0};
                constexpr int pb2[3] = {0, 1, 0};
#pragma unroll
                for (int tl = 0; tl < 2; ++tl) {
#pragma unroll
                    for (int q = 0; q < NPROD; ++q) {
                        const int sa = SPLIT == 2 ? pa2[q] : pa[q];
                        const int sb = SPLIT == 2 ? pb2[q] : pb[q];
#pragma unroll
                        for (int ks = 0; ks < 2; ++ks) {
                            const uint32_t aAddr = smem_addr(aBase + (sa * 2 + tl) * kTileBytes) + ks * 256;
                            const uint32_t bAddr = smem_addr(bBase + sb * kBBytes) + ks * 256;
                            umma_bf16(tmem + tl * 32, umma_smem_desc(aAddr, 128, 512),
                                      umma_smem_desc(bAddr, 128, 512), idesc, q > 0 || ks > 0);
                        }
                    }
                }
                umma_commit(bar);
            }
            const bool done = mbar_wait_bounded(bar, phase);
            if (__syncthreads_or(!done)) {
                failed = true;
                break;
            }
            phase ^= 1u;
            tc_fence_after_sync();
            float d[32];
            tmem_ld_32cols(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(tile * 32), d);
#pragma unroll
            for (int r = 0; r < 16; ++r) v[r] = make_float2(d[r], d[16 + r]);
            if (p < P - 1) {
                const int k = j & (Ns - 1);
                const int base = (j - k) * 16 + k;
#pragma unroll
                for (int r = 0; r < 16; ++r) xr[spad(base + r * Ns)] = v[r];
                tc_fence_before_sync();
                __syncthreads();
                // next pass's inputs: one radix-16 butterfly, or 16/RL radix-RL butterflies
                // j + s T (elements r N/RL) for the final CUDA-core pass
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    v[i] = p + 1 < PT ? xr[spad(j + i * (N / 16))]
                                      : xr[spad(j + (i / RL) * T + (i % RL) * (N / RL))];
            }
        }
        if constexpr (RL < 16) {   // final radix-RL pass in fp32 (Stockham, as fft_core.cuh)
            constexpr int Ns = N / RL;
            const float2* twp = tw + Sd::twoff(P - 1);
#pragma unroll
            for (int sb = 0; sb < 16 / RL; ++sb) {
                const int k = (j + sb * T) & (Ns - 1);
#pragma unroll
                for (int r = 1; r < RL; ++r)
                    v[sb * RL + r] = cmul<false>(v[sb * RL + r], __ldg(twp + (r - 1) * Ns + k));
                DFT<RL, false>::run(&v[sb * RL]);
            }
        }
        if (!failed && ok) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int idx = RL == 16 ? j + i * (N / 16) : j + (i / RL) * T + (i % RL) * (N / RL);
                st_stream(dst + idx, make_float2(v[i].x * scale, sgn * scale * v[i].y));
            }
        }
        // the exchange buffer and the A operand are rewritten by the next group
        tc_fence_before_sync();
        __syncthreads();
    }
    if (failed && tid == 0) {
        atomicOr(&g_tc_status, 1u);
        mbar_wait_bounded(bar, phase);   // let the MMAs in flight finish if they can
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 64);
}

template <int N, int SPLIT>
constexpr int tcSmemBytes() {
    return SPLIT * 2 * kTileBytes + SPLIT * kBBytes +
           (kTcThreads / (N / 16)) * smem_stride<N, 16, false>() * 8 + 16;
}

}  // namespace dev

namespace backend {

template <int N, int SPLIT>
static int launchTc(const void* in, void* out, uint64_t batch, bool inverse, float scale, const void* tw,
                    const void* table, void* stream) {
    constexpr int smem = dev::tcSmemBytes<N, SPLIT>();
    static std::atomic<int> residentOn[64];   // CTAs resident on each device (persistent grid)
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) return (int)cudaErrorInvalidDevice;
    int resident = residentOn[device].load();
    if (!resident) {
        int sms = 0, perSm = 0;
        if (optInSharedMemory((const void*)dev::k_c2c_tc<N, SPLIT>, smem) ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, dev::k_c2c_tc<N, SPLIT>, dev::kTcThreads, smem) !=
                cudaSuccess)
            return 1;
        resident = sms * (perSm > 0 ? perSm : 1);
        residentOn[device].store(resident);
    }
    constexpr int rows = dev::kTcThreads / (N / 16);
    const uint64_t groups = (batch + rows - 1) / rows;
    const unsigned grid = (unsigned)(groups < (uint64_t)resident ? groups : (uint64_t)resident);
    dev::k_c2c_tc<N, SPLIT><<<grid, dev::kTcThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const float2*>(in), static_cast<float2*>(out), static_cast<const float2*>(tw),
        static_cast<const unsigned char*>(table), batch, inverse ? 1 : -1, scale);
    return (int)cudaGetLastError();
}

bool hasTensorVariant(uint32_t n, int split) {
    return n >= 64 && n <= 4096 && !(n & (n - 1)) && (split == 2 || split == 3);
}

size_t tensorTableBytes(int split) { return (size_t)split * dev::kBBytes; }

int buildTensorTable(void* table, int split, void* stream) {
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (split == 2) dev::k_tc_dft_table<2><<<4, 256, 0, st>>>(static_cast<unsigned char*>(table));
    else if (split == 3) dev::k_tc_dft_table<3><<<4, 256, 0, st>>>(static_cast<unsigned char*>(table));
    else return (int)cudaErrorInvalidValue;
    return (int)cudaGetLastError();
}

int launchC2CTensor(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale,
                    const void* tw, const void* table, int split, void* stream) {
#define BFLY_TC(NN)                                                                                   \
    if (n == NN && split == 2) return launchTc<NN, 2>(in, out, batch, inverse, scale, tw, table, stream); \
    if (n == NN && split == 3) return launchTc<NN, 3>(in, out, batch, inverse, scale, tw, table, stream);
    BFLY_TC(64)
    BFLY_TC(128)
    BFLY_TC(256)
    BFLY_TC(512)
    BFLY_TC(1024)
    BFLY_TC(2048)
    BFLY_TC(4096)
#undef BFLY_TC
    return (int)cudaErrorInvalidValue;
}

int tensorStatus(unsigned* status, bool clear) {
    if (cudaMemcpyFromSymbol(status, dev::g_tc_status, sizeof(unsigned)) != cudaSuccess) return 1;
    if (clear && *status) {
        const unsigned zero = 0;
        if (cudaMemcpyToSymbol(dev::g_tc_status, &zero, sizeof(unsigned)) != cudaSuccess) return 1;
    }
    return 0;
}

}  // namespace backend
}  // namespace bfly
