// Split-BF16 tensor-core C2C for power-of-two lengths 64..4096: every radix-16 pass is a dense
// complex contraction on the 5th-generation tensor cores; lengths that are not powers of 16 end
// with one radix-2/4/8 pass on the CUDA cores in fp32 (64 = 16 x 4, 128 = 16 x 8,
// 512 = 16 x 16 x 2, 1024 = 16 x 16 x 4, 2048 = 16 x 16 x 8).
//
// Contraction.  A radix-16 butterfly's 16 (twiddled, fp32) inputs x_0..15 form one row of the A
// operand (K = 32 reals: Re x_0..15, Im x_0..15); the 32 x 32 real matrix of DFT-16 is the B
// operand (N = 32 outputs: Re y_0..15, Im y_0..15).  M = 128 butterflies per tile, two tiles per
// CTA (256 butterflies: one per thread).  Both operands are split into bf16 terms and
// D = sum over term pairs A_s * B_t accumulates in fp32 in tensor memory:
//   three terms: x = x0 + x1 + x2 EXACTLY, by truncation (x0 = the top 16 bits of x, x1 = the
//     top 16 bits of x - x0, x2 = the rest, which has at most 8 significant bits), packed two
//     values per 32-bit word with one byte permute -- no conversion instructions; the DFT terms
//     are round-to-nearest splits built in FP64; six products x_s W_t with s + t <= 2;
//   two terms: round-to-nearest x = x0 + x1 (+ a residual below 2^-17 |x|), three products.
//
// Exchange.  tcgen05.ld returns D's row to the thread that owns it: the 16 outputs of one
// butterfly.  Stockham pass p (Ns = 16^p) sends output r of butterfly j (k = j mod Ns) to
// element (j - k) 16 + k + r Ns, which pass p + 1 reads as input r' of butterfly j', with
// j' = base + r Ns and r' constant over r (for every pass followed by another tensor-core pass,
// Ns <= n / 256).  Ordering pass p + 1's A rows as l = a 16 Ns + 16 k + r for butterfly
// j' = a 16 Ns + r Ns + k makes those 16 destinations 16 consecutive rows at one K: the thread
// writes them straight into the next A operand in the MN-major layout (8 rows x 16 bytes per
// store), so the exchange between tensor-core passes is the operand write itself.  Pass 0's
// operand is written K-major (each thread its own row).  The first pass reads global memory,
// the last writes an fp32 staging buffer in natural order (or the final radix-2/4/8 pass reads
// it), from which the stores to global memory are coalesced.
// Twiddles of passes p >= 1 come from a table in the permuted row order (coalesced loads).
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
constexpr int kBBytes = 32 * 32 * 2;       // one B term: 32 rows x 32 bf16
// A tile: 128 rows x 32 bf16.  K-major: 8-row x 8-K core matrices of 128 bytes, LBO 128 (next 8
// K), SBO 512 (next 8 rows).  MN-major: core matrices of 8 rows x 8 K (16-byte lines along the
// rows), SBO 144 between 8-row groups (one 16-byte pad per group spreads the stores of lanes
// writing different row groups over the banks), LBO 16 * 144 between 8-K groups.
constexpr uint32_t kMnSbo = 144, kMnLbo = 16 * kMnSbo;
constexpr int kTileBytes = 4 * kMnLbo;     // 9216 (the K-major layout uses the first 8192)

__host__ __device__ constexpr uint32_t kmajor_chunk(int row, int kc) {   // 8 K values of one row
    return (uint32_t)((row >> 3) * 512 + kc * 128 + (row & 7) * 16);
}
__host__ __device__ constexpr uint32_t mnmajor_chunk(int row8, int k) {  // 8 rows (row8 % 8 == 0) at one K
    return (uint32_t)((k >> 3) * kMnLbo + (row8 >> 3) * kMnSbo + (k & 7) * 16);
}
__host__ __device__ constexpr uint32_t kmajor_offset(int row, int k) {
    return kmajor_chunk(row, k >> 3) + (uint32_t)(k & 7) * 2;
}

// Round-to-nearest split of a pair into SPLIT packed bf16x2 terms.
template <int SPLIT>
__device__ __forceinline__ void split_pair_rn(float a, float b, uint32_t (&t)[SPLIT]) {
    float ra = a, rb = b;
#pragma unroll
    for (int s = 0; s < SPLIT; ++s) {
        const __nv_bfloat162 h = __float22bfloat162_rn(make_float2(ra, rb));
        t[s] = *reinterpret_cast<const uint32_t*>(&h);
        ra = ra - __low2float(h);
        rb = rb - __high2float(h);
    }
}

// Exact three-term truncation split of a pair: each term holds the top 16 bits of what is left.
__device__ __forceinline__ void split_pair_trunc3(float a, float b, uint32_t (&t)[3]) {
    uint32_t ua = __float_as_uint(a), ub = __float_as_uint(b);
    t[0] = __byte_perm(ua, ub, 0x7632);
    const float ra = a - __uint_as_float(ua & 0xffff0000u);
    const float rb = b - __uint_as_float(ub & 0xffff0000u);
    ua = __float_as_uint(ra);
    ub = __float_as_uint(rb);
    t[1] = __byte_perm(ua, ub, 0x7632);
    const float qa = ra - __uint_as_float(ua & 0xffff0000u);
    const float qb = rb - __uint_as_float(ub & 0xffff0000u);
    t[2] = __byte_perm(__float_as_uint(qa), __float_as_uint(qb), 0x7632);
}

template <int SPLIT>
__device__ __forceinline__ void split_pair(float a, float b, uint32_t (&t)[SPLIT]) {
    if constexpr (SPLIT == 3) split_pair_trunc3(a, b, t);
    else split_pair_rn<SPLIT>(a, b, t);
}

// Split the 16 values of v into SPLIT terms and store the four 16-byte chunks of each term:
// chunk 0 = Re v_0..7, 1 = Re v_8..15, 2 = Im v_0..7, 3 = Im v_8..15, at byte offsets off[c] of
// every term's tile (term s of tile `tile` at aBase + (2 s + tile) kTileBytes).
template <int SPLIT>
__device__ __forceinline__ void store_terms(const float2 (&v)[16], unsigned char* aBase, int tile,
                                            const uint32_t (&off)[4]) {
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
            *reinterpret_cast<uint4*>(aBase + (s * 2 + tile) * kTileBytes + off[c]) =
                make_uint4(q[0][s], q[1][s], q[2][s], q[3][s]);
    }
}

// The SPLIT bf16 terms of the 32 x 32 real DFT-16 matrix in the K-major canonical layout
// (SPLIT x 2048 bytes), computed once in FP64 and split by rounding to nearest: row n = output
// (Re y_0..15, Im y_0..15), column k = input (Re x_0..15, Im x_0..15):
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
    float r = v;
#pragma unroll
    for (int s = 0; s < SPLIT; ++s) {
        const __nv_bfloat16 h = __float2bfloat16_rn(r);
        *reinterpret_cast<__nv_bfloat16*>(table + s * kBBytes + kmajor_offset(n, k)) = h;
        r -= __bfloat162float(h);
    }
}

// Row order of the A operand of tensor-core pass p >= 1 (Ns = 16^(p-1), the previous pass's
// span): row l = a 16 Ns + 16 k + r holds butterfly j = a 16 Ns + r Ns + k.
__host__ __device__ constexpr int tc_butterfly(int l, int nsPrev) {
    return (l / (16 * nsPrev)) * 16 * nsPrev + (l % 16) * nsPrev + (l % (16 * nsPrev)) / 16;
}

// Twiddles of the tensor-core passes p = 1 .. PT-1 by operand row: entry (p-1) 16 T + r T + l
// = exp(-2 pi i r k / (16 Ns_p)) for input r of the butterfly j in row l, k = j mod Ns_p (r = 0
// gives 1).  A writer stores input r of the 16 consecutive rows l0..l0+15 and reads their 16
// consecutive entries.  FP64, rounded once.
template <int N>
__global__ void k_tc_twiddles(float2* __restrict__ tw) {
    constexpr int T = N / 16;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int p = 1 + i / (16 * T);
    const int rem = i % (16 * T);
    const int r = rem / T, l = rem % T;
    int ns = 1;
    for (int q = 0; q < p; ++q) ns *= 16;
    if (ns * 16 > N) return;   // past the last tensor-core pass
    const int j = tc_butterfly(l, ns / 16);
    const int k = j % ns;
    double s, c;
    sincospi(-2.0 * (double)(r * k) / (double)(16 * ns), &s, &c);
    tw[i] = make_float2((float)c, (float)s);
}

template <int N>
__host__ __device__ constexpr int tcPasses() {   // radix-16 passes (on the tensor cores)
    int p = 0;
    for (int m = N; m >= 16; m /= 16) ++p;
    return p;
}

template <int N, int SPLIT>
__global__ void __launch_bounds__(kTcThreads, 3)
k_c2c_tc(const float2* __restrict__ in, float2* __restrict__ out, const float2* __restrict__ tw,
         const float2* __restrict__ twTc, const unsigned char* __restrict__ dftTable, uint64_t batch,
         int direction, float scale) {
    using Sd = Sched<N, 16>;
    constexpr int T = N / 16;                     // radix-16 butterflies per row = threads per row
    constexpr int ROWS = kTcThreads / T;
    static_assert(ROWS * T == kTcThreads, "rows fill the CTA");
    constexpr int S = smem_stride<N, 16, false>();
    constexpr int PT = tcPasses<N>();             // passes on the tensor cores
    constexpr int RL = N >> (4 * PT);             // 1: the last pass is radix 16; else 2/4/8 in fp32
    static_assert(PT >= 1 && (RL == 1 || RL == 2 || RL == 4 || RL == 8), "schedule");
    static_assert(PT <= 2 || T >= 256, "fused exchange needs Ns <= n/256 before every tensor-core pass");
    constexpr int NPROD = SPLIT == 2 ? 3 : 6;

    extern __shared__ __align__(1024) unsigned char smem_tc[];
    unsigned char* aBase = smem_tc;                                   // [SPLIT][2 tiles]
    unsigned char* bBase = smem_tc + SPLIT * 2 * kTileBytes;          // [SPLIT][2 KB]
    float2* stage = reinterpret_cast<float2*>(smem_tc);               // aliases the A tiles (after the last MMA)
    uint64_t* bar = reinterpret_cast<uint64_t*>(bBase + SPLIT * kBBytes);
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(bar + 1);
    static_assert(ROWS * S * 8 <= SPLIT * 2 * kTileBytes, "staging fits in the A tiles");

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
    for (int i = tid; i < SPLIT * kBBytes / 16; i += kTcThreads)
        reinterpret_cast<uint4*>(bBase)[i] = __ldg(reinterpret_cast<const uint4*>(dftTable) + i);
    fence_proxy_async_smem();
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tmem = *tmemSlot;

    const int tile = tid >> 7, m = tid & 127;     // this thread's D row
    const int rl = tid / T;                       // transform row in the group
    const int l = tid - rl * T;                   // A row within the transform
    const float sgn = direction > 0 ? -1.f : 1.f;
    const uint64_t groups = (batch + ROWS - 1) / ROWS;
    bool failed = false;
    uint32_t phase = 0;
#pragma unroll 1
    for (uint64_t grp = blockIdx.x; grp < groups && !failed; grp += gridDim.x) {
        const uint64_t row0 = grp * ROWS;
        float2 v[16];
        {   // pass 0 inputs: butterfly l reads x[l + r T]
            const uint64_t row = row0 + rl;
            const bool ok = row < batch;
            const float2* src = in + row * N;
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                const float2 x = ok ? ld_stream(src + l + r * T) : make_float2(0.f, 0.f);
                v[r] = make_float2(x.x, sgn * x.y);
            }
            const uint32_t off[4] = {kmajor_chunk(m, 0), kmajor_chunk(m, 1), kmajor_chunk(m, 2), kmajor_chunk(m, 3)};
            store_terms<SPLIT>(v, aBase, tile, off);
        }
#pragma unroll
        for (int p = 0; p < PT; ++p) {
            // ---- the contraction of pass p on the operand in shared memory
            fence_proxy_async_smem();
            tc_fence_before_sync();
            __syncthreads();
            if (tid == 0) {
                tc_fence_after_sync();
                const uint32_t idesc = umma_idesc_bf16(128, 32) | (p > 0 ? (1u << 15) : 0u);   // A MN-major after pass 0
                constexpr int pa[6] = {2, 1, 0, 1, 0, 0};   // (A term, B term), smallest products first
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
                            const uint32_t aTile = smem_addr(aBase + (sa * 2 + tl) * kTileBytes);
                            const uint64_t aDesc = p == 0 ? umma_smem_desc(aTile + ks * 256, 128, 512)
                                                          : umma_smem_desc(aTile + ks * 2 * kMnLbo, kMnLbo, kMnSbo);
                            const uint32_t bAddr = smem_addr(bBase + sb * kBBytes) + ks * 256;
                            umma_bf16(tmem + tl * 32, aDesc, umma_smem_desc(bAddr, 128, 512), idesc, q > 0 || ks > 0);
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
            {
                float d[32];
                tmem_ld_32cols(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(tile * 32), d);
#pragma unroll
                for (int r = 0; r < 16; ++r) v[r] = make_float2(d[r], d[16 + r]);
            }
            // ---- butterfly j of pass p (row l of its operand) produced outputs v[0..15]
            int nsPrev = 1;
#pragma unroll
            for (int q = 1; q < p; ++q) nsPrev *= 16;
            const int ns = p == 0 ? 1 : nsPrev * 16;
            const int j = p == 0 ? l : tc_butterfly(l, nsPrev);
            const int k = j & (ns - 1);
            if (p + 1 < PT) {
                // next operand: rows a 16 ns + 16 k + r at K = r' (MN-major), twiddled first
                const int i0 = (j - k) * 16 + k;
                const int rp = i0 / T;
                const int base = i0 % T;
                const int l0 = (base / (16 * ns)) * 16 * ns + 16 * k;
                // pass p + 1's twiddles of input r' for the destination rows l0 .. l0 + 15
                const float4* twp = reinterpret_cast<const float4*>(twTc + p * 16 * T + rp * T + l0);
#pragma unroll
                for (int h = 0; h < 8; ++h) {
                    const float4 w = __ldg(twp + h);
                    v[2 * h] = cmul<false>(v[2 * h], make_float2(w.x, w.y));
                    v[2 * h + 1] = cmul<false>(v[2 * h + 1], make_float2(w.z, w.w));
                }
                const int M0 = rl * T + l0;
                const int dt = M0 >> 7, dm = M0 & 127;
                const uint32_t off[4] = {mnmajor_chunk(dm, rp), mnmajor_chunk(dm + 8, rp),
                                         mnmajor_chunk(dm, 16 + rp), mnmajor_chunk(dm + 8, 16 + rp)};
                store_terms<SPLIT>(v, aBase, dt, off);
            } else {
                // last tensor-core pass: fp32 outputs to the staging buffer at their Stockham
                // positions (j - k) 16 + k + r ns of this transform row
                tc_fence_before_sync();
                __syncthreads();   // every thread's tcgen05.ld is done before the A tiles are reused
                float2* xr = stage + rl * S;
                const int base = (j - k) * 16 + k;
#pragma unroll
                for (int r = 0; r < 16; ++r) xr[spad(base + r * ns)] = v[r];
            }
        }
        if (failed) break;
        __syncthreads();
        if constexpr (RL == 1) {
            // natural order: coalesced stores of the whole group
#pragma unroll
            for (int s = 0; s < 16; ++s) {
                const int e = tid + s * kTcThreads;
                const int rr = e / N, i = e - rr * N;
                const uint64_t row = row0 + rr;
                if (row < batch) {
                    const float2 x = stage[rr * S + spad(i)];
                    st_stream(out + row * N + i, make_float2(x.x * scale, sgn * scale * x.y));
                }
            }
        } else {
            // final radix-RL pass in fp32 (Stockham, as fft_core.cuh): 16 / RL butterflies per thread
            constexpr int Ns = N / RL;
            const float2* twp = tw + Sd::twoff(Sd::P - 1);
            const float2* xr = stage + rl * S;
            const uint64_t row = row0 + rl;
#pragma unroll
            for (int sb = 0; sb < 16 / RL; ++sb) {
                const int jj = l + sb * T;
                const int k = jj & (Ns - 1);
                float2 w[RL];
#pragma unroll
                for (int r = 0; r < RL; ++r) w[r] = xr[spad(jj + r * (N / RL))];
#pragma unroll
                for (int r = 1; r < RL; ++r) w[r] = cmul<false>(w[r], __ldg(twp + (r - 1) * Ns + k));
                DFT<RL, false>::run(w);
                if (row < batch) {
#pragma unroll
                    for (int r = 0; r < RL; ++r)
                        st_stream(out + row * N + jj + r * (N / RL), make_float2(w[r].x * scale, sgn * scale * w[r].y));
                }
            }
        }
        // the staging buffer (the A tiles) is rewritten by the next group
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
constexpr int tcSmemBytes() {   // A tiles (the staging buffer aliases them), B terms, barrier + TMEM slot
    return SPLIT * 2 * kTileBytes + SPLIT * kBBytes + 16;
}
// Resident CTAs per SM: 256 threads at <= 85 registers and <= 72 KB of shared memory each fit
// three to an SM (TMEM: 3 x 64 of 512 columns).
constexpr int kTcCtasPerSm = 3;
static_assert(tcSmemBytes<4096, 3>() <= 72 * 1024, "three CTAs per SM");

}  // namespace dev

namespace backend {

template <int N, int SPLIT>
static int launchTc(const void* in, void* out, uint64_t batch, bool inverse, float scale, const void* tw,
                    const void* twTc, const void* table, void* stream) {
    constexpr int smem = dev::tcSmemBytes<N, SPLIT>();
    static std::atomic<int> residentOn[64];   // CTAs resident on each device (persistent grid)
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) return (int)cudaErrorInvalidDevice;
    int resident = residentOn[device].load();
    if (!resident) {
        int sms = 0;
        if (optInSharedMemory((const void*)dev::k_c2c_tc<N, SPLIT>, smem) ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
            return 1;
        resident = sms * dev::kTcCtasPerSm;
        residentOn[device].store(resident);
    }
    constexpr int rows = dev::kTcThreads / (N / 16);
    const uint64_t groups = (batch + rows - 1) / rows;
    const unsigned grid = (unsigned)(groups < (uint64_t)resident ? groups : (uint64_t)resident);
    dev::k_c2c_tc<N, SPLIT><<<grid, dev::kTcThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const float2*>(in), static_cast<float2*>(out), static_cast<const float2*>(tw),
        static_cast<const float2*>(twTc), static_cast<const unsigned char*>(table), batch, inverse ? 1 : -1, scale);
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

size_t tensorTwiddleCount(uint32_t n) {
    if (!hasTensorVariant(n, 3)) return 0;
    int pt = 0;
    for (uint32_t m = n; m >= 16; m /= 16) ++pt;
    return (size_t)(pt > 1 ? pt - 1 : 0) * 16 * (n / 16);
}

int buildTensorTwiddles(void* tw, uint32_t n, void* stream) {
    const size_t count = tensorTwiddleCount(n);
    if (!count) return 0;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const unsigned blocks = (unsigned)((count + 255) / 256);
    float2* t = static_cast<float2*>(tw);
    switch (n) {
        case 256: dev::k_tc_twiddles<256><<<blocks, 256, 0, st>>>(t); break;
        case 512: dev::k_tc_twiddles<512><<<blocks, 256, 0, st>>>(t); break;
        case 1024: dev::k_tc_twiddles<1024><<<blocks, 256, 0, st>>>(t); break;
        case 2048: dev::k_tc_twiddles<2048><<<blocks, 256, 0, st>>>(t); break;
        case 4096: dev::k_tc_twiddles<4096><<<blocks, 256, 0, st>>>(t); break;
        default: return (int)cudaErrorInvalidValue;
    }
    return (int)cudaGetLastError();
}

int launchC2CTensor(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale,
                    const void* tw, const void* twTc, const void* table, int split, void* stream) {
#define BFLY_TC(NN)                                                                                          \
    if (n == NN && split == 2) return launchTc<NN, 2>(in, out, batch, inverse, scale, tw, twTc, table, stream); \
    if (n == NN && split == 3) return launchTc<NN, 3>(in, out, batch, inverse, scale, tw, twTc, table, stream);
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
