// Overlap-add side of the one-kernel inverse STFT (k_istft in k_stft.cu for powers of two,
// k_istft_mixed in k_mixed.cu for other even lengths).
//   y[p] = sum_f w[j] x_f[j] / sum_f w[j]^2,  j = p - f*hop in [0, N);  out[s][i] = y[i + start],
//   i < outLen, zero past the last frame.
// CTA (s, c) owns padded samples [c*Q*hop, (c+1)*Q*hop) of signal s (the last CTA of a signal
// also the tail) and transforms frames c*Q - (K-1) .. (c+1)*Q - 1 (K = ceil(N/hop) frames cover a
// sample) in waves.  After a wave's frames sit in shared memory, wave() sums, per sample of the
// wave's span, the carried partial sum of earlier frames and the wave's frames covering it
// (frames in increasing order, so results are deterministic); samples no later frame touches are
// stored times 1 / envelope (a per-CTA table over p mod hop, exact sums within a frame of either
// end), the rest (N - hop samples) are carried to the next wave in the other half of a
// ping-pong buffer.  VEC = 4 sums four consecutive samples per thread with float4 shared and
// global accesses (N, hop, the output length and the frame buffers multiples of 4 / 16 bytes).
//
// ADJ: the same sums without the envelope, as the adjoint of an STFT (its gradient with
// respect to the signal, start = the centring pad).  A centred STFT read reflected samples
// x[-i] = x[i] and x[L-1+i] = x[L-1-i]: the sums at padded positions before `start` and after
// the signal fold onto outputs [1, pad] and [L-1-pad, L-2].  Those outputs collect their
// direct and folded terms in shared fold buffers (shared-memory atomic adds; each gets exactly
// two terms onto zero, so the sum does not depend on their order) and are stored at the end by
// the first and the last segment of the signal, which the launch makes span more than N
// samples so that they own both terms.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace bfly {
namespace dev {

struct IstftSegment {
    int N, K, CARRY, CTA;
    uint32_t hop, frames, fA, fB;
    int64_t padded, start, end, P0, P1;
    uint64_t outLen;
    const float* window;
    float* dst;
    float *cur, *nxt, *rinv;
    int pad = 0;                                  // ADJ: fold width (0: no reflect padding)
    float *foldL = nullptr, *foldR = nullptr;     // ADJ: outputs [0, pad] and [L-1-pad, L-1)

    // `scratch`: 2 (N - hop) + hop floats of shared memory (carry pair, then the envelope table).
    __device__ __forceinline__ void init(int n, uint32_t hop_, uint32_t frames_, uint32_t Q, uint32_t segs, int64_t start_,
                                         uint64_t outLen_, const float* window_, float* out, float* scratch) {
        N = n;
        hop = hop_;
        frames = frames_;
        CTA = blockDim.x;
        const uint32_t s = blockIdx.x / segs;
        const uint32_t c = blockIdx.x - s * segs;
        K = (N + (int)hop - 1) / (int)hop;
        CARRY = N - (int)hop;
        padded = (int64_t)N + (int64_t)hop * (frames - 1);
        const uint64_t first = (uint64_t)c * Q;
        fA = first >= (uint64_t)(K - 1) ? (uint32_t)(first - (K - 1)) : 0u;
        fB = (uint32_t)min((uint64_t)frames, first + Q);
        start = start_;
        outLen = outLen_;
        P0 = (int64_t)first * hop;
        end = start + (int64_t)outLen;
        if (c + 1 == segs) fB = frames;   // a last segment may be longer than Q (ADJ launches)
        P1 = c + 1 == segs ? (padded > end ? padded : end) : (int64_t)fB * hop;
        window = window_;
        dst = out + (uint64_t)s * outLen;
        cur = scratch;
        nxt = cur + CARRY;
        rinv = nxt + CARRY;
        for (int q = threadIdx.x; q < CARRY; q += CTA) cur[q] = 0.f;
        // 1 / (overlap-added squared window) of samples every frame slot of which exists
        // (N-1 <= p < frames*hop): periodic in p with period hop
        for (int r = threadIdx.x; r < (int)hop; r += CTA) {
            float e = 0.f;
            for (int j = r; j < N; j += (int)hop) {
                const float w = window ? __ldg(window + j) : 1.f;
                e += w * w;
            }
            rinv[r] = e > 0.f ? 1.f / e : 0.f;
        }
    }

    // ADJ set-up: fold buffers of 2 (pad + 1) floats at `scratch`, zeroed (pad = 0: none).
    __device__ __forceinline__ void initFold(int pad_, float* scratch) {
        pad = pad_;
        if (!pad) return;
        foldL = scratch;
        foldR = scratch + pad + 1;
        for (int q = threadIdx.x; q < 2 * (pad + 1); q += CTA) scratch[q] = 0.f;
    }

    // ADJ: one completed sum at padded position P (this segment's [P0, P1)).
    __device__ __forceinline__ void emitAdj(int64_t P, float val) {
        const int64_t L = (int64_t)outLen;
        int64_t t = P - start;   // output of the direct term
        if (pad) {
            if (t < 0) {                       // left padding: the mirror of output -t
                atomicAdd(foldL - t, val);
                return;
            }
            if (t >= L) {                      // right padding: the mirror of output 2 (L-1) - t
                atomicAdd(foldR + (2 * (L - 1) - t) - (L - 1 - pad), val);
                return;
            }
            if (t <= pad) {
                atomicAdd(foldL + t, val);
                return;
            }
            if (t >= L - 1 - pad && t < L - 1) {
                atomicAdd(foldR + (t - (L - 1 - pad)), val);
                return;
            }
        }
        if (t >= 0 && t < L) __stcs(dst + t, val);
    }

    // ADJ: store the fold outputs (after the last wave and zeroTail).
    __device__ __forceinline__ void finishFold(uint32_t segs) {
        if (!pad) return;
        __syncthreads();
        const int64_t L = (int64_t)outLen;
        const uint32_t c = blockIdx.x % segs;
        if (c == 0)
            for (int u = threadIdx.x; u <= pad; u += CTA) __stcs(dst + u, foldL[u]);
        if (c + 1 == segs)
            for (int u = threadIdx.x; u < pad; u += CTA) __stcs(dst + (L - 1 - pad) + u, foldR[u]);
    }

    // Samples near either end: the envelope of the frames that exist.
    __device__ __forceinline__ float edgeInv(int64_t p) const {
        float e = 0.f;
        const int64_t fh = p / hop;
        for (int64_t f = fh - K + 1 > 0 ? fh - K + 1 : 0; f <= fh && f < (int64_t)frames; ++f) {
            const int64_t j = p - f * hop;
            if (j < N) {
                const float w = window ? __ldg(window + j) : 1.f;
                e += w * w;
            }
        }
        return e > 0.f ? 1.f / e : 0.f;
    }

    // Overlap-add of the wave of frames f0 .. f0+R-1 held in shared memory: ld1(r, j) returns
    // w[j] x_(f0+r)[j], ld4(r, j) the float4 of samples j .. j+3 (j a multiple of 4).  Called by
    // every thread after a barrier that follows the frames' writes; swaps the carry halves.
    // CTA_C: the block size when known at compile time (0: blockDim.x).
    template <int VEC, int CTA_C, bool ADJ = false, class Ld1, class Ld4>
    __device__ __forceinline__ void wave(uint32_t f0, int R, Ld1&& ld1, Ld4&& ld4) {
        const int cta = CTA_C > 0 ? CTA_C : CTA;
        auto clampq = [](int64_t v, int hi) { return (int)(v < 0 ? 0 : (v > hi ? hi : v)); };
        const bool tail = f0 + R == frames;   // no later frame: every sample of the span is complete
        const int span = (R - 1) * (int)hop + N;
        const int done = tail ? span : R * (int)hop;
        const int64_t base = (int64_t)f0 * hop;
        // span offsets q this CTA stores ([wlo, whi)) and those with the periodic envelope; the
        // adjoint also emits the padding sums of its segment (folded onto the signal)
        const int wlo = clampq((ADJ ? P0 : (P0 > start ? P0 : start)) - base, done);
        const int whi = clampq((ADJ ? P1 : (P1 < end ? P1 : end)) - base, done);
        const int elo = clampq((int64_t)(N - 1) - base, span);
        const int ehi = clampq((int64_t)frames * hop - base, span);
        float* dq = dst + (base - start);   // output of span offset q at dq[q] (wlo <= q < whi)
        // each thread sums VEC consecutive samples: q += VEC*CTA, tracked as (q / hop, q % hop)
        const int stepH = VEC * cta / (int)hop, stepR = VEC * cta - stepH * (int)hop;
        int qh = VEC * (int)threadIdx.x / (int)hop;
        int qr = VEC * (int)threadIdx.x - qh * (int)hop;
        for (int q = VEC * threadIdx.x; q < span; q += VEC * cta) {
            const int rlo = qh - K + 1 > 0 ? qh - K + 1 : 0;
            const int rhi = qh < R - 1 ? qh : R - 1;
            if constexpr (VEC == 1) {
                float val = q < CARRY ? cur[q] : 0.f;
                for (int r = rlo; r <= rhi; ++r) {
                    const int j = qr + (qh - r) * (int)hop;
                    if (j < N) val += ld1(r, j);
                }
                if (q >= done) {
                    nxt[q - done] = val;
                } else if (q >= wlo && q < whi) {
                    if constexpr (ADJ) emitAdj(base + q, val);
                    else __stcs(dq + q, val * (q >= elo && q < ehi ? rinv[qr] : edgeInv(base + q)));
                }
            } else {
                float4 val = q < CARRY ? *reinterpret_cast<const float4*>(cur + q) : make_float4(0.f, 0.f, 0.f, 0.f);
                for (int r = rlo; r <= rhi; ++r) {
                    const int j = qr + (qh - r) * (int)hop;
                    if (j < N) {
                        const float4 x = ld4(r, j);
                        val.x += x.x;
                        val.y += x.y;
                        val.z += x.z;
                        val.w += x.w;
                    }
                }
                if (q >= done) {
                    *reinterpret_cast<float4*>(nxt + q - done) = val;
                } else if (ADJ && q >= wlo && q < whi) {
                    const int64_t t = base + q - start;
                    if (t >= pad + 1 && t + 3 < (int64_t)outLen - 1 - pad && q + 3 < whi) {
                        __stcs(reinterpret_cast<float4*>(dq + q), val);
                    } else {
                        const float vs[4] = {val.x, val.y, val.z, val.w};
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            if (q + u < whi) emitAdj(base + q + u, vs[u]);
                    }
                } else if (q >= wlo && q < whi) {
                    float4 e;
                    if (q >= elo && q + 3 < ehi) {
                        e = *reinterpret_cast<const float4*>(rinv + qr);
                    } else {
                        auto inv = [&](int u) { return q + u >= elo && q + u < ehi ? rinv[qr + u] : edgeInv(base + q + u); };
                        e = make_float4(inv(0), inv(1), inv(2), inv(3));
                    }
                    __stcs(reinterpret_cast<float4*>(dq + q), make_float4(val.x * e.x, val.y * e.y, val.z * e.z, val.w * e.w));
                }
            }
            qh += stepH;
            qr += stepR;
            if (qr >= (int)hop) {
                qr -= (int)hop;
                ++qh;
            }
        }
        float* sw = cur;
        cur = nxt;
        nxt = sw;
    }

    // Samples past the last frame up to outLen are zero (only the signal's last segment).
    __device__ __forceinline__ void zeroTail(uint32_t segs) {
        if (blockIdx.x % segs + 1 != segs) return;
        for (int64_t p = (padded > P0 ? padded : P0) + threadIdx.x; p < P1; p += CTA) {
            const int64_t i = p - start;
            if (i >= 0 && i < (int64_t)outLen) __stcs(dst + i, 0.f);
        }
    }
};

}  // namespace dev
}  // namespace bfly
