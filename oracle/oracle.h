/* Test infrastructure only: C restatements of the reference's CPU oracle and of the fp32
 * arithmetic of its device kernels (TruNcat3/ascend-fft).  Built into _build/liboracle.so by
 * oracle/Makefile; called from tests/ through ctypes. */
#ifndef BFLY_ORACLE_H
#define BFLY_ORACLE_H
#include <stddef.h>
#include <stdint.h>

/* ref_fft.c: FP64 radix-2 DIT, outputs rounded to fp32 (src/framework/reference.cpp:14-79) */
void orc_ref_fft(const float* in, float* out, uint32_t n);
void orc_ref_r2c(const float* in, float* out, uint32_t n);
void orc_ref_c2r(const float* in, float* out, uint32_t n);
double orc_max_rel_scaled(const float* got, const float* ref, size_t len);
float orc_pattern_at(size_t i);

/* kfft_fp32.c: fp32 arithmetic of kfft_fwd / kfft_r2c_post / kfft_c2r_prep+post */
uint32_t orc_plane_k(uint32_t n);
void orc_kfft_fwd(const float* in, float* out, uint32_t n, int sign);   /* sign -1 / +1 */
void orc_kfft_r2c(const float* in, float* out, uint32_t n);             /* [n] -> [n+2] */
void orc_kfft_c2r(const float* in, float* out, uint32_t n);             /* [n+2] -> [n] */

#endif
