/* mul.h — multiply kernels behind bigfloat_mul; same prototypes as the
 * reference's include/mul.h:1-3.
 *
 * _fft_mul (reference bigfloat/mul.c:108-174): CT[0..CL) = AT*BT mod
 * 2^(32*CL); CT may alias AT or BT.  Here it runs on the GPU through
 * bc_gpu_mul (include/bc_gpu.h) and returns the digit width used.  As in the
 * reference it has no status return: a GPU failure prints the reason and
 * aborts (the reference aborts on unsupported widths, fft/convert.c:66-68).
 * _basecase_mul / _karatzuba_mul are the host small-product paths the
 * reference dispatches to below 100 output limbs (bigfloat/mul.c:640-648);
 * both are the same exact schoolbook product here. */
#ifndef MUL_H
#define MUL_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

void _basecase_mul(uint32_t *CT, size_t CL, uint32_t *AT, size_t AL, uint32_t *BT, size_t BL);
void _karatzuba_mul(uint32_t *CT, size_t CL, uint32_t *AT, size_t AL, uint32_t *BT, size_t BL);
int _fft_mul(uint32_t *CT, size_t CL, uint32_t *AT, size_t AL, uint32_t *BT, size_t BL);

#ifdef __cplusplus
}
#endif
#endif
