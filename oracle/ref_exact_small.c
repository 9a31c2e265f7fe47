/* ref_exact_small.c — test infrastructure: routes the reference's small
 * products (bigfloat/mul.c:645-648, CL < 100) to its own schoolbook
 * _basecase_mul (bigfloat/mul.c:176-217) instead of _karatzuba_mul
 * (bigfloat/mul.c:367-553), which is inexact on some operands.  Linked into
 * oracle/_ref/exactsmall/libbcref.so next to a copy of the reference's mul.o
 * whose _karatzuba_mul is made weak, so this strong definition takes every
 * call.  Everything else is the reference's own code. */
#include <stddef.h>
#include <stdint.h>

void _basecase_mul(uint32_t *CT, size_t CL, uint32_t *AT, size_t AL, uint32_t *BT, size_t BL);

void _karatzuba_mul(uint32_t *CT, size_t CL, uint32_t *AT, size_t AL, uint32_t *BT, size_t BL) {
  _basecase_mul(CT, CL, AT, AL, BT, BL);
}
