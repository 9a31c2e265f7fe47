// Host-side check of the device carry helpers (bc_device.cuh / bc_kernels.cuh):
// compiled by tests/test_carry_logic.py with nvcc and run on the CPU.  Reads
// cases from stdin and prints results for comparison with Python integers.
#include <cstdio>
#include <cstdlib>
#include "bc_kernels.cuh"
using namespace bc;
int main() {
  char op[16];
  while (scanf("%15s", op) == 1) {
    if (op[0] == 'A') {  // A nbits h0 h1 h2 v  -> H+v mod 2^nbits, carry
      int nbits; unsigned long long h0, h1, h2; long long v;
      if (scanf("%d %llx %llx %llx %lld", &nbits, &h0, &h1, &h2, &v) != 5) return 1;
      U192 h = {{h0, h1, h2}};
      int c = u192_add_s64(h, v, nbits);
      printf("%d %llx %llx %llx %d %d\n", c, h.w[0], h.w[1], h.w[2], (int)u192_is_zero(h), (int)u192_is_ones(h, nbits));
    } else if (op[0] == 'R') {  // R b c0..c7 -> run record
      int b; double c[8];
      if (scanf("%d", &b) != 1) return 1;
      for (int u = 0; u < 8; u++) { long long x; if (scanf("%lld", &x) != 1) return 1; c[u] = (double)x; }
      RunRec r = make_run(c, b);
      printf("%llx %llx %llx %lld\n", r.h0, r.h1, r.h2, r.c);
    } else if (op[0] == 'W') {  // W h0 h1 h2 off -> 32 bits at off
      unsigned long long h0, h1, h2; int off;
      if (scanf("%llx %llx %llx %d", &h0, &h1, &h2, &off) != 4) return 1;
      U192 h = {{h0, h1, h2}};
      printf("%x\n", u192_bits32(h, off));
    }
  }
  return 0;
}
