/* main.c — command line: bluecrunch <digits> [--per-call | --levels]
 * Computes e to <digits> decimal digits into ./e.txt and ./e-hex.txt, like
 * the reference's main.c:169-219; products run on the GPU.  By default the
 * binary-splitting tree lives in device memory; --levels keeps the tree on
 * the host with each level's products in one GPU batch; --per-call uses the
 * reference's recursion with one GPU product per call. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bench.h"
#include "bigfloat.h"

int main(int argc, char *argv[]) {
  if (argc < 2) {
    printf("Usage %s <number of digits> [--per-call | --levels] - Computes Eulers constant\n", argv[0]);
    return 0;
  }
  size_t digits = strtoull(argv[1], NULL, 10);
  int mode = 2;
  for (int i = 2; i < argc; i++) {
    if (!strcmp(argv[i], "--per-call")) mode = 0;
    if (!strcmp(argv[i], "--levels")) mode = 1;
  }
  static const char *names[] = {"one product per call", "tree levels batched", "tree in device memory"};
  printf("Configuration:\n");
  printf("Digits:           %zu\n", digits);
  printf("Multiply:         B200 FP64 FFT (%s)\n", names[mode]);
  printf("Output File:      ./e.txt\n\n");
  task_start(0, "Starting calculation");
  int rc = bluecrunch_e(digits, mode, NULL);
  task_end(0);
  if (getenv("BC_STATS")) {
    bigfloat_mul_counters c;
    bigfloat_get_counters(&c);
    printf("GPU products: %zu in %zu calls, %.3f s inside GPU calls (%.3f s kernels of batches); "
           "host small products: %zu\n",
           c.gpu_products, c.gpu_calls, c.gpu_seconds, c.gpu_kernel_seconds, c.small_products);
  }
  return rc ? 1 : 0;
}
