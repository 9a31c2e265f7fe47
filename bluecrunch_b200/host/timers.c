/* timers.c — indented phase timers printed to stdout (same behaviour as the
 * reference's util/bench.c:11-41). */
#include <stdio.h>
#include <time.h>

#include "bench.h"

double wall_clock() {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1.0e-9 * t.tv_nsec;
}

#define MAX_LEVELS 4
static int last_level = 0;
static double started[MAX_LEVELS];

void task_start(int level, char *description) {
  if (last_level == level - 1) printf("\n");
  printf("%*s%s...", 2 * level, "", description);
  fflush(stdout);
  started[level] = wall_clock();
  last_level = level;
}

void task_end(int level) {
  double t = wall_clock();
  if (last_level != level) printf("%*sDone [%f seconds]\n", 2 * level, "", t - started[level]);
  else printf(" done [%f seconds]\n", t - started[level]);
  started[level] = 0;
}
