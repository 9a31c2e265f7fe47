/* bench.h — indented phase timers (same prototypes as the reference's
 * include/bench.h:1-3 / util/bench.c). */
#ifndef BENCH_H
#define BENCH_H
#ifdef __cplusplus
extern "C" {
#endif
void task_start(int level, char *description);
void task_end(int level);
double wall_clock();
#ifdef __cplusplus
}
#endif
#endif
