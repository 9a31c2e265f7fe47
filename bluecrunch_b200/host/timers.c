/* timers.c — nested phase timers on stdout.
 *
 * The printed format is the interface of the reference's include/bench.h
 * (prototypes kept): a phase prints "<indent><name>..." when it opens; if
 * no inner phase opened meanwhile it closes on the same line with
 * " done [<s> seconds]", otherwise its line was already ended by the first
 * inner phase and it closes with "<indent>Done [<s> seconds]" on a line of
 * its own.  Indentation is two spaces per level.
 *
 * Implementation: a stack of the phases that are open.  Each entry knows
 * whether its "..." line is still waiting for its closing text; opening a
 * phase below one whose line is still open ends that line first.
 */
#include <stdio.h>
#include <time.h>

#include "bench.h"

double wall_clock() {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1.0e-9 * t.tv_nsec;
}

typedef struct {
  int level;       /* indentation level the caller gave */
  int line_open;   /* 1 while "name..." awaits " done" on the same line */
  double t0;       /* wall_clock() at open */
} phase_t;

enum { PHASE_DEPTH = 16 };
static phase_t phases[PHASE_DEPTH];
static int depth = 0; /* entries in use */

void task_start(int level, char *description) {
  if (depth > 0 && phases[depth - 1].line_open && phases[depth - 1].level < level) {
    putchar('\n');
    phases[depth - 1].line_open = 0;
  }
  printf("%*s%s...", 2 * level, "", description);
  fflush(stdout);
  if (depth < PHASE_DEPTH) {
    phases[depth].level = level;
    phases[depth].line_open = 1;
    phases[depth].t0 = wall_clock();
    depth++;
  }
}

void task_end(int level) {
  const double now = wall_clock();
  /* close the innermost open phase of this level (inner ones left open by
   * the caller are dropped with it) */
  int i = depth - 1;
  while (i >= 0 && phases[i].level != level) i--;
  if (i < 0) return;
  const double secs = now - phases[i].t0;
  if (phases[i].line_open && i == depth - 1) printf(" done [%f seconds]\n", secs);
  else printf("%*sDone [%f seconds]\n", 2 * level, "", secs);
  fflush(stdout);
  depth = i;
}
