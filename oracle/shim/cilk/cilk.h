/* Stand-in for <cilk/cilk.h> so the reference C sources compile with gcc 13,
 * which dropped Cilk Plus.  Test infrastructure for the oracle build only.
 *
 * Default: the three keywords disappear and every spawn runs inline (serial).
 * With -DBC_REF_OPENMP (and -fopenmp) a spawn becomes an OpenMP task, a sync a
 * taskwait and cilk_for a taskloop, all with shared data so that spawned calls
 * write into the caller's bigfloat_t objects as they do under Cilk. */
#ifndef BC_REF_CILK_SHIM_H
#define BC_REF_CILK_SHIM_H
#ifdef BC_REF_OPENMP
#define cilk_spawn _Pragma("omp task default(shared)")
#define cilk_sync  _Pragma("omp taskwait")
#define cilk_for   _Pragma("omp taskloop default(shared)") for
#else
#define cilk_spawn
#define cilk_sync
#define cilk_for for
#endif
#endif
