/* Stand-in for <cilk/cilk_api.h> (oracle build only): worker-count queries. */
#ifndef BC_REF_CILK_API_SHIM_H
#define BC_REF_CILK_API_SHIM_H
int __cilkrts_get_nworkers(void);
int __cilkrts_set_param(const char *name, const char *value);
#endif
