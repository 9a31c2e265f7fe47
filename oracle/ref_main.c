/* Entry point of the reference CLI build (oracle/_ref/{serial,omp}/bluecrunch_ref):
 * runs the reference main() (main.c:169-219, compiled as bcref_main) inside
 * one OpenMP parallel region when the OpenMP shim is on. */
int bcref_main(int argc, char *argv[]);

int main(int argc, char *argv[]) {
  int r = 0;
#ifdef BC_REF_OPENMP
#pragma omp parallel
#pragma omp single
#endif
  r = bcref_main(argc, argv);
  return r;
}
