/* Parallel-file-IO and tag-server stand-ins for the oracle build of the
 * reference code.  Only PerformanceTimers references them, to write timing
 * reports; the oracle never asks for those reports.  Test infrastructure. */
#include <stddef.h>
#include <mpi.h>
typedef struct oracle_pfile PFILE;
PFILE* Popen(const char* f, const char* m, MPI_Comm c) { (void)f; (void)m; (void)c; return 0; }
int Pclose(PFILE* f) { (void)f; return 0; }
int Pprintf(PFILE* f, const char* fmt, ...) { (void)f; (void)fmt; return 0; }
size_t Pwrite(const void* p, size_t s, size_t n, PFILE* f) { (void)p; (void)s; (void)f; return n; }
int getUniqueTag(MPI_Comm c) { (void)c; return 1; }
