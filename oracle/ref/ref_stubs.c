/* Tag-server stand-in for the oracle build of the reference code (one rank:
 * any tag is unique).  The parallel file IO itself (simUtil/src/pio.c) is
 * compiled from the reference.  Test infrastructure. */
#include <stddef.h>
#include <mpi.h>
int getUniqueTag(MPI_Comm c) { (void)c; return 1; }
