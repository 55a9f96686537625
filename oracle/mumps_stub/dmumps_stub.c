/* Oracle-only MUMPS stand-in: JOB_INIT (-1) and JOB_END (-2) succeed, any
 * other job aborts because the sparse Schur path is never exercised by the
 * oracle (see dmumps_c.h in this directory). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "dmumps_c.h"

void dmumps_c(DMUMPS_STRUC_C* id)
{
  if (id->job == -1 || id->job == -2) {
    memset(id->infog, 0, sizeof(id->infog));
    memset(id->rinfog, 0, sizeof(id->rinfog));
    return;
  }
  fprintf(stderr, "oracle MUMPS stub: job %d requested (sparse Schur path is not built)\n",
          id->job);
  abort();
}
