/* Minimal stand-in for the MUMPS C interface header, written for the oracle
 * build only (test infrastructure, never shipped).
 *
 * The reference solver includes <dmumps_c.h> from sdpa_chordal.h and keeps a
 * DMUMPS_STRUC_C inside class Chordal.  On the dense Schur-complement path
 * (every instance this project checks) the only MUMPS calls are JOB_INIT and
 * JOB_END (sdpa_chordal.cpp:84-101, :106-112), so this header declares just
 * the fields that sdpa_chordal.cpp touches and a dmumps_c() that accepts
 * those two jobs and aborts on any other (the sparse Schur path is out of
 * scope).  MUMPS 5.7.3 itself is absent from the reference tree. */
#ifndef ORACLE_DMUMPS_C_STUB_H
#define ORACLE_DMUMPS_C_STUB_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int job;
  int comm_fortran;
  int par;
  int sym;
  int icntl[60];
  int infog[80];
  double rinfog[40];
  int n;
  int nz;
  int* irn;
  int* jcn;
  double* a;
  double* rhs;
  char write_problem[256];
} DMUMPS_STRUC_C;

void dmumps_c(DMUMPS_STRUC_C* id);

#ifdef __cplusplus
}
#endif

#endif
