/*
 * coo2csr_f90abi.c -- the Fortran-ABI entry point of
 * sparse_matrix/coo2csr_lib.f90:6-41 (module coo2csr_lib, subroutine
 * coo2csr_canonical), restated in C because this image has no Fortran
 * compiler.  Linked only into the reference build (oracle/_ref).
 *
 * TEST INFRASTRUCTURE ONLY.
 *
 * Replays the reference's observable side effects: all arguments by
 * pointer; Bp/Bj/Bx zero-filled over their full extent first (:24-26); the
 * caller's Ai/Aj arrays are left incremented by one (:27-28); the output is
 * 0-based (:36-37).
 */
#include "sfo.h"

void __coo2csr_lib_MOD_coo2csr_canonical(int *nnz, int *Bp_size, int *csr_size, int *Ai, int *Aj,
                                         double *Ax, int *Bp, int *Bj, double *Bx)
{
    int n = *nnz, ps = *Bp_size;
    for (int i = 0; i < ps; i++) Bp[i] = 0;
    for (int i = 0; i < n; i++) { Bj[i] = 0; Bx[i] = 0.0; }
    *csr_size = sfo_coo2csr_canonical(n, ps, Ai, Aj, Ax, Bp, Bj, Bx);
    for (int i = 0; i < n; i++) { Ai[i] += 1; Aj[i] += 1; }
}
