/*
 * Force-included (-include) when compiling the reference's sources for the oracle.
 * calculateProcessGrid is called by src/Decompositions/pblasDecomposition.cpp:31 but
 * is declared and defined nowhere in the reference tree; the test double defines it
 * (fake_cuda.cpp) to return the process grid the caller requested.
 */
#ifndef ORACLE_SHIM_DECLS_H
#define ORACLE_SHIM_DECLS_H
void calculateProcessGrid(int* dRow, int* dCol, int size);
#endif
