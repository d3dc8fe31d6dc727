/* Test double: Open MPI extension header (the reference includes it for CUDA-aware probing). */
#ifndef ORACLE_FAKE_MPI_EXT_H
#define ORACLE_FAKE_MPI_EXT_H
#endif
