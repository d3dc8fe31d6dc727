/* Test double: the CBLAS enums the reference's headers name (no CBLAS routine is called). */
#ifndef ORACLE_FAKE_CBLAS_H
#define ORACLE_FAKE_CBLAS_H
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef CBLAS_LAYOUT CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
#endif
