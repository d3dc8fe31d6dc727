/*
 * Test double for the reference's include/cmatrix.h: same declarations the hot-path
 * files use, without the cuRAND device headers (the oracle seeds matrices itself).
 */
#ifndef CMATRIX_H
#define CMATRIX_H
#include <cstdio>
#include <iostream>
#include <string>
#include <cstring>
#include <algorithm>
#include <cuda_runtime.h>
#include "errorHandling.hpp"
#include "generalUtilities.hpp"

template <typename T>
void MatrixInit(T* matrix, const long long rows, const long long columns, int loc);
template <typename T>
void MatrixInit(T* matrix, const long long size, int loc);
#endif
