/* Test-infrastructure stand-in for the file the reference's CMake generates
 * from cmake/config.h.cmake: RELEASE build, BLAS/LAPACK symbols with a
 * trailing underscore (the OpenBLAS convention), restrict spelled for g++. */
#pragma once
#define HIFDE3D_VERSION_MAJOR 0
#define HIFDE3D_VERSION_MINOR 2
#define RELEASE
#define BLAS_POST
#define LAPACK_POST
#define RESTRICT __restrict__
