/*
 * Stand-in for the reference's src/misc.h for drivers built against this
 * library: the MatrixMarket reader and string helpers it declares
 * (matrixMarketToCSR, pathToMatrixName, strconcat) come from
 * libspike_pstrsv_b200.so and are declared in spike_pstrsv.h, which also
 * declares matrixReordering (the reference's profiler calls it without a
 * declaration in scope).
 */
#ifndef SPK_COMPAT_MISC_H
#define SPK_COMPAT_MISC_H
#include "mkl.h"
#include "spike_pstrsv.h"
#endif
