/*
 * Force-included (gcc -include) in front of every reference source file when
 * the reference is compiled into the CPU checker library oracle/_ref/.
 * Test infrastructure only.
 *
 * The reference fixes its pool sizes at compile time
 * (src/spike_pstrsv_globals.h:4-6: MAXSIZE 4,194,304 rows, MAXNNZS
 * 25,165,824 nonzeros, MAXTHREADCOUNT 128).  The large banded workload
 * (m = 4,194,304, nnz = 71,303,032, up to 1024 partitions) exceeds all three,
 * and ID[] needs 2m+1 entries (src/spike_pstrsv_ops.c:43 with
 * src/spike_pstrsv_ops.c:823).  Instead of editing the sources, this prelude
 * defines the header's include guard first, so the reference header is
 * skipped and the declarations below (the same names and types as
 * src/spike_pstrsv_globals.h:13-79) apply with larger limits.
 */
#ifndef SPK_REF_PRELUDE_H
#define SPK_REF_PRELUDE_H

#include "mkl.h"

#define SPIKE_PSTRSV_GLOBALS_H

#ifndef SPK_REF_MAXSIZE
#define SPK_REF_MAXSIZE 4194368
#endif
#ifndef SPK_REF_MAXNNZS
#define SPK_REF_MAXNNZS 72000000
#endif
#ifndef SPK_REF_MAXTHREADS
#define SPK_REF_MAXTHREADS 4096
#endif

#define MAXSIZE SPK_REF_MAXSIZE
#define MAXNNZS SPK_REF_MAXNNZS
#define MAXTHREADCOUNT SPK_REF_MAXTHREADS
#define INF 2147483640
#define MEMSIZE 17179869184
#define max(a, b) (((a) > (b)) ? (a) : (b))

extern MKL_INT partition_numRows[MAXTHREADCOUNT];
extern MKL_INT partition_starts[MAXTHREADCOUNT];
extern MKL_INT partition_ends[MAXTHREADCOUNT];
extern double D[MAXNNZS * 2];
extern MKL_INT ID[MAXSIZE * 2];
extern MKL_INT JD[MAXNNZS * 2];
extern MKL_INT dependents[MAXSIZE];
extern double T[MAXNNZS];
extern MKL_INT IT[MAXSIZE];
extern MKL_INT JT[MAXNNZS];
extern double T2[3 * MAXNNZS];
extern MKL_INT IT2[3 * MAXSIZE];
extern MKL_INT JT2[3 * MAXNNZS];
extern MKL_INT starts_D[MAXTHREADCOUNT];
extern MKL_INT ends_D[MAXTHREADCOUNT];
extern MKL_INT starts_R[MAXTHREADCOUNT];
extern MKL_INT ends_R[MAXTHREADCOUNT];
extern char isReducedSystemNecessary;
extern char hasDependences[MAXTHREADCOUNT];
extern char hasReflections[MAXTHREADCOUNT];
extern double *S;
extern MKL_INT numRows_S[MAXTHREADCOUNT];
extern MKL_INT numCols_S[MAXTHREADCOUNT];
extern long long starts_S[MAXTHREADCOUNT];
extern long long ends_S[MAXTHREADCOUNT];
extern MKL_INT starts_D0[MAXTHREADCOUNT];
extern MKL_INT ends_D0[MAXTHREADCOUNT];
extern MKL_INT starts_D1[MAXTHREADCOUNT];
extern MKL_INT ends_D1[MAXTHREADCOUNT];
extern MKL_INT starts_D2[MAXTHREADCOUNT];
extern MKL_INT ends_D2[MAXTHREADCOUNT];
extern double *compressedX;
extern MKL_INT *mapR;
extern MKL_INT starts_mapR[MAXTHREADCOUNT];
extern MKL_INT ends_mapR[MAXTHREADCOUNT];
extern double reducedX[MAXSIZE];
extern MKL_INT numRowsReducedSystem;
extern MKL_INT start_intervals[MAXTHREADCOUNT];
extern MKL_INT end_intervals[MAXTHREADCOUNT];
extern char isOptimizeds[MAXTHREADCOUNT];
extern char PSTRSV_VERBOSE;
extern char FORCE_LOAD_BALANCE;
extern char IS_MATRIX_PARTITIONED;

extern double memoryAlloc_timer_pstrsv3;
extern double preprocessD_timer_pstrsv3;
extern double preprocessR_timer_pstrsv3;
extern double setDependents_timer_pstrsv3;
extern double preprocessS_timer_pstrsv3;
extern double preprocessMappings_timer_pstrsv3;
extern double produceCompressedR_timer_pstrsv3;
extern double produceS_timer_pstrsv3;
extern double produceReducedSystem_timer_pstrsv3;
extern double init_vars_pstrsv3;
extern double reduced_solver_timer_pstrsv3;
extern double temp_timer[MAXTHREADCOUNT];
extern double waitBefore_timer_pstrsv3[MAXTHREADCOUNT];
extern double computeY_timer[MAXTHREADCOUNT];
extern double solveIndependent_timer[MAXTHREADCOUNT];
extern double subtract_Rx_timer[MAXTHREADCOUNT];
extern double waitAfter_timer_pstrsv3[MAXTHREADCOUNT];
extern double solveD2_timer[MAXTHREADCOUNT];
extern double solveD_timer[MAXTHREADCOUNT];

#endif
