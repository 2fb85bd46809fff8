/*
 * Placeholder for <metis.h>, which the reference's profiler includes
 * (test/runtime_analysis.c:15) without calling METIS itself: its only METIS user
 * is matrixReordering, which this library provides with a partitioner of its own
 * (declared in spike_pstrsv.h).  Nothing of METIS is declared here.
 */
#ifndef SPK_COMPAT_METIS_H
#define SPK_COMPAT_METIS_H
#endif
