/*
 * Stand-in for the reference's src/spike_pstrsv_globals.h for drivers built
 * against this library.  The flags, partition bounds and phase timers it
 * declares are exported by libspike_pstrsv_b200.so and declared in
 * spike_pstrsv.h (the partition and per-thread timer arrays hold
 * SPK_MAX_EXPORTED_PARTS entries); the reference's pools (D, T2, S, ...) live on
 * the GPU and are read through spk_debug_array instead.  The constants keep the
 * reference's values (src/spike_pstrsv_globals.h:4-9) except MAXTHREADCOUNT,
 * which is the exported arrays' length.
 */
#ifndef SPK_COMPAT_GLOBALS_H
#define SPK_COMPAT_GLOBALS_H
#include "mkl.h"
#include "spike_pstrsv.h"
#define MAXSIZE 4194304
#define MAXNNZS 25165824
#define MAXTHREADCOUNT SPK_MAX_EXPORTED_PARTS
#define INF 2147483640
#define MEMSIZE 17179869184
#ifndef max
#define max(a, b) (((a) > (b)) ? (a) : (b))
#endif
#endif
