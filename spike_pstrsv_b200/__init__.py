"""spike_pstrsv on NVIDIA B200 (sm_100a).

Host-side mirror of the reference's C API (src/spike_pstrsv.h:7-38) over the
C-ABI library ``libspike_pstrsv_b200.so`` built from ``csrc/``:
``spike_pstrsv_preproc``, ``spike_pstrsv_solve``, ``spike_pstrsv`` and the timed
``_`` variants, the reference's global flags and timers, and the handle-based
``System`` extension.  ``synth`` holds the seeded workload generators.
"""
from .capi import (  # noqa: F401
    SpkError,
    System,
    _spike_pstrsv_preproc,
    _spike_pstrsv_solve,
    free_PSTRSV3,
    get_flag,
    get_global,
    last_error,
    legacy_structure,
    lib,
    logPSTRSV3,
    reorder,
    reorder_plan,
    set_flag,
    set_partitions,
    spike_pstrsv,
    spike_pstrsv_preproc,
    spike_pstrsv_solve,
)
from . import synth  # noqa: F401
