/*
 * Stand-in for METIS's <metis.h>, used ONLY to compile the reference's
 * matrix_reordering.c into the CPU checker library (test infrastructure).
 * METIS is not installed here.  The declarations follow METIS 5's public API
 * (the names the reference calls, src/matrix_reordering.c:125-141).
 * METIS_PartGraphKway does not partition: it returns the partition vector a
 * test injected with spk_ref_set_partition (ref/fixups.c), so the reference's
 * steps after the partitioner can be compared with the GPU library's for the
 * same partition.
 */
#ifndef SPK_METIS_SHIM_H
#define SPK_METIS_SHIM_H

typedef int idx_t;
typedef float real_t;

#define METIS_NOPTIONS 40
enum { METIS_OK = 1, METIS_ERROR_INPUT = -2, METIS_ERROR = -4 };
enum { METIS_PTYPE_RB = 0, METIS_PTYPE_KWAY = 1 };
enum { METIS_OBJTYPE_CUT = 0, METIS_OBJTYPE_VOL = 1 };
enum {
    METIS_OPTION_PTYPE = 0, METIS_OPTION_OBJTYPE, METIS_OPTION_CTYPE, METIS_OPTION_IPTYPE,
    METIS_OPTION_RTYPE, METIS_OPTION_DBGLVL, METIS_OPTION_NITER, METIS_OPTION_NCUTS,
    METIS_OPTION_SEED, METIS_OPTION_NO2HOP, METIS_OPTION_MINCONN, METIS_OPTION_CONTIG,
    METIS_OPTION_COMPRESS, METIS_OPTION_CCORDER, METIS_OPTION_PFACTOR, METIS_OPTION_NSEPS,
    METIS_OPTION_UFACTOR, METIS_OPTION_NUMBERING
};

int METIS_SetDefaultOptions(idx_t *options);
int METIS_PartGraphKway(idx_t *nvtxs, idx_t *ncon, idx_t *xadj, idx_t *adjncy, idx_t *vwgt, idx_t *vsize,
                        idx_t *adjwgt, idx_t *nparts, real_t *tpwgts, real_t *ubvec, idx_t *options,
                        idx_t *objval, idx_t *part);

/* Test hook: the partition METIS_PartGraphKway returns next (n entries). */
void spk_ref_set_partition(const int *part, int n);

#endif
