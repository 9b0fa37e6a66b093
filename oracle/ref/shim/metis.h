/*
 * Stand-in for the METIS 5.1.0 API subset the reference calls (src/partition/graph_partitioner.cpp:
 * METIS_SetDefaultOptions, METIS_PartGraphKway).  TEST INFRASTRUCTURE ONLY: METIS is not installed
 * here.  The partition comes from the binary int32 file named by $S2L_PART_FILE (the setup phase's
 * partition, so both sides decompose identically); without it, a deterministic recursive bisection
 * of breadth-first orders is used.
 */
#ifndef S2L_METIS_STANDIN_H
#define S2L_METIS_STANDIN_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef int32_t idx_t;
typedef float real_t;
#define METIS_NOPTIONS 40
enum { METIS_OK = 1, METIS_ERROR_INPUT = -2, METIS_ERROR = -4 };
enum { METIS_OPTION_PTYPE = 0, METIS_OPTION_OBJTYPE, METIS_OPTION_CTYPE, METIS_OPTION_IPTYPE, METIS_OPTION_RTYPE,
       METIS_OPTION_DBGLVL, METIS_OPTION_NITER, METIS_OPTION_NCUTS, METIS_OPTION_SEED, METIS_OPTION_NO2HOP,
       METIS_OPTION_MINCONN, METIS_OPTION_CONTIG, METIS_OPTION_COMPRESS, METIS_OPTION_CCORDER, METIS_OPTION_PFACTOR,
       METIS_OPTION_NSEPS, METIS_OPTION_UFACTOR, METIS_OPTION_NUMBERING };
enum { METIS_OBJTYPE_CUT = 0, METIS_OBJTYPE_VOL = 1, METIS_OBJTYPE_NODE = 2 };
int METIS_SetDefaultOptions(idx_t* options);
int METIS_PartGraphKway(idx_t* nvtxs, idx_t* ncon, idx_t* xadj, idx_t* adjncy, idx_t* vwgt, idx_t* vsize,
                        idx_t* adjwgt, idx_t* nparts, real_t* tpwgts, real_t* ubvec, idx_t* options, idx_t* edgecut,
                        idx_t* part);
#ifdef __cplusplus
}
#endif
#endif
