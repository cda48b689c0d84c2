/* Shim for the reference build: constants and prototype of METIS as used by
   Mesh::ddm_metis (Mesh.cpp:354-452).  The harness runs with metis=false, so
   the stub in lapack_standin.cpp aborts if it is ever reached. */
#ifndef HTF_SHIM_METIS_H
#define HTF_SHIM_METIS_H
typedef int idx_t;
typedef float real_t;
#define METIS_NOPTIONS 40
enum { METIS_OPTION_PTYPE, METIS_OPTION_OBJTYPE, METIS_OPTION_CTYPE, METIS_OPTION_IPTYPE,
       METIS_OPTION_RTYPE, METIS_OPTION_DBGLVL, METIS_OPTION_NITER, METIS_OPTION_NCUTS,
       METIS_OPTION_SEED, METIS_OPTION_NO2HOP, METIS_OPTION_MINCONN, METIS_OPTION_CONTIG,
       METIS_OPTION_COMPRESS, METIS_OPTION_CCORDER, METIS_OPTION_PFACTOR, METIS_OPTION_NSEPS,
       METIS_OPTION_UFACTOR, METIS_OPTION_NUMBERING };
enum { METIS_PTYPE_RB, METIS_PTYPE_KWAY };
enum { METIS_OBJTYPE_CUT, METIS_OBJTYPE_VOL, METIS_OBJTYPE_NODE };
enum { METIS_CTYPE_RM, METIS_CTYPE_SHEM };
enum { METIS_IPTYPE_GROW, METIS_IPTYPE_RANDOM, METIS_IPTYPE_EDGE, METIS_IPTYPE_NODE };
enum { METIS_RTYPE_FM, METIS_RTYPE_GREEDY, METIS_RTYPE_SEP2SIDED, METIS_RTYPE_SEP1SIDED };
enum { METIS_DBG_INFO = 1 };
#ifdef __cplusplus
extern "C"
#endif
int METIS_PartMeshDual(idx_t *ne, idx_t *nn, idx_t *eptr, idx_t *eind, idx_t *vwgt,
                       idx_t *vsize, idx_t *ncommon, idx_t *nparts, real_t *tpwgts,
                       idx_t *options, idx_t *objval, idx_t *epart, idx_t *npart);
#endif
