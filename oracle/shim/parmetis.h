/*
 * Stand-in for the two ParMETIS routines the reference's mesh reader calls (mesh/dual.c:26, :104;
 * ParMETIS 4.x `ParMETIS_V3_Mesh2Dual` and `ParMETIS_V3_PartKway`). Test infrastructure only:
 * ParMETIS is not in this image, and the oracle runs one rank, where the dual graph is the one
 * METIS_MeshToDual's rule gives (shim_metis.c) and every cell lies in part 0.
 */
#pragma once

#include <inttypes.h> /* as the real metis.h / parmetis.h headers provide */

#include "metis.h"
#include "mpi.h"

typedef double real_t;

int ParMETIS_V3_Mesh2Dual(idx_t *elmdist, idx_t *eptr, idx_t *eind, idx_t *numflag, idx_t *ncommonnodes,
                          idx_t **xadj, idx_t **adjncy, MPI_Comm *comm);
int ParMETIS_V3_PartKway(idx_t *vtxdist, idx_t *xadj, idx_t *adjncy, idx_t *vwgt, idx_t *adjwgt, idx_t *wgtflag,
                         idx_t *numflag, idx_t *ncon, idx_t *nparts, real_t *tpwgts, real_t *ubvec, idx_t *options,
                         idx_t *edgecut, idx_t *part, MPI_Comm *comm);
