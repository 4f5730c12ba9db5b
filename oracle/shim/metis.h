/*
 * Stand-in for the one METIS routine the reference's mesh generation calls
 * (mesh/generate.c:35-43, METIS 5.x `METIS_MeshToDual`). Test infrastructure only: METIS is not in
 * this image. The published METIS 5 rule is restated in shim_metis.c; it decides connectivity
 * (which cells are neighbours) and the order neighbours are listed in, never any arithmetic.
 */
#pragma once

typedef long idx_t;

#define METIS_OK 1
#define METIS_ERROR (-4)

int METIS_MeshToDual(idx_t *ne, idx_t *nn, idx_t *eptr, idx_t *eind, idx_t *ncommon,
                     idx_t *numflag, idx_t **xadj, idx_t **adjncy);
int METIS_Free(void *ptr);
