/*
 * Restatement of METIS 5's dual-graph rule for `METIS_MeshToDual` (METIS 5.1.0, libmetis/mesh.c,
 * CreateGraphDual / FindCommonElements; the dependency is absent from the reference tree, which
 * only calls it at mesh/generate.c:35-43). Test infrastructure only.
 *
 * Two elements i and j are joined when the number of nodes they share, `overlap`, satisfies
 *     overlap >= ncommon || overlap >= len(i) - 1 || overlap >= len(j) - 1.
 * For element i the neighbours are listed in order of first encounter while scanning i's nodes in
 * order and, for each node, the elements that hold it in increasing element number.
 */
#include <stdlib.h>

#include "metis.h"

int METIS_MeshToDual(idx_t *ne_, idx_t *nn_, idx_t *eptr, idx_t *eind, idx_t *ncommon_,
                     idx_t *numflag, idx_t **xadj_out, idx_t **adjncy_out)
{
    idx_t ne = *ne_, nn = *nn_, ncommon = *ncommon_;
    if (*numflag != 0 || ne < 0 || nn < 0) {
        return METIS_ERROR;
    }

    /* node -> element lists, elements ascending */
    idx_t *nptr = calloc((size_t)nn + 1, sizeof(idx_t));
    for (idx_t e = 0; e < ne; e++) {
        for (idx_t k = eptr[e]; k < eptr[e + 1]; k++) {
            nptr[eind[k] + 1] += 1;
        }
    }
    for (idx_t n = 0; n < nn; n++) {
        nptr[n + 1] += nptr[n];
    }
    idx_t *nind = malloc(((size_t)nptr[nn] + 1) * sizeof(idx_t));
    idx_t *cur = malloc(((size_t)nn + 1) * sizeof(idx_t));
    for (idx_t n = 0; n < nn; n++) {
        cur[n] = nptr[n];
    }
    for (idx_t e = 0; e < ne; e++) {
        for (idx_t k = eptr[e]; k < eptr[e + 1]; k++) {
            nind[cur[eind[k]]++] = e;
        }
    }

    idx_t *marker = calloc((size_t)ne + 1, sizeof(idx_t));
    idx_t *nbrs = malloc(((size_t)ne + 1) * sizeof(idx_t));

    /* two passes: count, then fill */
    idx_t *xadj = calloc((size_t)ne + 1, sizeof(idx_t));
    idx_t *adjncy = 0;
    for (int pass = 0; pass < 2; pass++) {
        for (idx_t e = 0; e < ne; e++) {
            idx_t len_e = eptr[e + 1] - eptr[e];
            idx_t nnbrs = 0;
            for (idx_t k = eptr[e]; k < eptr[e + 1]; k++) {
                idx_t node = eind[k];
                for (idx_t m = nptr[node]; m < nptr[node + 1]; m++) {
                    idx_t other = nind[m];
                    if (other == e) {
                        continue;
                    }
                    if (marker[other] == 0) {
                        nbrs[nnbrs++] = other;
                    }
                    marker[other] += 1;
                }
            }
            idx_t kept = 0;
            for (idx_t m = 0; m < nnbrs; m++) {
                idx_t other = nbrs[m];
                idx_t overlap = marker[other];
                idx_t len_o = eptr[other + 1] - eptr[other];
                if (overlap >= ncommon || overlap >= len_e - 1 || overlap >= len_o - 1) {
                    if (pass == 1) {
                        adjncy[xadj[e] + kept] = other;
                    }
                    kept += 1;
                }
                marker[other] = 0;
            }
            if (pass == 0) {
                xadj[e + 1] = kept;
            }
        }
        if (pass == 0) {
            for (idx_t e = 0; e < ne; e++) {
                xadj[e + 1] += xadj[e];
            }
            adjncy = malloc(((size_t)xadj[ne] + 1) * sizeof(idx_t));
        }
    }

    free(nptr);
    free(nind);
    free(cur);
    free(marker);
    free(nbrs);
    *xadj_out = xadj;
    *adjncy_out = adjncy;
    return METIS_OK;
}

int METIS_Free(void *ptr)
{
    free(ptr);
    return METIS_OK;
}

/* ---- ParMETIS on one rank (parmetis.h) ------------------------------------------------------ */

#include "parmetis.h"

/* ParMETIS' dual graph joins two elements when they share at least `ncommonnodes` nodes (its
 * documented rule; unlike METIS_MeshToDual there is no rule for elements sharing all but one of
 * their nodes). On one rank the order of each element's neighbours does not reach the reader's
 * result; here it is the order of first encounter, as above. */
int ParMETIS_V3_Mesh2Dual(idx_t *elmdist, idx_t *eptr, idx_t *eind, idx_t *numflag, idx_t *ncommonnodes,
                          idx_t **xadj_out, idx_t **adjncy_out, MPI_Comm *comm)
{
    int size = 1;
    MPI_Comm_size(*comm, &size);
    if (size != 1 || elmdist[0] != 0 || *numflag != 0) {
        return METIS_ERROR;
    }
    idx_t ne = elmdist[1], nn = 0, ncommon = *ncommonnodes;
    for (idx_t k = 0; k < eptr[ne]; k++) {
        if (eind[k] + 1 > nn) nn = eind[k] + 1;
    }
    idx_t *nptr = calloc((size_t)nn + 1, sizeof(idx_t));
    for (idx_t k = 0; k < eptr[ne]; k++) nptr[eind[k] + 1] += 1;
    for (idx_t n = 0; n < nn; n++) nptr[n + 1] += nptr[n];
    idx_t *nind = malloc((size_t)(nptr[nn] > 0 ? nptr[nn] : 1) * sizeof(idx_t));
    idx_t *fill = calloc((size_t)nn + 1, sizeof(idx_t));
    for (idx_t e = 0; e < ne; e++) {
        for (idx_t k = eptr[e]; k < eptr[e + 1]; k++) nind[nptr[eind[k]] + fill[eind[k]]++] = e;
    }
    idx_t *count = calloc((size_t)(ne > 0 ? ne : 1), sizeof(idx_t));
    idx_t *seen = malloc((size_t)(ne > 0 ? ne : 1) * sizeof(idx_t));
    idx_t *xadj = malloc(((size_t)ne + 1) * sizeof(idx_t));
    size_t cap = 16, len = 0;
    idx_t *adjncy = malloc(cap * sizeof(idx_t));
    xadj[0] = 0;
    for (idx_t e = 0; e < ne; e++) {
        idx_t nseen = 0;
        for (idx_t k = eptr[e]; k < eptr[e + 1]; k++) {
            idx_t n = eind[k];
            for (idx_t m = nptr[n]; m < nptr[n + 1]; m++) {
                idx_t f = nind[m];
                if (f == e) continue;
                if (count[f] == 0) seen[nseen++] = f;
                count[f] += 1;
            }
        }
        for (idx_t q = 0; q < nseen; q++) {
            idx_t f = seen[q];
            if (count[f] >= ncommon) {
                if (len == cap) {
                    cap *= 2;
                    adjncy = realloc(adjncy, cap * sizeof(idx_t));
                }
                adjncy[len++] = f;
            }
            count[f] = 0;
        }
        xadj[e + 1] = (idx_t)len;
    }
    free(nptr);
    free(nind);
    free(fill);
    free(count);
    free(seen);
    *xadj_out = xadj;
    *adjncy_out = adjncy;
    return METIS_OK;
}

int ParMETIS_V3_PartKway(idx_t *vtxdist, idx_t *xadj, idx_t *adjncy, idx_t *vwgt, idx_t *adjwgt, idx_t *wgtflag,
                         idx_t *numflag, idx_t *ncon, idx_t *nparts, real_t *tpwgts, real_t *ubvec, idx_t *options,
                         idx_t *edgecut, idx_t *part, MPI_Comm *comm)
{
    (void)xadj;
    (void)adjncy;
    (void)vwgt;
    (void)adjwgt;
    (void)wgtflag;
    (void)numflag;
    (void)ncon;
    (void)tpwgts;
    (void)ubvec;
    (void)options;
    int size = 1;
    MPI_Comm_size(*comm, &size);
    if (size != 1 || *nparts != 1) {
        return METIS_ERROR;
    }
    for (idx_t i = 0; i < vtxdist[1] - vtxdist[0]; i++) {
        part[i] = 0;
    }
    *edgecut = 0;
    return METIS_OK;
}
