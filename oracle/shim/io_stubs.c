/*
 * Link stubs for the reference's HDF5 output/restart routines (mesh/write.c, equations/write.c,
 * equations/read.c), which need parallel HDF5 (absent here) and lie off the residual /
 * time-integration path. The oracle harness never asks for output (empty prefix, no restart), so
 * reaching one of these is an error.
 */
#include <stdio.h>
#include <stdlib.h>

#include "equations.h"
#include "mesh.h"

void mesh_write(const Mesh *mesh, const char *name)
{
    (void)mesh;
    fprintf(stderr, "oracle: mesh_write(%s) is not available (no HDF5)\n", name);
    abort();
}

void equations_write(const Equations *eqns, const char *name, double time, int index)
{
    (void)eqns;
    (void)time;
    (void)index;
    fprintf(stderr, "oracle: equations_write(%s) is not available (no HDF5)\n", name);
    abort();
}

void equations_read(const Equations *eqns, const char *fname, double *time, int *index)
{
    (void)eqns;
    (void)time;
    (void)index;
    fprintf(stderr, "oracle: equations_read(%s) is not available (no HDF5)\n", fname);
    abort();
}
