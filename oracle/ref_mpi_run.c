/*
 * The reference solver on all host cores: teal's own MPI domain decomposition of the Taylor-Green
 * vortex run (mesh_create's Cartesian split, halo exchanges, global reductions), over the
 * multi-process MPI subset of shim/shim_mpi_fork.c. CPU-baseline infrastructure only (bench.py's
 * reference arm and its test); it calls the reference's public API and computes nothing itself
 * beyond the initial field.
 *
 *   TEAL_SHIM_RANKS=16 _ref/teal_ref_mpi [--n 128] [--steps 10] [--warmup 2]
 *
 * Case: [0, 2 pi]^3 fully periodic, n^3 hexahedra, Navier-Stokes with roe + venkatakrishnan(1),
 * dynamic viscosity 1/1600, lserk {3, 3} at CFL 0.99; initial field as
 * run/taylor_green_vortex/run.c:10-21 (Mach 0.1, gamma 1.4). Rank 0 prints one JSON line: ranks,
 * global inner cells, steps, the slowest rank's seconds over the timed steps (after a barrier) and
 * the residual of the last step.
 */
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "equations.h"
#include "mesh.h"
#include "navierstokes.h"
#include "simulation.h"
#include "sync.h"
#include "teal.h"

static void taylor_green(const Mesh *mesh, Equations *eqns)
{
    const double gamma = 1.4, mach = 0.1;
    const double p0 = 1 / (gamma * mach * mach);
    int stride = eqns->primitive.stride;
    double *prim = eqns->primitive.data;
    for (int i = 0; i < mesh->cells.num_inner; i++) {
        Vector c = mesh->cells.center[i];
        double *q = prim + (size_t)i * stride;
        q[1] = sin(c.x) * cos(c.y) * cos(c.z);
        q[2] = -cos(c.x) * sin(c.y) * cos(c.z);
        q[3] = 0;
        q[4] = p0 + (((cos(2 * c.x) + cos(2 * c.y)) * (cos(2 * c.z) + 2)) / 16);
        q[0] = q[4] / p0;
    }
}

int main(int argc, char **argv)
{
    int n = 128, steps = 10, warmup = 2;
    for (int i = 1; i + 1 < argc; i += 2) {
        if (!strcmp(argv[i], "--n")) n = atoi(argv[i + 1]);
        else if (!strcmp(argv[i], "--steps")) steps = atoi(argv[i + 1]);
        else if (!strcmp(argv[i], "--warmup")) warmup = atoi(argv[i + 1]);
        else {
            fprintf(stderr, "usage: %s [--n N] [--steps K] [--warmup W]\n", argv[0]);
            return 2;
        }
    }
    static char arg0[] = "teal_ref_mpi";
    static char arg1[] = "-q";
    char *targv_store[] = {arg0, arg1, 0};
    int targc = 2;
    char **targv = targv_store;
    teal_init(&targc, &targv);

    const double two_pi = 2 * acos(-1.0);
    Mesh *mesh = mesh_create((Vector){0, 0, 0}, (Vector){two_pi, two_pi, two_pi}, (Triple){n, n, n},
                             (Triple){1, 1, 1});
    mesh_generate(mesh);
    Equations *eqns = navierstokes_create(mesh);
    equations_set_convective_flux(eqns, "roe");
    equations_set_limiter(eqns, "venkatakrishnan", 1.0);
    equations_set_property(eqns, "dynamic viscosity", 1.0 / 1600);
    taylor_green(mesh, eqns);

    Simulation *sim = simulation_create(eqns, "");
    RungeKutta rk = {3, 3};
    simulation_set_advance(sim, "lserk", 0.99, &rk);

    double time = 0, residual[5] = {0, 0, 0, 0, 0};
    for (int s = 0; s < warmup; s++) {
        sim->advance.method(eqns, &time, residual, DBL_MAX, sim->advance.courant, sim->advance.context);
    }
    double start = 0;
    sync_sum(&start, 1, MPI_DOUBLE); /* every rank here before the clock starts */
    start = MPI_Wtime();
    for (int s = 0; s < steps; s++) {
        sim->advance.method(eqns, &time, residual, DBL_MAX, sim->advance.courant, sim->advance.context);
    }
    double seconds = MPI_Wtime() - start;
    sync_max(&seconds, 1, MPI_DOUBLE);
    long cells = mesh->cells.num_inner;
    sync_sum(&cells, 1, MPI_LONG);
    if (sync.rank == 0) {
        printf("{\"ranks\": %d, \"cells\": %ld, \"steps\": %d, \"seconds\": %.9g, \"time\": %.17g, "
               "\"residual\": [%.17g, %.17g, %.17g, %.17g, %.17g]}\n",
               sync.size, cells, steps, seconds, time, residual[0], residual[1], residual[2], residual[3],
               residual[4]);
        fflush(stdout);
    }
    simulation_destroy(sim);
    equations_destroy(eqns);
    mesh_destroy(mesh);
    teal_deinit();
    return 0;
}
