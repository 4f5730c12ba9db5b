/*
 * The drop-in, run inside teal itself — TEST INFRASTRUCTURE ONLY. Compiled (oracle/Makefile,
 * `make -C oracle dropin`) against the reference's own headers and sources, compiled in place, and
 * linked with teal_b200/libteal_b200.so. It builds a run case with teal's public API exactly as
 * teal's run programs do (run/isentropic_vortex/run.c, run/taylor_green_vortex/run.c) and runs
 * teal's own `simulation_run` (src/simulation/run.c:22-113) either stock or with the device Advance
 * method installed into `Simulation.advance.method` (src/simulation.h:36-41) through the binding
 * INTEGRATION.md shows (tg_mesh_of / tg_equations_of / tg_bind below are that binding, verbatim).
 *
 *   teal_dropin <vortex|tgv|implicit> <stock|device> [--precision exact|fp64] [--steps N]
 *               [--out FILE]
 *
 * teal's own run-loop lines go to stdout; FILE receives the final time and the inner cells'
 * primitive state (double time, then double[num_inner][5]).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "equations.h"
#include "euler.h"
#include "mesh.h"
#include "navierstokes.h"
#include "simulation.h"
#include "teal.h"
#include "teal_b200.h"

/* ---- the binding ------------------------------------------------------------- */

/* teal's Mesh -> tg_mesh: pointers only, no copies (src/mesh.h:13-72) */
static tg_mesh tg_mesh_of(const Mesh *m)
{
    tg_mesh t = {0};
    t.num_cells = m->cells.num;
    t.num_inner_cells = m->cells.num_inner;
    t.off_boundary_cells = m->cells.off_boundary;
    t.off_periodic_cells = m->cells.off_periodic;
    t.cell_cell_off = m->cells.cell.off;
    t.cell_cell_idx = m->cells.cell.idx;
    t.cell_volume = m->cells.volume;
    t.cell_center = (const double *)m->cells.center;
    t.cell_projection = (const double *)m->cells.projection;
    t.cell_offset = (const double *)m->cells.offset;
    t.sum_volume = m->cells.sum_volume;
    t.num_faces = m->faces.num;
    t.num_inner_faces = m->faces.num_inner;
    t.off_boundary_faces = m->faces.off_boundary;
    t.face_cell = (const int *)m->faces.cell_idx;
    t.face_area = m->faces.area;
    t.face_basis = (const double *)m->faces.basis;
    t.face_weight = (const double *)m->faces.weight;
    t.face_offset = (const double *)m->faces.offset;
    t.face_correction = (const double *)m->faces.correction;
    t.num_entities = m->entities.num;
    t.num_inner_entities = m->entities.num_inner;
    t.off_boundary_entities = m->entities.off_boundary;
    t.entity_face_off = m->entities.face_off;
    t.num_neighbors = m->neighbors.num;
    t.neighbor_tag = (const int *)m->neighbors.tag;
    t.neighbor_recv_off = m->neighbors.recv_off;
    t.neighbor_send_off = m->neighbors.send.off;
    t.neighbor_send_idx = m->neighbors.send.idx;
    return t;
}

/* teal's Equations -> tg_equations: the plugin table by name (src/equations.h:97-111) */
static tg_equations tg_equations_of(const Equations *e, int *kind, double *ctx)
{
    tg_equations t = {0};
    t.physics = strcmp(e->name, "navier-stokes") ? TG_EULER : TG_NAVIERSTOKES;
    t.space_order = e->space_order;
    t.convective = e->convective.flux ? tg_convective_select(e->convective.name) : TG_FLUX_NONE;
    t.viscous = e->viscous.flux ? tg_viscous_select(e->viscous.name) : TG_VISCOUS_NONE;
    t.limiter = e->limiter.kind;                /* same numbering as limiter.h */
    t.limiter_parameter = e->limiter.parameter; /* Venkatakrishnan eps^2, or null */
    for (int i = 0; i < e->properties.num && i < 3; i++) t.property[i] = e->properties.data[i];
    t.num_boundaries = e->boundary.num;
    for (int i = 0; i < e->boundary.num; i++) {
        kind[i] = tg_boundary_select(e->boundary.name[i], t.physics); /* "custom": TG_BC_CUSTOM */
        if (e->boundary.context[i]) memcpy(&ctx[5 * i], e->boundary.context[i], 5 * sizeof(double));
    }
    t.boundary_kind = kind;
    t.boundary_context = ctx;
    return t;
}

/* ---- run cases (teal's own run programs, smaller meshes) --------------------------------------- */

static double wrap(double x, double xmin, double xmax)
{
    return (x >= 0 ? xmin : xmax) + fmod(x, xmax - xmin);
}

/* run/isentropic_vortex/run.c:10-27 */
static void vortex(void *primitive_, const double *property, Vector center, double time, const void *context)
{
    (void)context;
    EulerPrimitive *primitive = primitive_;
    double gamma = property[EULER_HEAT_CAPACITY_RATIO];
    Vector position = {.x = 5, .y = 5}, velocity = {.x = 1, .y = 1};
    double strength = 5;
    double dx = wrap(center.x - (velocity.x * time), 0, 10) - position.x;
    double dy = wrap(center.y - (velocity.y * time), 0, 10) - position.y;
    double r2 = (dx * dx) + (dy * dy);
    primitive->density =
        pow(1 - ((gamma - 1) * sq(strength) / (8 * gamma * sq(M_PI)) * exp(1 - r2)), 1 / (gamma - 1));
    primitive->velocity.x = velocity.x - (strength / (2 * M_PI) * exp((1 - r2) / 2) * dy);
    primitive->velocity.y = velocity.y + (strength / (2 * M_PI) * exp((1 - r2) / 2) * dx);
    primitive->velocity.z = 0;
    primitive->pressure = pow(primitive->density, gamma);
}

/* run/taylor_green_vortex/run.c:10-21 (Mach 0.1) */
static void taylor_green(void *primitive_, const double *property, Vector center, double time,
                         const void *context)
{
    (void)time, (void)context;
    NavierStokesPrimitive *primitive = primitive_;
    double gamma = property[NAVIERSTOKES_HEAT_CAPACITY_RATIO];
    double mach = 0.1;
    double p0 = 1 / (gamma * sq(mach));
    primitive->velocity.x = sin(center.x) * cos(center.y) * cos(center.z);
    primitive->velocity.y = -cos(center.x) * sin(center.y) * cos(center.z);
    primitive->velocity.z = 0;
    primitive->pressure = p0 + ((cos(2 * center.x) + cos(2 * center.y)) * (cos(2 * center.z) + 2) / 16);
    primitive->density = primitive->pressure / p0;
}

static Advance *device_method(const char *name)
{
    switch (tg_advance_select(name)) {
        case TG_ADVANCE_EULER: return tg_teal_euler;
        case TG_ADVANCE_LSERK: return tg_teal_lserk;
        case TG_ADVANCE_IMPLICIT_EULER: return tg_teal_implicit_euler;
        default: teal_error("no device method for advance \"%s\"", name);
    }
}

int main(int argc, char **argv)
{
    if (argc < 3) {
        fprintf(stderr, "usage: %s <vortex|tgv|implicit> <stock|device> [--precision exact|fp64] "
                        "[--steps N] [--out FILE]\n", argv[0]);
        return 2;
    }
    const char *kase = argv[1], *mode = argv[2], *out = 0;
    int precision = TG_PRECISION_FP64_EXACT, steps = -1;
    for (int i = 3; i + 1 < argc; i += 2) {
        if (!strcmp(argv[i], "--precision")) precision = strcmp(argv[i + 1], "fp64") ? TG_PRECISION_FP64_EXACT
                                                                                     : TG_PRECISION_FP64;
        else if (!strcmp(argv[i], "--steps")) steps = atoi(argv[i + 1]);
        else if (!strcmp(argv[i], "--out")) out = argv[i + 1];
    }
    int targc = 1;
    char arg0[] = "teal_dropin";
    char *targv_store[] = {arg0, 0};
    char **targv = targv_store;
    teal_init(&targc, &targv);

    Mesh *mesh;
    Equations *eqns;
    Simulation *sim;
    if (!strcmp(kase, "tgv")) { /* run/taylor_green_vortex/run.c, 24^3 */
        Vector lo = {0, 0, 0}, hi = {2 * M_PI, 2 * M_PI, 2 * M_PI};
        mesh = mesh_create(lo, hi, (Triple){24, 24, 24}, (Triple){1, 1, 1});
        mesh_generate(mesh);
        eqns = navierstokes_create(mesh);
        equations_set_convective_flux(eqns, "roe");
        equations_set_limiter(eqns, "venkatakrishnan", 1);
        equations_set_property(eqns, "dynamic viscosity", 1.0 / 1600);
        equations_set_initial_condition(eqns, "domain", taylor_green, 0);
        sim = simulation_create(eqns, "");
        simulation_set_advance(sim, "lserk", 0.99, (RungeKutta[]){{3, 3}});
        simulation_set_max_iter(sim, steps > 0 ? steps : 20);
        simulation_set_out_iter(sim, 5);
    }
    else { /* run/isentropic_vortex/run.c on the 64 x 64 x 4 box of the parity workload */
        Vector lo = {0, 0, 0}, hi = {10, 10, 0.625};
        mesh = mesh_create(lo, hi, (Triple){64, 64, 4}, (Triple){1, 1, 1});
        mesh_generate(mesh);
        eqns = euler_create(mesh); /* hllc + Barth-Jespersen ("minmod") by default */
        equations_set_initial_condition(eqns, "domain", vortex, 0);
        sim = simulation_create(eqns, "");
        if (!strcmp(kase, "implicit")) {
            simulation_set_advance(sim, "implicit euler", 5, (NewtonKrylov[]){{0.1, 0.3, 30}});
            simulation_set_max_iter(sim, steps > 0 ? steps : 3);
            simulation_set_out_iter(sim, 1);
        }
        else {
            simulation_set_advance(sim, "lserk", 0.5, (RungeKutta[]){{3, 3}});
            simulation_set_max_iter(sim, steps > 0 ? steps : 200);
            simulation_set_out_iter(sim, 20);
        }
    }

    tg_ctx *gpu = 0;
    int kind[16];
    double ctx[16 * 5] = {0};
    if (!strcmp(mode, "device")) {
        tg_mesh tm = tg_mesh_of(mesh);
        tg_equations te = tg_equations_of(eqns, kind, ctx);
        if (tg_create(&tm, &te, precision, &gpu) || tg_bind(eqns, gpu, eqns->primitive.data))
            teal_error("%s", tg_last_error());
        /* install the device Advance method with teal's signature (src/simulation.h:6-7) */
        sim->advance.method = device_method(sim->advance.name);
    }
    else if (strcmp(mode, "stock")) {
        teal_error("invalid mode (%s)", mode);
    }

    double time = simulation_run(sim);

    if (out) {
        FILE *f = fopen(out, "wb");
        if (!f) teal_error("cannot open %s", out);
        int n = mesh->cells.num_inner, stride = eqns->primitive.stride;
        fwrite(&time, sizeof(time), 1, f);
        for (int i = 0; i < n; i++) fwrite((double *)eqns->primitive.data + (size_t)i * stride, sizeof(double), 5, f);
        fclose(f);
    }
    if (gpu) {
        tg_unbind(eqns);
        tg_destroy(gpu);
    }
    simulation_destroy(sim);
    equations_destroy(eqns);
    mesh_destroy(mesh);
    teal_deinit();
    return 0;
}
