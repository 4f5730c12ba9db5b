/*
 * ctypes-callable harness around the reference solver compiled in place (oracle/_ref). Test
 * infrastructure only: tests, fixtures and the CPU-baseline leg of bench.py call it to obtain the
 * reference's own results. It only calls the reference's public API (src/*.h) and reads its
 * structs; it computes nothing itself.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "equations.h"
#include "euler.h"
#include "mesh.h"
#include "navierstokes.h"
#include "simulation.h"
#include "teal.h"
#include "kdtree.h"

int ref_init(void)
{
    static int done = 0;
    if (!done) {
        static char arg0[] = "teal_ref";
        static char arg1[] = "-q";
        static char *argv_store[] = {arg0, arg1, 0};
        int argc = 2;
        char **argv = argv_store;
        teal_init(&argc, &argv);
        done = 1;
    }
    return 0;
}

void ref_set_quiet(int quiet)
{
    teal.quiet = quiet;
}

/* ---- mesh ----------------------------------------------------------------------------------- */

void *ref_mesh_cartesian(const double *min, const double *max, const int *num, const int *periodic)
{
    Vector lo = {min[0], min[1], min[2]};
    Vector hi = {max[0], max[1], max[2]};
    Triple n = {num[0], num[1], num[2]};
    Triple p = {periodic[0], periodic[1], periodic[2]};
    Mesh *mesh = mesh_create(lo, hi, n, p);
    return mesh;
}

/* A one-rank mesh from nodes, cells (node lists: inner cells, then boundary face cells) and entity
 * cell ranges, in the state mesh_read leaves it before mesh_generate (src/mesh/read.c): all nodes
 * and cells local, no periodic entities, no neighbour ranks (as create_neighbors leaves a rank
 * without neighbours, src/mesh/create.c:388-440). Entities whose range ends within the inner cells
 * are inner entities. */
void *ref_mesh_cells(int num_nodes, const double *coord, int num_cells, int num_inner, const int *node_off,
                     const int *node_idx, int num_entities, const char *const *names, const int *cell_off)
{
    Mesh *mesh = teal_calloc(1, sizeof(*mesh));
    mesh->nodes.num = num_nodes;
    mesh->nodes.num_inner = num_nodes;
    mesh->nodes.global = teal_calloc(num_nodes, sizeof(*mesh->nodes.global));
    mesh->nodes.coord = teal_calloc(num_nodes, sizeof(*mesh->nodes.coord));
    for (int i = 0; i < num_nodes; i++) {
        mesh->nodes.global[i] = i;
        mesh->nodes.coord[i] = (Vector){coord[(3 * i) + 0], coord[(3 * i) + 1], coord[(3 * i) + 2]};
    }
    mesh->cells.num = num_cells;
    mesh->cells.num_inner = num_inner;
    mesh->cells.off_boundary = num_cells;
    mesh->cells.off_periodic = num_cells;
    mesh->cells.node.off = teal_calloc(num_cells + 1, sizeof(int));
    mesh->cells.node.idx = teal_calloc(node_off[num_cells], sizeof(int));
    memcpy(mesh->cells.node.off, node_off, (num_cells + 1) * sizeof(int));
    memcpy(mesh->cells.node.idx, node_idx, node_off[num_cells] * sizeof(int));
    int num_inner_entities = 0;
    for (int i = 0; i < num_entities; i++) {
        if (cell_off[i + 1] <= num_inner) num_inner_entities = i + 1;
    }
    mesh->entities.num = num_entities;
    mesh->entities.num_inner = num_inner_entities;
    mesh->entities.off_boundary = num_entities;
    mesh->entities.name = teal_calloc(num_entities, sizeof(*mesh->entities.name));
    mesh->entities.cell_off = teal_calloc(num_entities + 1, sizeof(int));
    mesh->entities.rotation = teal_calloc(num_entities, sizeof(*mesh->entities.rotation));
    mesh->entities.translation = teal_calloc(num_entities, sizeof(*mesh->entities.translation));
    for (int i = 0; i < num_entities; i++) {
        strncpy(mesh->entities.name[i], names[i], sizeof(mesh->entities.name[i]) - 1);
    }
    memcpy(mesh->entities.cell_off, cell_off, (num_entities + 1) * sizeof(int));
    mesh->neighbors.num = 0;
    mesh->neighbors.tag = teal_calloc(1, sizeof(*mesh->neighbors.tag));
    mesh->neighbors.rank = teal_calloc(1, sizeof(int));
    mesh->neighbors.recv_off = teal_calloc(1, sizeof(int));
    mesh->neighbors.recv_off[0] = num_cells;
    mesh->neighbors.send.off = teal_calloc(1, sizeof(int));
    mesh->neighbors.send.idx = teal_calloc(1, sizeof(int));
    return mesh;
}

/* teal's mesh_read of a Gmsh 4.1 file (mesh/read.c:901-917, one rank), before mesh_generate */
void *ref_mesh_read(const char *fname)
{
    return mesh_read(fname);
}

/* apply a node displacement table (in node order at the time of the call) before generation */
static const double *displacement = 0;
static int displacement_num = 0;
static int displacement_cur = 0;
static void displace(Vector *coord)
{
    if (displacement_cur < displacement_num) {
        coord->x += displacement[(3 * displacement_cur) + 0];
        coord->y += displacement[(3 * displacement_cur) + 1];
        coord->z += displacement[(3 * displacement_cur) + 2];
    }
    displacement_cur += 1;
}

void ref_mesh_displace(void *mesh, const double *disp, int num)
{
    displacement = disp;
    displacement_num = num;
    displacement_cur = 0;
    mesh_modify(mesh, displace);
    displacement = 0;
}

void ref_mesh_split(void *mesh, const char *entity, const double *root, const double *normal)
{
    mesh_split(mesh, entity, (Vector){root[0], root[1], root[2]},
               (Vector){normal[0], normal[1], normal[2]});
}

void ref_mesh_generate(void *mesh)
{
    mesh_generate(mesh);
}

void ref_mesh_validate(void *mesh)
{
    mesh_validate(mesh);
}

void ref_mesh_destroy(void *mesh)
{
    mesh_destroy(mesh);
}

/* counts[0..15]: nodes.num, nodes.num_inner, cells.num, cells.num_inner, cells.off_boundary,
 * cells.off_periodic, faces.num, faces.num_inner, faces.off_boundary, cells.cell nnz,
 * entities.num, entities.num_inner, entities.off_boundary, neighbors.num, neighbors.send nnz,
 * cells.node nnz */
void ref_mesh_counts(const void *mesh_, long *counts)
{
    const Mesh *mesh = mesh_;
    counts[0] = mesh->nodes.num;
    counts[1] = mesh->nodes.num_inner;
    counts[2] = mesh->cells.num;
    counts[3] = mesh->cells.num_inner;
    counts[4] = mesh->cells.off_boundary;
    counts[5] = mesh->cells.off_periodic;
    counts[6] = mesh->faces.num;
    counts[7] = mesh->faces.num_inner;
    counts[8] = mesh->faces.off_boundary;
    counts[9] = mesh->cells.cell.off[mesh->cells.num];
    counts[10] = mesh->entities.num;
    counts[11] = mesh->entities.num_inner;
    counts[12] = mesh->entities.off_boundary;
    counts[13] = mesh->neighbors.num;
    counts[14] = mesh->neighbors.send.off[mesh->neighbors.num];
    counts[15] = mesh->cells.node.off[mesh->cells.num];
}

double ref_mesh_sum_volume(const void *mesh_)
{
    return ((const Mesh *)mesh_)->cells.sum_volume;
}

const void *ref_mesh_array(const void *mesh_, const char *name)
{
    const Mesh *mesh = mesh_;
    if (!strcmp(name, "nodes.coord")) return mesh->nodes.coord;
    if (!strcmp(name, "cells.node.off")) return mesh->cells.node.off;
    if (!strcmp(name, "cells.node.idx")) return mesh->cells.node.idx;
    if (!strcmp(name, "cells.cell.off")) return mesh->cells.cell.off;
    if (!strcmp(name, "cells.cell.idx")) return mesh->cells.cell.idx;
    if (!strcmp(name, "cells.volume")) return mesh->cells.volume;
    if (!strcmp(name, "cells.center")) return mesh->cells.center;
    if (!strcmp(name, "cells.projection")) return mesh->cells.projection;
    if (!strcmp(name, "cells.offset")) return mesh->cells.offset;
    if (!strcmp(name, "faces.cell_idx")) return mesh->faces.cell_idx;
    if (!strcmp(name, "faces.area")) return mesh->faces.area;
    if (!strcmp(name, "faces.center")) return mesh->faces.center;
    if (!strcmp(name, "faces.basis")) return mesh->faces.basis;
    if (!strcmp(name, "faces.weight")) return mesh->faces.weight;
    if (!strcmp(name, "faces.offset")) return mesh->faces.offset;
    if (!strcmp(name, "faces.correction")) return mesh->faces.correction;
    if (!strcmp(name, "entities.cell_off")) return mesh->entities.cell_off;
    if (!strcmp(name, "entities.face_off")) return mesh->entities.face_off;
    if (!strcmp(name, "neighbors.tag")) return mesh->neighbors.tag;
    if (!strcmp(name, "neighbors.rank")) return mesh->neighbors.rank;
    if (!strcmp(name, "neighbors.recv_off")) return mesh->neighbors.recv_off;
    if (!strcmp(name, "neighbors.send.off")) return mesh->neighbors.send.off;
    if (!strcmp(name, "neighbors.send.idx")) return mesh->neighbors.send.idx;
    return 0;
}

const char *ref_mesh_entity_name(const void *mesh_, int idx)
{
    const Mesh *mesh = mesh_;
    if (idx < 0 || idx >= mesh->entities.num) {
        return 0;
    }
    return mesh->entities.name[idx];
}

/* ---- equations ------------------------------------------------------------------------------ */

void *ref_equations(void *mesh, int navierstokes)
{
    return navierstokes ? navierstokes_create(mesh) : euler_create(mesh);
}

void ref_set_space_order(void *eqns, int order)
{
    equations_set_space_order(eqns, order);
}

void ref_set_convective(void *eqns, const char *name)
{
    equations_set_convective_flux(eqns, (name && name[0]) ? name : 0);
}

void ref_set_viscous(void *eqns, const char *name)
{
    equations_set_viscous_flux(eqns, (name && name[0]) ? name : 0);
}

void ref_set_limiter(void *eqns, const char *name, double coefficient)
{
    equations_set_limiter(eqns, (name && name[0]) ? name : 0, coefficient);
}

/* Source terms as teal's run cases write them (host callbacks handed to equations_set_source):
 * kind 1, a body force with acceleration (p0, p1, p2) (run/rayleigh_taylor_instability/run.c:17-24,
 * there (0, -gravity, 0)); kind 2, bulk forcing of the x velocity towards p0 with time scale p1,
 * its Prepare averaging the state over "domain" with the reference's equations_average
 * (run/periodic_hill/run.c:8-21, there p0 = 1, p1 = 0.001). One source setting per process. */
static double src_par[4];
static double src_average[5];

static void src_body_force(void *source_, const double *property, Vector center, double time, const void *context)
{
    double *source = source_;
    const double *primitive = context;
    (void)property, (void)center, (void)time;
    source[1] = src_par[0] * primitive[0];
    source[2] = src_par[1] * primitive[0];
    source[3] = src_par[2] * primitive[0];
    source[4] = ((source[1] * primitive[1]) + (source[2] * primitive[2])) + (source[3] * primitive[3]);
}

static void src_bulk_prepare(const Equations *eqns, const void *primitive)
{
    equations_average(eqns, "domain", primitive, src_average);
}

static void src_bulk_forcing(void *source_, const double *property, Vector center, double time,
                             const void *context)
{
    double *source = source_;
    const double *primitive = context;
    (void)property, (void)center, (void)time;
    double s1 = primitive[0] * (src_par[0] - src_average[1]) / src_par[1];
    source[1] = s1;
    source[4] = primitive[1] * s1;
}

/* kind 3: a time- and position-dependent momentum forcing f = rho (0.1 sin(x + t), 0.05 cos(y - t), 0)
 * with its work u . f as the energy source; the device-function tests compile the same formula */
static void src_unsteady(void *source_, const double *property, Vector center, double time, const void *context)
{
    double *source = source_;
    const double *primitive = context;
    (void)property;
    double fx = 0.1 * primitive[0] * sin(center.x + time);
    double fy = 0.05 * primitive[0] * cos(center.y - time);
    source[0] = 0;
    source[1] = fx;
    source[2] = fy;
    source[3] = 0;
    source[4] = (primitive[1] * fx) + (primitive[2] * fy);
}

void ref_set_source(void *eqns, int kind, const double *par)
{
    for (int i = 0; i < 4; i++) src_par[i] = par ? par[i] : 0.0;
    if (kind == 1) equations_set_source(eqns, src_body_force, 0);
    else if (kind == 2) equations_set_source(eqns, src_bulk_forcing, src_bulk_prepare);
    else if (kind == 3) equations_set_source(eqns, src_unsteady, 0);
    else equations_set_source(eqns, 0, 0);
}

/* Custom boundary conditions (teal's "custom" kind with a Compute callback, boundary.c:27-33) as the
 * run cases write them; the device-function tests compile the same formulas. Kind 1: a wall moving
 * with speed bc_speed along x (run/lid_driven_cavity/run.c:7-17, there speed 1); kind 2: an
 * unsteady inflow state of the ghost centre and time. One setting per process. */
static double bc_speed = 1.0;

static void bc_moving_wall(void *outer_, const double *property, Vector center, double time, const void *context)
{
    double *outer = outer_;
    const double *inner = context;
    (void)property, (void)center, (void)time;
    outer[0] = inner[0];
    outer[1] = (2 * bc_speed) - inner[1];
    outer[2] = -inner[2];
    outer[3] = -inner[3];
    outer[4] = inner[4];
}

static void bc_unsteady_inflow(void *outer_, const double *property, Vector center, double time,
                               const void *context)
{
    double *outer = outer_;
    (void)context;
    outer[0] = 1 + (0.1 * sin(center.x - time));
    outer[1] = 0.5 + (0.05 * cos(center.y + (2 * time)));
    outer[2] = 0.01 * center.z;
    outer[3] = 0;
    outer[4] = (1 / property[0]) + (0.02 * sin(3 * time));
}

void ref_set_boundary_custom(void *eqns, const char *entity, int kind, double speed)
{
    bc_speed = speed;
    equations_set_boundary_condition(eqns, entity, "custom", kind == 1 ? bc_moving_wall : bc_unsteady_inflow, 0);
}

void ref_set_property(void *eqns, const char *name, double value)
{
    equations_set_property(eqns, name, value);
}

void ref_set_boundary(void *eqns, const char *entity, const char *name, const double *context)
{
    double *copy_ = 0;
    if (context) {
        copy_ = malloc(5 * sizeof(double)); /* lives as long as the process: BCs keep the pointer */
        memcpy(copy_, context, 5 * sizeof(double));
    }
    equations_set_boundary_condition(eqns, entity, name, 0, copy_);
}

double *ref_primitive(void *eqns)
{
    return ((Equations *)eqns)->primitive.data;
}

const double *ref_limiter_parameter(void *eqns)
{
    return ((Equations *)eqns)->limiter.parameter;
}

void ref_derivative(void *eqns, double *primitive, double *derivative, double time)
{
    equations_derivative(eqns, primitive, derivative, time);
}

void ref_boundary(void *eqns, double *primitive, double time)
{
    equations_boundary(eqns, primitive, time);
}

void ref_gradient(void *eqns, double *primitive, double *gradient)
{
    equations_gradient(eqns, primitive, gradient);
}

void ref_limiter(void *eqns, const double *primitive, double *gradient)
{
    equations_limiter(eqns, primitive, gradient);
}

double ref_timestep(void *eqns, const double *primitive)
{
    return equations_timestep(eqns, primitive);
}

void ref_residual(void *eqns, const double *derivative, double *residual)
{
    equations_residual(eqns, derivative, residual);
}

void ref_equations_destroy(void *eqns)
{
    equations_destroy(eqns);
}

/* ---- simulation ----------------------------------------------------------------------------- */

/* method: "euler", "lserk" or "implicit euler"; iparam/dparam: RungeKutta{time_order, num_stages}
 * or NewtonKrylov{newton_tolerance, krylov_tolerance, krylov_dimension} (null = defaults) */
void *ref_simulation(void *eqns, const char *method, double courant, const int *iparam,
                     const double *dparam)
{
    Simulation *sim = simulation_create(eqns, "");
    if (!strcmp(method, "lserk") && iparam) {
        RungeKutta rk = {iparam[0], iparam[1]};
        simulation_set_advance(sim, method, courant, &rk);
    }
    else if (!strcmp(method, "implicit euler") && dparam) {
        NewtonKrylov nk = {dparam[0], dparam[1], (int)dparam[2]};
        simulation_set_advance(sim, method, courant, &nk);
    }
    else {
        simulation_set_advance(sim, method, courant, 0);
    }
    return sim;
}

void ref_simulation_set_max_iter(void *sim, int iter)
{
    simulation_set_max_iter(sim, iter);
}

void ref_simulation_set_max_time(void *sim, double time)
{
    simulation_set_max_time(sim, time);
}

void ref_simulation_set_out_time(void *sim, double time)
{
    simulation_set_out_time(sim, time);
}

void ref_simulation_set_out_iter(void *sim, int iter)
{
    simulation_set_out_iter(sim, iter);
}

void ref_simulation_set_termination(void *sim, const char *condition, double threshold)
{
    simulation_set_termination(sim, condition, threshold);
}

double ref_simulation_run(void *sim)
{
    return simulation_run(sim);
}

/* one call of the configured Advance method, as simulation_run makes it (run.c:69-70) */
double ref_advance(void *sim_, double *time, double *residual, double max_step)
{
    Simulation *sim = sim_;
    return sim->advance.method(sim->eqns, time, residual, max_step, sim->advance.courant,
                               sim->advance.context);
}

void ref_simulation_destroy(void *sim)
{
    simulation_destroy(sim);
}

/* Nearest point of `point` [num][3] for each of `query` [num_query][3], with the reference's own kd-tree
 * (src/core/kdtree.c, the search teal's restart interpolation uses, src/equations/read.c:101-144). */
void ref_kdtree_nearest(const double *point, int num, const double *query, int num_query, int *index)
{
    Kdtree *tree = kdtree_init((const Vector *)point, num);
    for (int i = 0; i < num_query; i++) {
        Vector q = {query[3 * i], query[3 * i + 1], query[3 * i + 2]};
        index[i] = -1;
        kdtree_nearest(tree, q, &index[i], 1);
    }
    kdtree_deinit(tree);
}
