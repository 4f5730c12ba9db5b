/*
 * CPU restatement of teal's residual / time-integration path. TEST INFRASTRUCTURE ONLY (the
 * oracle): tests and the CPU-baseline leg of bench.py use it as a checker; the product never links
 * it. Meshes and equations use the C ABI's descriptions (include/teal_b200.h). States are teal's
 * AoS arrays: primitive [num_cells][5] (ghost rows are written), derivative [num_inner][5].
 * Parity is pinned against the reference compiled from its own sources (oracle/_ref) and against
 * the golden vectors in tests/golden.
 */
#pragma once

#include "../include/teal_b200.h"

/* equations_derivative (src/equations/derivative.c:269-305) */
int oracle_derivative(const tg_mesh *mesh, const tg_equations *eqns, double *primitive,
                      double *derivative, double time);
/* equations_boundary + equations_gradient (+ equations_limiter): gradient [num_cells][5][3] */
int oracle_gradient(const tg_mesh *mesh, const tg_equations *eqns, double *primitive, int limited,
                    double *gradient);
/* equations_timestep (src/equations/timestep.c:7-30) */
double oracle_timestep(const tg_mesh *mesh, const tg_equations *eqns, const double *primitive);
/* equations_residual (src/equations/residual.c:8-33) */
void oracle_residual(const tg_mesh *mesh, const double *derivative, double *residual);
/* Advance methods (src/simulation/advance.c:11-195): advance *primitive by one step, return step0 */
double oracle_euler(const tg_mesh *mesh, const tg_equations *eqns, double *primitive, double *time,
                    double *residual, double max_step, double courant);
double oracle_lserk(const tg_mesh *mesh, const tg_equations *eqns, double *primitive, double *time,
                    double *residual, double max_step, double courant, int time_order,
                    int num_stages);
double oracle_implicit_euler(const tg_mesh *mesh, const tg_equations *eqns, double *primitive,
                             double *time, double *residual, double max_step, double courant,
                             double newton_tolerance, double krylov_tolerance,
                             int krylov_dimension);
