// Device-resident mesh and state layout of one teal_b200 context, and the kernel entry points.
//
// Index spaces
//   inner cells      [0, C)            teal's cells [0, num_inner)
//   boundary ghosts  [C, N)            teal's cells [num_inner, off_boundary): state rows only
//   periodic ghosts  -                 not stored: every reference is redirected to the owner cell
//   faces            [0, F)            teal's face order: two-sided inner faces [0, F_in), one-sided
//                                      boundary faces [F_in, F_bd), one-sided periodic faces [F_bd, F)
// Per-cell face lists ("slots") are ELL-packed: slot j of cell c lives at [j * C + c], j < 6,
// sorted by face index so every per-cell sum runs in teal's face order.
#pragma once

#include <cstdint>

#include "physics.cuh"

namespace tg {

constexpr int MAX_SLOTS = 6;  // teal's MAX_CELL_FACES (src/mesh.h:7-11)
constexpr int MAX_BOUNDARIES = 16;

// geometry and connectivity; `G` is the geometry element type (double, or float for the FP32
// flux form, which keeps its own copies)
template <typename G>
struct Geometry {
    const int2 *lr;       // [F] left, right (right redirected to the owner for periodic faces)
    const G *area;        // [F]
    const G *basis;       // [9][F] rows x, y, z
    const G *offl;        // [3][F] face centre - left centre
    const G *offr;        // [3][F] face centre - right centre (teal's ghost centre for ghosts)
    const G *corr;        // [4][F] unit vector left->right centre, distance (Navier–Stokes)
    const int *slot_nbr;  // [6][C] neighbour state row
    const int *slot_face; // [6][C] face index f (cell is left) or ~f (cell is right)
    const uint8_t *slot_cnt; // [C]
    const G *slot_w;      // [3][6][C] least-squares weight of this cell's side
    const G *slot_off;    // [3][6][C] face centre - cell centre (limiter)
};

struct CellData {
    const double *volume;     // [C]
    const double *projection; // [3][C]
    const double *eps2;       // [C] Venkatakrishnan parameter (or null)
};

struct BoundaryTable {
    int num;
    int kind[MAX_BOUNDARIES];
    double ctx[MAX_BOUNDARIES][5];
};

struct Sizes {
    int C, N, F, F_in, F_bd;
};

// step bookkeeping kept on the device so a whole step can be replayed from a CUDA graph
struct StepState {
    double time;
    double step;       // step of the current / last step (after clipping)
    double step0;      // unclipped step of the current / last step
    double max_step;   // clip for the next step (tg_advance)
    double max_time;   // clip time for the next step (tg_run)
    double residual[5];
    int use_max_time;
    int error;         // nonzero once a non-finite norm or step was seen
};

}  // namespace tg
