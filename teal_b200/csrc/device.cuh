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
    const int *slot_nbr;  // [6][SL] neighbour state row
    const int *slot_face; // [6][SL] face index f (cell is left) or ~f (cell is right)
    const uint8_t *slot_cnt; // [C]
    // gradient tiles: the slot geometry of 32 consecutive cells in one contiguous block (see
    // grad_tile_bytes), as many slots as the tile's cell with the most faces has
    const unsigned char *gtile;
    const long long *gtile_off;  // [tiles + 1] byte offset of each tile
};

// One gradient tile of J slots for element type G: neighbour rows [J][32] int, least-squares
// weights [J][3][32] G (slot j, component d at row 3 j + d), face offsets [J][3][32] G; every part
// a multiple of 16 bytes, so the three parts are bulk copies of their own.
template <typename G>
__host__ __device__ constexpr long long grad_tile_nbr_bytes(int J)
{
    return (long long)J * 32 * sizeof(int);
}
template <typename G>
__host__ __device__ constexpr long long grad_tile_vec_bytes(int J)
{
    return (long long)J * 3 * 32 * sizeof(G);
}
template <typename G>
__host__ __device__ constexpr long long grad_tile_bytes(int J)
{
    return grad_tile_nbr_bytes<G>(J) + 2 * grad_tile_vec_bytes<G>(J);
}

struct CellData {
    const double *volume;     // [C]
    const double *projection; // [3][C]
    const double *eps2;       // [C] Venkatakrishnan parameter (or null)
};

struct Sizes {
    int C, N, F, F_in, F_bd;
    int SL;  // leading dimension of the per-cell slot arrays: C rounded up to 4 (16-byte rows)
    // work range of one launch of the gradient, face and cell kernels, which a step whose host copies
    // overlap its kernels splits in chunks: cells [lo, hi) (gradient: lo a multiple of 32; cell
    // kernel) or faces [lo, hi) (face kernels); the launchers set it, [0, C) / [0, F) when unsplit
    int lo, hi;
};

// Instances packed in one arena (a single mesh is one instance). Inner cells of instance i are
// [inst_cell_off[i], inst_cell_off[i+1]); reductions run over "pieces", cell ranges of at most
// PIECE cells that never straddle two instances, first per piece, then per instance in piece order.
constexpr int PIECE = 4096;

struct Segments {
    int ninst;
    int npieces;
    const int *cell_inst;      // [C]
    const int *inst_cell_off;  // [ninst + 1]
    const int *piece_beg;      // [npieces + 1]
    const int *inst_piece_off; // [ninst + 1]
    const double *sum_volume;  // [ninst]
};

// Per-instance step bookkeeping in device memory, so whole steps replay from a CUDA graph and
// instances stop on their own (max iterations, residual threshold, end time).
struct Steps {
    double *time;
    double *step;      // step of the current / last step (after clipping)
    double *step0;     // unclipped step of the current / last step
    double *max_step;  // clip of the next step (one Advance call)
    double *max_time;  // end time (run loops)
    double *threshold; // residual threshold (<= 0: none)
    double *residual;  // [ninst][5]
    int *variable;     // residual variable tested (-1: the maximum)
    int *iter;
    int *max_iter;
    int *active;       // updates and clocks of an inactive instance stand still
    int *fail;         // nonzero once the instance's time step or residual was non-finite (it stops)
    int *num_active;   // active instances after the last step
    int *error;        // nonzero once a non-finite step or norm was seen
    int use_max_time;  // clip by max_time - time instead of max_step
};

}  // namespace tg
