/*
 * teal_b200 — C ABI of the B200 (sm_100a) residual / time-integration path of the teal
 * finite-volume solver (compressible Euler and Navier–Stokes on unstructured meshes).
 *
 * Plain pointers and sizes only. Every array argument uses teal's own host layout (AoS doubles,
 * `int` pairs) so a teal program can hand its `Mesh` / `Equations` arrays over unchanged; the
 * library owns the device copies and never frees caller memory. All functions return TG_OK (0) or
 * a nonzero TG_ERR_* status; `tg_last_error()` gives the message (teal itself exits through
 * `teal_error`, src/core/teal.c:134-144; a host wrapper maps a nonzero status onto that).
 *
 * Reference interfaces replaced (paths inside the teal source tree):
 *   tg_mesh               <- Mesh arrays produced by mesh_create + mesh_generate (src/mesh.h:13-72)
 *   tg_equations          <- Equations plugin table selected by name (src/equations.h:97-111)
 *   tg_derivative         <- equations_derivative (src/equations.h:175; equations/derivative.c:269)
 *   tg_gradient           <- equations_gradient (+ equations_limiter) (src/equations.h:169-172)
 *   tg_timestep           <- equations_timestep (src/equations.h:163; equations/timestep.c:7)
 *   tg_residual           <- equations_residual (src/equations.h:178; equations/residual.c:8)
 *   tg_advance            <- Advance methods euler / lserk / implicit_euler (src/simulation.h:6-7;
 *                            simulation/advance.c:11-195, simulation/gmres.c:52-149)
 *   tg_teal_{euler,lserk,implicit_euler}
 *                         <- the same, with teal's exact `Advance` signature, for installing into
 *                            `Simulation.advance.method` (src/simulation.h:36-41)
 *   tg_run                <- simulation_run's step loop with the state resident on the device
 *                            (simulation/run.c:22-113)
 */
#ifndef TEAL_B200_H
#define TEAL_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ----------------------------------------------------------------------------- */
enum {
    TG_OK = 0,
    TG_ERR_INVALID = 1,    /* bad argument, unsupported plugin name or mesh layout */
    TG_ERR_CUDA = 2,       /* CUDA runtime failure (message has the CUDA error string) */
    TG_ERR_OOM = 3,        /* device allocation failed */
    TG_ERR_NONFINITE = 4,  /* a non-finite value reached the state or a norm */
    TG_ERR_TIMEOUT = 5,    /* a bounded device-side wait gave up */
    TG_ERR_NO_DEVICE = 6   /* no CUDA device / the library was built without one in reach */
};

/* ---- plugin kinds (selected by teal's names; see the *_select functions) ----------------------- */
enum { TG_EULER = 0, TG_NAVIERSTOKES = 1 };

/* convective fluxes of euler_convective (src/euler/convective.c:593-623); godunov is rejected */
enum {
    TG_FLUX_NONE = 0,
    TG_FLUX_ROE = 1,
    TG_FLUX_HLL = 2,
    TG_FLUX_HLLC = 3,
    TG_FLUX_HLLE = 4,
    TG_FLUX_AUSMD = 5,
    TG_FLUX_AUSMDV = 6,
    TG_FLUX_LXF = 7,
    TG_FLUX_CENTRAL = 8
};

/* viscous fluxes of navierstokes_viscous (src/navierstokes/viscous.c:41-47) */
enum { TG_VISCOUS_NONE = 0, TG_VISCOUS_CENTRAL = 1 };

/* limiter kinds, same numbering as teal's LimiterKind (src/equations/limiter.h:5-9) */
enum { TG_LIMITER_NONE = 0, TG_LIMITER_BARTH_JESPERSEN = 1, TG_LIMITER_VENKATAKRISHNAN = 2 };

/* boundary conditions of euler_boundary / navierstokes_boundary
 * (src/euler/boundary.c:273-297, src/navierstokes/boundary.c:20-26) */
enum {
    TG_BC_SYMMETRY = 1, /* "symmetry", "slipwall" */
    TG_BC_SUPERSONIC_INFLOW = 2,
    TG_BC_SUPERSONIC_OUTFLOW = 3,
    TG_BC_SUBSONIC_INFLOW = 4,
    TG_BC_SUBSONIC_OUTFLOW = 5,
    TG_BC_PRESSURE_OUTFLOW = 6,
    TG_BC_FARFIELD = 7,
    TG_BC_ADIABATIC_WALL = 8, /* "adiabatic wall", "wall" (Navier–Stokes only) */
    TG_BC_CUSTOM = 9          /* "custom": teal's Compute callback (src/equations/boundary.c:27-33) as
                                 a registered device function, tg_bind_boundary_function */
};

/* Source terms run on the device (teal's Equations.source, src/equations.h:27-41, is a host
 * callback pair; the device runs these kinds in its place, selected by tg_source_select):
 *   TG_SOURCE_BODY_FORCE    constant acceleration g = source_parameter[0..2]:
 *                           S = (0, rho g, rho g . u)   (run/rayleigh_taylor_instability/run.c:17-24)
 *   TG_SOURCE_BULK_FORCING  forcing of the bulk x velocity to U = source_parameter[0] with time
 *                           scale tau = source_parameter[1]: s = rho (U - <u_x>) / tau,
 *                           S = (0, s, 0, 0, u_x s), <u_x> the volume average over the inner cells of
 *                           the state being differentiated (run/periodic_hill/run.c:8-21) */
enum { TG_SOURCE_NONE = 0, TG_SOURCE_BODY_FORCE = 1, TG_SOURCE_BULK_FORCING = 2, TG_SOURCE_DEVICE = 3 };
/*   TG_SOURCE_DEVICE        teal's source Compute callback (src/equations/derivative.c:242-266) as a
 *                           registered device function, tg_bind_source_function */

/* time integrators of simulation_set_advance (src/simulation/set.c:74-131) */
enum { TG_ADVANCE_EULER = 0, TG_ADVANCE_LSERK = 1, TG_ADVANCE_IMPLICIT_EULER = 2 };

/* arithmetic of the face-flux path:
 *   TG_PRECISION_FP64        plain FP64; quotients that share a denominator take one reciprocal and
 *                            multiply-adds are contracted: within a few ulps of teal per operation
 *   TG_PRECISION_FP32_FLUX   FP32 gradients/limiter/fluxes with FP64 accumulation, state update and
 *                            Krylov arithmetic
 *   TG_PRECISION_FP64_EXACT  FP64 with teal's own operations in teal's order (every quotient a
 *                            division, no contraction, the viscous face terms of a cell summed before
 *                            the convective ones as in derivative.c:279-292): residuals, gradients,
 *                            time steps and explicit steps equal teal's bit for bit; slower than
 *                            TG_PRECISION_FP64 (two flux records per face with a viscous flux) */
enum { TG_PRECISION_FP64 = 0, TG_PRECISION_FP32_FLUX = 1, TG_PRECISION_FP64_EXACT = 2 };

/* Return the kind for a teal plugin name, or -1 when teal has no such name or this library does not
 * run it on the device (then teal would call teal_error). */
int tg_convective_select(const char *name);
int tg_viscous_select(const char *name);
int tg_limiter_select(const char *name);
int tg_boundary_select(const char *name, int physics);
int tg_advance_select(const char *name);
int tg_source_select(const char *name); /* "body force", "bulk forcing" */

/* ---- mesh: teal's Mesh arrays (src/mesh.h:13-72), one process ---------------------------------- */
typedef struct {
    /* MeshCells */
    int num_cells;          /* inner + boundary ghosts + periodic ghosts */
    int num_inner_cells;
    int off_boundary_cells; /* first periodic ghost */
    int off_periodic_cells; /* first neighbour-rank ghost (== num_cells on one process) */
    const int *cell_cell_off;      /* [num_cells + 1] CSR of face neighbours */
    const int *cell_cell_idx;      /* [cell_cell_off[num_cells]] */
    const double *cell_volume;     /* [num_cells] */
    const double *cell_center;     /* [num_cells][3] */
    const double *cell_projection; /* [num_cells][3] */
    const double *cell_offset;     /* [cell_cell_off[num_inner_cells]][3] */
    double sum_volume;
    /* MeshFaces */
    int num_faces; /* inner (two-sided) + boundary + periodic (one-sided copies) */
    int num_inner_faces;
    int off_boundary_faces;
    const int *face_cell;          /* [num_faces][2] left, right */
    const double *face_area;       /* [num_faces] */
    const double *face_basis;      /* [num_faces][3][3] rows: normal, tangent, tangent */
    const double *face_weight;     /* [num_faces][2][3] LS weights of the left / right cell */
    const double *face_offset;     /* [num_faces][2][3] face centre minus left / right centre */
    const double *face_correction; /* [num_faces][4] unit vector left->right centre, distance */
    /* MeshEntities */
    int num_entities;
    int num_inner_entities;
    int off_boundary_entities;
    const int *entity_face_off; /* [num_entities + 1] */
    /* MeshNeighbors (periodic self-exchange on one process) */
    int num_neighbors;
    const int *neighbor_tag;      /* [num_neighbors][2] receive tag, send tag */
    const int *neighbor_recv_off; /* [num_neighbors + 1] ghost cell ranges */
    const int *neighbor_send_off; /* [num_neighbors + 1] */
    const int *neighbor_send_idx; /* [neighbor_send_off[num_neighbors]] inner cells sent */
} tg_mesh;

/* ---- equations: the Equations plugin table, by kind (src/equations.h:97-111) -------------------- */
typedef struct {
    int physics;     /* TG_EULER / TG_NAVIERSTOKES */
    int space_order; /* 1 or 2 */
    int convective;  /* TG_FLUX_* */
    int viscous;     /* TG_VISCOUS_* (Navier–Stokes only) */
    int limiter;     /* TG_LIMITER_* */
    /* Venkatakrishnan eps^2 per inner cell (teal's limiter.parameter); null = computed from
     * limiter_coefficient as teal does (src/equations/limiter.c:8-21) */
    const double *limiter_parameter;
    double limiter_coefficient;
    double property[3]; /* heat capacity ratio, dynamic viscosity, Prandtl number */
    int num_boundaries; /* off_boundary_entities - num_inner_entities */
    const int *boundary_kind;       /* [num_boundaries] TG_BC_* */
    const double *boundary_context; /* [num_boundaries][5] primitive state (may be null) */
    int source;                     /* TG_SOURCE_* */
    double source_parameter[4];     /* see TG_SOURCE_* */
} tg_equations;

/* contexts of the Advance methods, teal's layouts (src/simulation.h:25-34) */
typedef struct {
    int time_order;
    int num_stages;
} tg_runge_kutta;

typedef struct {
    double newton_tolerance;
    double krylov_tolerance;
    int krylov_dimension;
} tg_newton_krylov;

/* ---- context lifecycle ------------------------------------------------------------------------- */
typedef struct tg_ctx tg_ctx;

/* Upload mesh + equations to the current CUDA device: structure-of-arrays geometry, periodic ghost
 * -> owner redirection, per-cell face lists in face order. Host arrays may be freed afterwards. */
int tg_create(const tg_mesh *mesh, const tg_equations *eqns, int precision, tg_ctx **ctx);
int tg_destroy(tg_ctx *ctx);

/* Thread-local message of the last failing call on this thread. */
const char *tg_last_error(void);

/* Run all device work of this context on `stream` (a cudaStream_t; null = the context's own). */
int tg_set_stream(tg_ctx *ctx, void *stream);

/* Failure-detection control, no counterpart in teal. Every device-side wait of this context (the
 * gradient kernel's and the staged face kernel's waits for their bulk copies of slot and face
 * geometry) tries at most `polls` times, each try suspending the thread for up to about a
 * microsecond, before it gives up; the call then returns TG_ERR_TIMEOUT, the blocks that gave up
 * first let their copies land, and the context stays usable. Default and maximum 1048576 tries
 * (about a second); 0 makes every such wait give up at once, which is how the timeout path is
 * tested without a fault. */
int tg_set_wait_limit(tg_ctx *ctx, int polls);

/* Resident primitive state: [num_cells][5] in teal's cell order (density, velocity, pressure).
 * set: reads inner cells (ghost rows are ignored). get: writes inner cells, boundary ghosts as the
 * last boundary pass left them, and periodic ghosts as copies of their owners. */
int tg_set_primitive(tg_ctx *ctx, const double *primitive);
int tg_get_primitive(tg_ctx *ctx, double *primitive);

/* equations_derivative: boundary pass, gradient, limiter, viscous and convective fluxes, finalize.
 * primitive: [num_cells][5] host array (inner rows are read; null = the resident state, whose
 * boundary ghost rows are refreshed); a host-given state is evaluated in scratch memory and leaves
 * the resident state unchanged. derivative: [num_inner][5]. */
int tg_derivative(tg_ctx *ctx, const double *primitive, double *derivative, double time);

/* equations_gradient (+ equations_limiter when `limited`) of the resident state after a boundary
 * pass: gradient [num_inner][5][3]. */
int tg_gradient(tg_ctx *ctx, double time, int limited, double *gradient);

/* equations_timestep of the resident state (minimum stable step, before the Courant factor). */
int tg_timestep(tg_ctx *ctx, double *step);

/* equations_residual of a derivative [num_inner][5] given on the host -> residual[5]. */
int tg_residual(tg_ctx *ctx, const double *derivative, double *residual);

/* One Advance step on the resident state: method TG_ADVANCE_*, context tg_runge_kutta /
 * tg_newton_krylov (null = teal's defaults). Returns the unclipped step in *step0 and advances
 * *time by min(step0, max_step); residual[5] gets equations_residual of the last derivative. */
int tg_advance(tg_ctx *ctx, int method, const void *context, double courant, double *time,
               double max_step, double *residual, double *step0);

/* tg_set_primitive(prim_in) + tg_advance + tg_get_primitive(prim_out) as one call, with the
 * download overlapped with the step's last stage (explicit methods on a single mesh, prim_out in
 * pinned or registered host memory): that stage's face fluxes and cell updates run in chunks of
 * cells and each chunk's rows are copied to the host as soon as they are final. The results are
 * the bits of the three calls in sequence. prim_in (its first num_inner rows of 5) or null (the
 * resident state), prim_out [num_cells][5] or null. Pageable prim_out, the implicit method and
 * partitions run the three calls in sequence. The first chunked call builds the context's chunk plan
 * (one host pass over the faces). This is the work of teal's Advance (src/simulation.h:6-7) on
 * eqns->primitive.data, which the drop-in methods (tg_teal_*) call. */
int tg_advance_host(tg_ctx *ctx, int method, const void *context, double courant, double *time,
                    double max_step, const double *prim_in, double *prim_out, double *residual, double *step0);

/* Unclipped step (step0) of the last step taken by `instance` (0 for a single mesh), as teal's run
 * loop prints it (simulation/run.c:95-96). */
int tg_last_step(tg_ctx *ctx, int instance, double *step0);

/* simulation_run's loop with the state resident: up to max_iter steps or until max_time, or until
 * the residual of `variable` (-1 = maximum) drops below `threshold` (threshold <= 0: never).
 * Steps are replayed from CUDA graphs; the host synchronises only when it must test the residual.
 * On return *time and *iter hold the end state, residual[5] the last residual. */
int tg_run(tg_ctx *ctx, int method, const void *context, double courant, int max_iter,
           double max_time, int variable, double threshold, double *time, int *iter,
           double *residual);

/* ---- batches: several meshes packed into one device arena ---------------------------------------
 * Instances share the equations, schemes and properties (one "lane"); boundary conditions,
 * Venkatakrishnan parameters and states differ per instance. The arena keeps all inner cells first
 * (instance order), then all boundary ghosts; faces likewise, so every kernel runs once over all
 * instances. Each instance keeps its own time step (CFL over its own cells), time, residual norm
 * and stop tests, exactly as if it ran alone; the whole batch step replays from one CUDA graph. */
int tg_batch_create(const tg_mesh *meshes, const tg_equations *eqns, int num, int precision, tg_ctx **ctx);
int tg_batch_size(tg_ctx *ctx, int *num);
int tg_batch_set_primitive(tg_ctx *ctx, int instance, const double *primitive);
int tg_batch_get_primitive(tg_ctx *ctx, int instance, double *primitive);
/* Run every instance until its own limit: max_iter[i] steps, max_time[i] (null: none), or the
 * residual of variable[i] (-1: maximum; null: all -1) below threshold[i] (null or <= 0: none).
 * time[i] is read and updated; iter[i] and residual[i][5] return the end state. Every method
 * (explicit, and implicit Euler with each instance's own Newton-GMRES). An instance whose time step
 * or residual becomes non-finite stops on its own while the others go on (a single-mesh context
 * returns TG_ERR_NONFINITE instead): tg_batch_status reports it, and it stays stopped until
 * tg_batch_set_primitive gives it a new state. */
int tg_batch_run(tg_ctx *ctx, int method, const void *context, double courant, const int *max_iter,
                 const double *max_time, const int *variable, const double *threshold, double *time,
                 int *iter, double *residual);
/* status[i] = TG_OK, or TG_ERR_NONFINITE for an instance that stopped on a non-finite value. No
 * counterpart in teal (one mesh per process there). */
int tg_batch_status(tg_ctx *ctx, int *status);

/* ---- partitions: one rank's share of a mesh (several GPUs) ---------------------------------------
 * teal decomposes a mesh over MPI ranks and exchanges one layer of ghost cells (src/equations/
 * exchange.c:8-51, src/mesh/create.c:351-440). A partition here is the same idea for one GPU per
 * rank: `mesh` holds the rank's inner cells [0, C), the boundary ghosts of its boundary faces
 * [C, off_boundary) and the periodic ghosts of its periodic faces [off_boundary, num_cells), and
 * the global mesh's faces that touch its inner cells, in global order and orientation. An inner
 * face may reference a halo row, off_boundary + h for h < num_halo: an inner cell of another rank.
 * owner[p] is the state row (an inner cell or a halo row) whose state periodic ghost off_boundary + p
 * takes; send_rows are the inner cells whose states and gradient records other ranks' halos receive.
 * mesh->sum_volume is the whole mesh's. Explicit methods only; no source terms or custom boundaries.
 * Every rank's own cells then sum their faces in the global order, and a face shared by two ranks
 * is computed on both from the same inputs: the state after a step equals the single-mesh run's. */
int tg_create_partition(const tg_mesh *mesh, const tg_equations *eqns, int precision, const int *owner,
                        int num_halo, const int *send_rows, int num_send, tg_ctx **ctx);
/* Device pointers of the exchange buffers: states send_q[num_send][5] and recv_q[num_halo][5]
 * (FP64), gradient records send_rec[num_send] and recv_rec[num_halo] of *record_bytes each. The
 * caller moves send data into the receiving ranks' recv buffers in their halo order. */
int tg_part_buffers(tg_ctx *ctx, void **send_q, void **recv_q, void **send_rec, void **recv_rec,
                    long *record_bytes);
/* A step: tg_part_step_begin gives the minimum stable step of this rank's cells (equations_timestep
 * over its share); the caller takes the minimum over ranks, times the CFL number and clipped, and
 * sets it with tg_part_set_step; each RK stage runs tg_part_phase 0, 1, 2 with alpha_{i+1} (and
 * last on the final stage), exchanging states after phase 0 and records after phase 1 (phase 0
 * packs, phase 1 and 2 unpack first); tg_part_residual_sums gives this rank's sums of V R^2 of the
 * last stage (the norm is sqrt of their sum over ranks divided by the total volume). The context's
 * stream (tg_stream_of) orders everything; the host functions that return values synchronise it. */
int tg_part_step_begin(tg_ctx *ctx, double *local_min);
int tg_part_set_step(tg_ctx *ctx, double step, double time);
int tg_part_phase(tg_ctx *ctx, int phase, double alpha, int last);
int tg_part_residual_sums(tg_ctx *ctx, double *sums);
int tg_stream_of(tg_ctx *ctx, void **stream);
/* teal's low-storage RK coefficients alpha[0..stages] (src/simulation/advance.c:50-75) */
int tg_lserk_alpha(int order, int stages, double *alpha);

/* ---- drop-in Advance methods with teal's signature (src/simulation.h:6-7) ----------------------- */

/* Bind a teal `Equations *` (used only as a lookup key) to a single-mesh context and to the host
 * primitive array teal reads (`eqns->primitive.data`, [num_cells][5]). The host state is uploaded
 * now; every drop-in Advance call copies the new state back into that array while its last stage
 * runs (tg_advance_host). A pageable array is page-locked in place (cudaHostRegister) until
 * tg_unbind, which must come before teal frees it (equations_destroy). */
int tg_bind(const void *eqns, tg_ctx *ctx, double *host_primitive);
int tg_unbind(const void *eqns);

/* On failure these print tg_last_error() to stderr and exit(EXIT_FAILURE), as teal_error does. */
double tg_teal_euler(const void *eqns, double *time, void *residual, double max_step,
                     double courant, const void *context);
double tg_teal_lserk(const void *eqns, double *time, void *residual, double max_step,
                     double courant, const void *context);
double tg_teal_implicit_euler(const void *eqns, double *time, void *residual, double max_step,
                              double courant, const void *context);

/* ---- host mesh generation (the single-process Cartesian case of mesh_create + mesh_generate,
 *      src/mesh/create.c:509-544, src/mesh/generate.c:779-815) ---------------------------------- */
typedef struct tg_host_mesh tg_host_mesh;

/* Build a Cartesian hex box [min, max] with num cells per axis and per-axis periodicity; node
 * displacement (optional, [(nx+1)(ny+1)(nz+1)][3], node order x fastest) is added before the
 * geometry is generated, as mesh_modify would. */
int tg_host_mesh_cartesian(const double *min_coord, const double *max_coord, const int *num_cells,
                           const int *periodic, const double *displacement, tg_host_mesh **mesh);
/* Generate a single-process mesh given as nodes, cells and entities, as teal holds it between
 * mesh_read (src/mesh/read.c) and mesh_generate: coord [num_nodes][3]; cells as node lists in CSR
 * (node_off [num_cells + 1], node_idx), first num_inner_cells volume cells (tetrahedron 4,
 * pyramid 5, prism 6, hexahedron 8 nodes, Gmsh order), then boundary face cells (3 or 4 nodes);
 * entities as names and cell ranges (entity_cell_off [num_entities + 1]): the inner entities
 * first, then one entity per boundary. No periodic entities. */
int tg_host_mesh_cells(int num_nodes, const double *coord, int num_cells, int num_inner_cells,
                       const int *node_off, const int *node_idx, int num_entities,
                       const char *const *entity_names, const int *entity_cell_off, tg_host_mesh **mesh);
/* The same with periodic entities, as mesh_read leaves a mesh with periodic links on one process
 * (src/mesh/read.c:294-372): after the boundary face cells [num_inner_cells, off_boundary_cells)
 * the periodic face cells [off_boundary_cells, num_cells), one entity per periodic surface after
 * the boundary entities (off_boundary_entities), each with its rotation [9] (rows) and translation
 * [3] (entity_rotation [num_entities][9], entity_translation [num_entities][3]: owner side to ghost
 * side, read.c via gmsh.c:784-817), and the self-exchange of the periodic ghosts: num_neighbors
 * entries of (receive tag, send tag) (neighbor_tag [num_neighbors][2]), ghost row ranges
 * (neighbor_recv_off [num_neighbors + 1], from off_boundary_cells) and the inner cells each entry
 * sends (neighbor_send_off [num_neighbors + 1], neighbor_send_idx), matched by tag as
 * equations/exchange.c:8-51 does on one rank. */
int tg_host_mesh_cells_periodic(int num_nodes, const double *coord, int num_cells, int num_inner_cells,
                                int off_boundary_cells, const int *node_off, const int *node_idx, int num_entities,
                                int off_boundary_entities, const char *const *entity_names,
                                const int *entity_cell_off, const double *entity_rotation,
                                const double *entity_translation, int num_neighbors, const int *neighbor_tag,
                                const int *neighbor_recv_off, const int *neighbor_send_off,
                                const int *neighbor_send_idx, int num_splits, const char *const *split_entity,
                                const double *split_root, const double *split_normal, tg_host_mesh **mesh);
/* tg_host_mesh_cartesian with teal's mesh_split (src/mesh/split.c) applied before generation, in
 * order: split i cuts the inner or boundary entity split_entity[i] by the plane through
 * split_root[i][3] with normal split_normal[i][3] into "<name>-a" (cell node means on the
 * non-positive side) and "<name>-b". tg_host_mesh_cells_periodic takes the same split lists. */
int tg_host_mesh_cartesian_split(const double *min_coord, const double *max_coord, const int *num_cells,
                                 const int *periodic, const double *displacement, int num_splits,
                                 const char *const *split_entity, const double *split_root,
                                 const double *split_normal, tg_host_mesh **mesh);
/* View of the generated arrays (pointers stay owned by the host mesh). */
int tg_host_mesh_view(const tg_host_mesh *mesh, tg_mesh *view);
/* Entity names (teal's: "domain", "left", "right", ...) and their cell ranges. */
int tg_host_mesh_entity(const tg_host_mesh *mesh, int index, const char **name, int *cell_beg,
                        int *cell_end);
/* Nodes and cell node lists (pointers stay owned by the host mesh): coord [num_nodes][3], the node
 * list of cell i at cell_node_idx[cell_node_off[i] .. cell_node_off[i + 1]) in teal's cell order
 * (Gmsh node order), inner cells first; what teal's VTKHDF writer outputs (src/mesh/write.c). */
int tg_host_mesh_nodes(const tg_host_mesh *mesh, int *num_nodes, const double **coord,
                       const int **cell_node_off, const int **cell_node_idx);
int tg_host_mesh_destroy(tg_host_mesh *mesh);

/* ---- measurement -------------------------------------------------------------------------------
 * tg_profile: reset the per-kernel timers and enable (1) or disable (0) CUDA-event timing of every
 * hot-path launch; while enabled, steps run as plain launches instead of graph replays.
 * tg_profile_read: accumulated milliseconds and launch counts per category TG_PROF_*.
 * tg_launch_count: kernels this context has launched on its hot path (graph replays included). */
enum {
    TG_PROF_BOUNDARY = 0,
    TG_PROF_GRADIENT = 1,
    TG_PROF_FACE = 2,
    TG_PROF_CELL = 3,
    TG_PROF_REDUCE = 4,
    TG_PROF_CATEGORIES = 5
};
int tg_profile(tg_ctx *ctx, int enable);
int tg_profile_read(tg_ctx *ctx, double *ms, long *launches);
int tg_launch_count(tg_ctx *ctx, long *count);

/* ---- device layout introspection (tests of the device upload) --------------------------------
 * Copy a device layout array to `out` (count elements of the named array's type):
 *   "face_lr"   int[num_faces][2]  left, right with periodic ghosts redirected to their owners
 *   "slot_face" int[6][num_inner]  face f (cell is left) or ~f (cell is right), sorted by face
 *   "slot_nbr"  int[6][num_inner]  neighbour state row of each slot (padding: the cell itself)
 *   "slot_cnt"  uint8[num_inner]   faces per cell
 *   "owner"     int[num periodic ghosts]  owner cell of each periodic ghost
 * Returns TG_ERR_INVALID for an unknown name or a count that does not match. */
int tg_layout(tg_ctx *ctx, const char *name, void *out, long count);

/* ---- residual norm with no device allocation -----------------------------------------------------
 * No counterpart in the reference. It computes what equations_residual does (equations/residual.c:8),
 * residual[k] = sqrt(sum_c volume[c] * derivative[c][k]^2 / sum_volume), for a derivative that is
 * already on the device, without a context and without allocating device memory. It is meant for
 * callers that cannot allocate while they solve: a server that committed its whole HBM budget to
 * state arenas up front, or a host loop that must not stall the device (cudaMalloc and cudaFree
 * can synchronise it).
 *   derivative  device double[num_cells][5] (teal's row layout)
 *   volume      device double[num_cells]
 *   sum_volume  the divisor (teal's mesh->cell.sum_volume), finite and > 0, else TG_ERR_INVALID
 *   residual    device double[5], written on `stream` (a cudaStream_t; null = legacy default)
 * All three buffers must be 8-byte aligned memory of the current device, or managed memory, else
 * TG_ERR_INVALID (memory of another GPU is refused before any launch).
 * The partial sums go to a fixed 640 KiB array compiled into the library, one per device, which
 * limits num_cells to TG_NOALLOC_MAX_CELLS; a larger num_cells returns TG_ERR_INVALID.
 * The first call on each device does a set-up (it looks up that array's device address, which can
 * initialise the device's CUDA context); make that first call before any stream capture. The
 * address is kept for the life of the process: do not cudaDeviceReset a device after calling this
 * on it.
 * Calls that overlap in time on the same device (other streams, other host threads) share the
 * array and race: serialise them. The result equals tg_residual's on the same derivative. */
#define TG_NOALLOC_MAX_CELLS 67108864
int tg_residual_noalloc(const double *derivative, const double *volume, int num_cells, double sum_volume,
                        double *residual, void *stream);

/* ---- version / build info ---------------------------------------------------------------------- */
const char *tg_build_info(void);

/* ---- device functions: teal's host Compute callbacks (src/equations.h:27-41) as CUDA C --------- */
/* kinds of device function */
enum { TG_FUNCTION_BOUNDARY = 1, TG_FUNCTION_SOURCE = 2 };

/* Register `source`, CUDA C that defines
 *   __device__ void <name>(double *out, const double *property, const double *center, double time,
 *                          const double *context)
 * with the arguments teal passes its Compute callback: out = the ghost cell's primitive state
 * (boundary; it holds the ghost row's current values on entry, as teal's in-place call does) or the
 * cell's source in conserved variables (source; zero on entry); property = the equations'
 * properties (heat capacity ratio, then dynamic viscosity and Prandtl number for Navier-Stokes);
 * center = the ghost cell's centre (boundary) or the cell's centre (source), 3 doubles; time = the
 * time of the residual being evaluated (teal's stage time); context = the inner cell's primitive
 * state (boundary) or the cell's primitive state (source), 5 doubles; a source bound with
 * TG_PREPARE_AVERAGE finds 5 more after them (tg_bind_source_prepare). The function is compiled at
 * once with NVRTC for sm_100a without FMA contraction (libnvrtc is loaded at run time, no device
 * needed); a compile error returns TG_ERR_INVALID with the compiler log in `log` (`log_size` bytes,
 * may be null). A second registration of a name replaces the first for later bindings. */
int tg_function_register(const char *name, int kind, const char *source, char *log, long log_size);

/* Use the registered boundary function `name` for boundary `boundary` (the index into
 * tg_equations.boundary_kind, whose kind must be TG_BC_CUSTOM). One-mesh contexts only; every
 * custom boundary must be bound before the first residual. */
int tg_bind_boundary_function(tg_ctx *ctx, int boundary, const char *name);

/* Use the registered source function `name` (tg_equations.source must be TG_SOURCE_DEVICE). One-mesh
 * contexts only. */
int tg_bind_source_function(tg_ctx *ctx, const char *name);

/* teal's source Prepare (src/equations.h:40-41, called before the source of every cell,
 * src/equations/derivative.c:248-250) for a device source: TG_PREPARE_NONE (the default) or
 * TG_PREPARE_AVERAGE, the pass of run/periodic_hill/run.c:8-11, equations_average over the inner
 * cells (src/equations/average.c:8-40): the volume average of the primitive state being
 * differentiated, sum of V_c q_c over the inner cells / their volume, summed in a fixed order. The
 * source function reads it as context[5..9], after the cell's own state (zeros without it). */
enum { TG_PREPARE_NONE = 0, TG_PREPARE_AVERAGE = 1 };
int tg_bind_source_prepare(tg_ctx *ctx, int prepare);

#ifdef __cplusplus
}
#endif

#endif /* TEAL_B200_H */
