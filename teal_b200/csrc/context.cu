// Host side of teal_b200: device upload of teal's mesh / equations, kernel sequencing of
// equations_derivative and of the Advance methods, CUDA-graph replay of steps, and the C ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/teal_b200.h"
#include "functions.h"
#include "gmres.cuh"
#include "aux_kernels.cuh"
#include "launch.cuh"

using namespace tg;

// ---- errors ----------------------------------------------------------------------------------

static thread_local std::string g_error;

static int fail(int code, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

#define CU(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            return fail(e_ == cudaErrorMemoryAllocation ? TG_ERR_OOM : TG_ERR_CUDA, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(e_), __FILE__, __LINE__);                      \
        }                                                                                        \
    } while (0)

#define TRY(call)                                                                                \
    do {                                                                                         \
        int r_ = (call);                                                                         \
        if (r_ != TG_OK) {                                                                       \
            return r_;                                                                           \
        }                                                                                        \
    } while (0)

extern "C" const char *tg_last_error(void)
{
    return g_error.c_str();
}

// lets the library's other translation units report through tg_last_error
int tg_record_error(int code, const char *msg)
{
    return fail(code, "%s", msg);
}

extern "C" const char *tg_build_info(void)
{
    return "teal_b200 sm_100a " __DATE__;
}

// ---- plugin selection by teal's names ---------------------------------------------------------

extern "C" int tg_convective_select(const char *name)
{
    if (!name) return -1;
    static const struct {
        const char *n;
        int k;
    } t[] = {{"roe", TG_FLUX_ROE},     {"hll", TG_FLUX_HLL},       {"hllc", TG_FLUX_HLLC},
             {"hlle", TG_FLUX_HLLE},   {"ausmd", TG_FLUX_AUSMD},   {"ausmdv", TG_FLUX_AUSMDV},
             {"lxf", TG_FLUX_LXF},     {"central", TG_FLUX_CENTRAL}};
    for (auto &e : t) {
        if (!strcmp(name, e.n)) return e.k;
    }
    return -1;  // includes "godunov" (exact Riemann solver): not run on the device
}

extern "C" int tg_viscous_select(const char *name)
{
    if (name && !strcmp(name, "central")) return TG_VISCOUS_CENTRAL;
    return -1;
}

extern "C" int tg_limiter_select(const char *name)
{
    if (!name) return -1;
    if (!strcmp(name, "barth jespersen") || !strcmp(name, "minmod")) return TG_LIMITER_BARTH_JESPERSEN;
    if (!strcmp(name, "venkatakrishnan")) return TG_LIMITER_VENKATAKRISHNAN;
    return -1;
}

extern "C" int tg_boundary_select(const char *name, int physics)
{
    if (!name) return -1;
    if (physics == TG_NAVIERSTOKES && (!strcmp(name, "adiabatic wall") || !strcmp(name, "wall")))
        return TG_BC_ADIABATIC_WALL;
    if (!strcmp(name, "symmetry") || !strcmp(name, "slipwall")) return TG_BC_SYMMETRY;
    if (!strcmp(name, "supersonic inflow")) return TG_BC_SUPERSONIC_INFLOW;
    if (!strcmp(name, "supersonic outflow")) return TG_BC_SUPERSONIC_OUTFLOW;
    if (!strcmp(name, "subsonic inflow")) return TG_BC_SUBSONIC_INFLOW;
    if (!strcmp(name, "subsonic outflow")) return TG_BC_SUBSONIC_OUTFLOW;
    if (!strcmp(name, "pressure outflow")) return TG_BC_PRESSURE_OUTFLOW;
    if (!strcmp(name, "farfield")) return TG_BC_FARFIELD;
    if (!strcmp(name, "custom")) return TG_BC_CUSTOM;
    return -1;
}

extern "C" int tg_source_select(const char *name)
{
    if (!name) return -1;
    if (!strcmp(name, "body force")) return TG_SOURCE_BODY_FORCE;
    if (!strcmp(name, "bulk forcing")) return TG_SOURCE_BULK_FORCING;
    if (!strcmp(name, "device function")) return TG_SOURCE_DEVICE;
    return -1;
}

extern "C" int tg_advance_select(const char *name)
{
    if (!name) return -1;
    if (!strcmp(name, "euler")) return TG_ADVANCE_EULER;
    if (!strcmp(name, "lserk")) return TG_ADVANCE_LSERK;
    if (!strcmp(name, "implicit euler")) return TG_ADVANCE_IMPLICIT_EULER;
    return -1;
}

// ---- context ---------------------------------------------------------------------------------

template <typename T>
static int dalloc(T **p, size_t n)
{
    *p = nullptr;
    if (n == 0) n = 1;
    // 64 bytes of slack: bulk copies of a tile may read up to 15 bytes past the last element
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(T) + 64);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(TG_ERR_OOM, "cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
    }
    return TG_OK;
}

struct GeomBuf {
    double *area = nullptr, *basis = nullptr, *offl = nullptr, *offr = nullptr, *corr = nullptr;
    double *slot_w = nullptr, *slot_off = nullptr;  // pitched slot geometry (mesh upload only)
    float *area32 = nullptr, *basis32 = nullptr, *offl32 = nullptr, *offr32 = nullptr, *corr32 = nullptr;
    unsigned char *tile64 = nullptr, *tile32 = nullptr;  // gradient tiles, FP64 and FP32 geometry
    long long *toff64 = nullptr, *toff32 = nullptr;       // their byte offsets, [tiles + 1]
};

// workspace of the Jacobian-free Newton-GMRES implicit step
struct Gmres {
    int dim = 0;
    double *U = nullptr;      // [5][C] Newton iterate (conserved)
    double *Ustart = nullptr; // [5][C] conserved state at the start of the step
    double *r = nullptr;      // [5][C] Newton residual
    double *delta = nullptr;  // [5][C] increment
    double *V = nullptr;      // [dim + 1][5][C] Krylov basis
    double *w = nullptr;      // [5][C]
    double *q1 = nullptr;     // [5][N] perturbed primitive state
    double *R1 = nullptr;     // [5][C] derivative of the perturbed state
    double *part = nullptr;   // per-piece partial sums
    double *sc = nullptr;     // per-instance device scalars (GmresScalar)
    int *flag = nullptr;      // per-instance progress (GmresFlag)
    int *count = nullptr;     // [2] instances still iterating (Newton, Arnoldi)
    int *ctl = nullptr;       // [GC_COUNT] loop counters of the graph-driven loops
    double *Rm = nullptr;     // [5][C] FP32-flux form: the matvec's base residual, in FP32 fluxes
};

// Host mirror of the per-instance step arrays (pinned; one copy per direction moves all of them):
// doubles: time, step, step0, max_step, max_time, threshold, residual[5]; ints: variable, iter,
// max_iter, active, then num_active and error.
enum { SD_TIME, SD_STEP, SD_STEP0, SD_MAX_STEP, SD_MAX_TIME, SD_THRESHOLD, SD_RESIDUAL, SD_COUNT = SD_RESIDUAL + 5 };
enum { SI_VARIABLE, SI_ITER, SI_MAX_ITER, SI_ACTIVE, SI_FAIL, SI_COUNT };

// Chunks of a single-mesh context for steps whose host copies overlap the kernels (tg_advance_host):
// cell chunks of consecutive cells (multiples of the gradient's 32-cell tiles), the inner faces whose
// left cell lies in each chunk (teal sorts inner faces by their left cell), and the face chunks whose
// flux records each cell chunk gathers (bit masks: at most 64 chunks)
struct IoPlan {
    int K = 0;
    std::vector<int> cell_off;        // [K + 1]
    std::vector<int> face_off;        // [K + 1]
    std::vector<uint64_t> cell_face;  // [K]
    cudaStream_t copy = nullptr;      // host copies
    std::vector<cudaEvent_t> ev;      // [K + 1] a chunk's rows are gathered for the copy
};

struct tg_ctx {
    int device = 0;
    int source = TG_SOURCE_NONE;  // device source term kind and its parameters
    double src_par[4] = {0, 0, 0, 0};
    double *src_avg = nullptr;    // [ninst][5] volume averages (bulk forcing)
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;

    // sizes
    Sizes s{};
    int num_periodic = 0;  // periodic ghosts of the arena (redirected to their owners)
    // work range of the next gradient / cell launches (cells) and face launches (faces); hi < 0: all
    int cell_lo = 0, cell_hi = -1, face_lo = 0, face_hi = -1;
    IoPlan *io = nullptr;  // chunks of the steps with overlapped host copies (built on first use)

    // equations (shared by every instance of the arena)
    int physics = 0, order = 2, flux = 0, viscous = 0, limiter = 0, precision = 0;
    double prop[3] = {1.4, 0, 0.71};

    // instances
    int ninst = 1;
    std::vector<int> inst_row_off;  // teal rows of each instance in the row map
    int *rowmap = nullptr;          // teal row of an instance -> arena state row (periodic: owner)
    std::vector<int> h_inst_cell_off;
    int *cell_inst = nullptr, *inst_cell_off = nullptr, *piece_beg = nullptr, *inst_piece_off = nullptr;
    double *sum_volume = nullptr;
    int npieces = 0;
    Segments seg{};

    // device mesh
    int2 *lr = nullptr;
    int *slot_nbr = nullptr, *slot_face = nullptr;
    uint8_t *slot_cnt = nullptr;
    bool full_slots = true;    // every inner cell has MAX_SLOTS faces
    int *owner = nullptr;      // periodic ghost -> owner cell
    int *bface_ent = nullptr;  // boundary face -> boundary index
    int *bkind = nullptr;      // boundary index -> TG_BC_*
    double *bctx = nullptr;    // boundary index -> primitive context [5]
    double *volume = nullptr, *proj = nullptr, *eps2 = nullptr;
    GeomBuf gb;
    Geometry<double> g64{};
    Geometry<float> g32{};

    // state
    double *q = nullptr, *U0 = nullptr, *R = nullptr;
    double *qs = nullptr;  // scratch state for derivatives of host-given states (allocated on use)
    void *grad = nullptr, *G = nullptr;  // gradient records [C][5][4], face flux records [F][4] + [F]
    double *dtc = nullptr;               // per-cell stable step
    double *part_min = nullptr, *part_sum = nullptr;
    double *sd = nullptr;  // device step doubles [SD_COUNT][ninst]
    int *si = nullptr;     // device step ints [SI_COUNT][ninst] + num_active + error
    double *hd = nullptr;  // pinned mirrors
    int *hi = nullptr;
    Steps st{};
    double *aos = nullptr;     // device scratch for teal-layout transfers
    size_t aos_len = 0;
    double *pinned = nullptr;  // pinned host staging buffer
    size_t pinned_len = 0;
    bool prepared = false;     // U0, dtc and the piece minima valid for the resident state

    // implicit solver workspace (allocated on first use)
    Gmres gm{};

    // kernel launch count and optional per-kernel event timing
    long launches = 0;
    long graph_kernels = 0;
    bool prof_on = false;
    std::vector<cudaEvent_t> prof_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_open;
    double prof_ms[TG_PROF_CATEGORIES] = {0};
    long prof_n[TG_PROF_CATEGORIES] = {0};

    // device functions in place of teal's Compute callbacks (one-mesh contexts)
    std::vector<std::pair<int, int>> bd_range;  // boundary index -> teal face range [beg, end)
    std::vector<const void *> bd_kernel;        // boundary index -> bound kernel (custom kinds)
    std::vector<int> bd_kind;                   // boundary index -> TG_BC_* (host copy)
    double *bcenter = nullptr;  // [F_bd - F_in][3] ghost cell centres of the boundary faces
    double *ccenter = nullptr;  // [C][3] cell centres (device source)
    double *S = nullptr;        // [5][C] device source values of the residual being evaluated
    double *pref = nullptr;     // [ninst] reference pressure of the FP32-flux form (Local::dp)
    std::vector<double> h_pref; // its host copy (the source of each upload stays alive)
    double *dprop = nullptr;    // [3] properties
    const void *src_kernel = nullptr;
    int src_prepare = TG_PREPARE_NONE;
    // time of the residual being evaluated: time[0] + coef * step[0] on the device (inside step
    // sequences), else host
    const double *t_time = nullptr, *t_step = nullptr;
    double t_coef = 0, t_host = 0;

    // step graph cache
    cudaGraphExec_t graph = nullptr;
    int graph_method = -1, graph_stages = 0;
    double graph_courant = 0;
    int graph_use_max_time = -1;

    // polls of the staged face kernel's first bounded wait (lowered only by tg_set_wait_limit)
    int wait_polls = MBAR_POLLS;
    // created by tg_batch_create: an instance that goes non-finite stops alone (tg_batch_status)
    bool batch = false;

    // a partition (tg_create_partition): halo rows [N - halo, N), rows sent to other ranks, and the
    // packed exchange buffers
    int halo = 0, nsend = 0;
    int *send_rows = nullptr;
    double *send_q = nullptr, *recv_q = nullptr;  // [nsend][5], [halo][5]
    void *send_rec = nullptr, *recv_rec = nullptr;  // [nsend][20], [halo][20] records (R)

    // implicit step graph (device-driven Newton / Arnoldi / Gram-Schmidt loops) and its key
    cudaGraphExec_t igraph = nullptr;
    long igraph_kernels = 0;
    double ig_courant = 0, ig_newton_tol = 0, ig_krylov_tol = 0;
    int ig_dim = 0, ig_use_max_time = -1;
    cudaStream_t cap_stream[3] = {nullptr, nullptr, nullptr};  // body captures of nested loops
};

static double &hd_at(tg_ctx *c, int field, int i) { return c->hd[(size_t)field * c->ninst + i]; }
static int &hi_at(tg_ctx *c, int field, int i) { return c->hi[(size_t)field * c->ninst + i]; }
static int &hi_num_active(tg_ctx *c) { return c->hi[(size_t)SI_COUNT * c->ninst]; }
static int &hi_error(tg_ctx *c) { return c->hi[(size_t)SI_COUNT * c->ninst + 1]; }

static const double LSERK_ALPHA[3][6][7] = {
    // tabulated low-storage RK coefficients, teal's table (src/simulation/advance.c:50-75)
    {
        {0.0000, 1.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000},
        {0.0000, 0.3333, 1.0000, 0.0000, 0.0000, 0.0000, 0.0000},
        {0.0000, 0.1481, 0.4000, 1.0000, 0.0000, 0.0000, 0.0000},
        {0.0000, 0.0833, 0.2069, 0.4265, 1.0000, 0.0000, 0.0000},
        {0.0000, 0.0533, 0.1263, 0.2375, 0.4414, 1.0000, 0.0000},
        {0.0000, 0.0370, 0.0851, 0.1521, 0.2562, 0.4512, 1.0000},
    },
    {
        {0.0000, 1.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000},
        {0.0000, 0.4242, 1.0000, 0.0000, 0.0000, 0.0000, 0.0000},
        {0.0000, 0.1918, 0.4929, 1.0000, 0.0000, 0.0000, 0.0000},
        {0.0000, 0.1084, 0.2602, 0.5052, 1.0000, 0.0000, 0.0000},
        {0.0000, 0.0695, 0.1602, 0.2898, 0.5060, 1.0000, 0.0000},
        {0.0000, 0.0482, 0.1085, 0.1885, 0.3050, 0.5063, 1.0000},
    },
    {
        {0.0000, 1.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000},
        {0.0000, 0.6612, 1.0000, 0.0000, 0.0000, 0.0000, 0.0000},
        {0.0000, 0.2884, 0.5010, 1.0000, 0.0000, 0.0000, 0.0000},
        {0.0000, 0.1666, 0.3027, 0.5275, 1.0000, 0.0000, 0.0000},
        {0.0000, 0.1067, 0.1979, 0.3232, 0.5201, 1.0000, 0.0000},
        {0.0000, 0.0742, 0.1393, 0.2198, 0.3302, 0.5181, 1.0000},
    },
};

static void free_ctx(tg_ctx *c)
{
    if (!c) return;
    for (auto &e : c->prof_pool) cudaEventDestroy(e);
    for (auto &p : c->prof_open) {
        cudaEventDestroy(p.second.first);
        cudaEventDestroy(p.second.second);
    }
    if (c->graph) cudaGraphExecDestroy(c->graph);
    if (c->igraph) cudaGraphExecDestroy(c->igraph);
    for (cudaStream_t s : c->cap_stream) {
        if (s) cudaStreamDestroy(s);
    }
    void *ptrs[] = {c->bcenter, c->ccenter, c->S, c->dprop, c->pref,
                    c->lr, c->slot_nbr, c->slot_face, c->slot_cnt, c->owner, c->bface_ent, c->bkind, c->bctx,
                    c->volume, c->proj, c->eps2, c->gb.area, c->gb.basis, c->gb.offl, c->gb.offr, c->gb.corr,
                    c->gb.slot_w, c->gb.slot_off, c->gb.area32, c->gb.basis32, c->gb.offl32, c->gb.offr32,
                    c->gb.corr32, c->gb.tile64, c->gb.tile32, c->gb.toff64, c->gb.toff32, c->q, c->U0, c->R, c->qs, c->grad, c->G,
                    c->dtc, c->part_min, c->part_sum, c->sd, c->si, c->aos, c->rowmap, c->cell_inst,
                    c->inst_cell_off, c->piece_beg, c->inst_piece_off, c->sum_volume, c->src_avg,
                    c->send_rows, c->send_q, c->recv_q, c->send_rec, c->recv_rec};
    for (void *p : ptrs) {
        if (p) cudaFree(p);
    }
    void *gp[] = {c->gm.U, c->gm.Ustart, c->gm.r, c->gm.delta, c->gm.V, c->gm.w, c->gm.q1, c->gm.R1,
                  c->gm.part, c->gm.sc, c->gm.flag, c->gm.count, c->gm.ctl, c->gm.Rm};
    for (void *p : gp) {
        if (p) cudaFree(p);
    }
    if (c->hd) cudaFreeHost(c->hd);
    if (c->hi) cudaFreeHost(c->hi);
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->io) {
        if (c->io->copy) cudaStreamDestroy(c->io->copy);
        for (cudaEvent_t e : c->io->ev) cudaEventDestroy(e);
        delete c->io;
    }
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

static int grid_of(long n)
{
    return (int)((n + BLOCK - 1) / BLOCK);
}

// per-kernel event timing of the hot-path launches (categories TG_PROF_*)
static cudaEvent_t prof_event(tg_ctx *c)
{
    if (!c->prof_pool.empty()) {
        cudaEvent_t e = c->prof_pool.back();
        c->prof_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

struct Launch {
    tg_ctx *c;
    int cat;
    cudaEvent_t a = nullptr, b = nullptr;
    Launch(tg_ctx *c_, int cat_) : c(c_), cat(cat_)
    {
        c->launches += 1;
        if (c->prof_on) {
            a = prof_event(c);
            b = prof_event(c);
            cudaEventRecord(a, c->stream);
        }
    }
    ~Launch()
    {
        if (c->prof_on) {
            cudaEventRecord(b, c->stream);
            c->prof_open.push_back({cat, {a, b}});
        }
    }
};

// ---- mesh input: one teal mesh, or several packed into one arena -------------------------------

// Arena arrays in teal's layouts plus what the device upload needs beyond them.
struct MeshInput {
    tg_mesh m{};                    // views into the vectors below, or the caller's arrays
    std::vector<int> face_cell;     // merged arrays (batches only)
    std::vector<double> area, basis, weight, offset, correction, volume, projection;
    std::vector<int> owner;         // periodic ghost (row - off_boundary_cells) -> inner owner
    std::vector<int> bent;          // boundary face (f - F_in) -> boundary index
    std::vector<int> bkind;         // boundary index -> TG_BC_*
    std::vector<double> bctx;       // boundary index -> [5]
    std::vector<double> eps2;       // Venkatakrishnan parameter per inner cell (empty: none)
    std::vector<int> inst_cell_off; // inner cells per instance
    std::vector<double> sum_volume; // per instance
    std::vector<int> inst_row_off;  // teal rows per instance
    std::vector<int> rowmap;        // teal row -> arena row (periodic ghosts: the owner's row)
    int halo = 0;                   // partitions: halo rows after the boundary ghosts
    std::vector<int> send_rows;     // partitions: rows whose state / records other ranks receive
};

// periodic ghost -> owner cell, by matching each receive tag with the send posted under it
// (the single-process halo exchange of src/equations/exchange.c:8-36 and src/mesh/create.c:351-440)
static int build_owner_map(const tg_mesh *m, std::vector<int> &owner)
{
    int off = m->off_boundary_cells;
    int num = m->num_cells - off;
    owner.assign(num, -1);
    std::vector<char> used(m->num_neighbors, 0);
    for (int k = 0; k < m->num_neighbors; k++) {
        int tag = m->neighbor_tag[2 * k + 0];
        int match = -1;
        for (int j = 0; j < m->num_neighbors; j++) {
            if (!used[j] && m->neighbor_tag[2 * j + 1] == tag) {
                match = j;
                break;
            }
        }
        if (match < 0) {
            return fail(TG_ERR_INVALID, "periodic receive with tag %d has no matching send", tag);
        }
        used[match] = 1;
        int nrecv = m->neighbor_recv_off[k + 1] - m->neighbor_recv_off[k];
        int nsend = m->neighbor_send_off[match + 1] - m->neighbor_send_off[match];
        if (nrecv != nsend) {
            return fail(TG_ERR_INVALID, "periodic exchange size mismatch (%d vs %d)", nrecv, nsend);
        }
        for (int i = 0; i < nrecv; i++) {
            int ghost = m->neighbor_recv_off[k] + i - off;
            int src = m->neighbor_send_idx[m->neighbor_send_off[match] + i];
            if (ghost < 0 || ghost >= num || src < 0 || src >= m->num_inner_cells) {
                return fail(TG_ERR_INVALID, "periodic exchange index out of range");
            }
            owner[ghost] = src;
        }
    }
    for (int i = 0; i < num; i++) {
        if (owner[i] < 0) {
            return fail(TG_ERR_INVALID, "ghost cell %d receives no state", off + i);
        }
    }
    return TG_OK;
}

static int validate(const tg_mesh *m, const tg_equations *e)
{
    if (!m || !e) return fail(TG_ERR_INVALID, "null mesh or equations");
    if (m->num_inner_cells <= 0 || m->num_cells < m->num_inner_cells ||
        m->off_boundary_cells < m->num_inner_cells || m->off_boundary_cells > m->num_cells)
        return fail(TG_ERR_INVALID, "invalid cell counts");
    if (m->off_periodic_cells != m->num_cells)
        return fail(TG_ERR_INVALID, "neighbour-rank ghost cells are not supported (one process)");
    if (m->num_faces <= 0 || m->num_inner_faces < 0 || m->num_inner_faces > m->off_boundary_faces ||
        m->off_boundary_faces > m->num_faces)
        return fail(TG_ERR_INVALID, "invalid face counts");
    if (!m->face_cell || !m->face_area || !m->face_basis || !m->face_weight || !m->face_offset ||
        !m->cell_volume || !m->cell_projection)
        return fail(TG_ERR_INVALID, "missing mesh array");
    if (e->physics != TG_EULER && e->physics != TG_NAVIERSTOKES)
        return fail(TG_ERR_INVALID, "invalid physics %d", e->physics);
    if (e->space_order != 1 && e->space_order != 2)
        return fail(TG_ERR_INVALID, "invalid space order (%d)", e->space_order);
    if (e->convective < TG_FLUX_NONE || e->convective > TG_FLUX_CENTRAL)
        return fail(TG_ERR_INVALID, "invalid convective flux kind %d", e->convective);
    if (e->viscous != TG_VISCOUS_NONE && e->viscous != TG_VISCOUS_CENTRAL)
        return fail(TG_ERR_INVALID, "invalid viscous flux kind %d", e->viscous);
    if (e->viscous == TG_VISCOUS_CENTRAL && e->physics != TG_NAVIERSTOKES)
        return fail(TG_ERR_INVALID, "viscous flux needs the Navier-Stokes equations");
    if (e->viscous == TG_VISCOUS_CENTRAL && !m->face_correction)
        return fail(TG_ERR_INVALID, "viscous flux needs face corrections");
    if (e->limiter < TG_LIMITER_NONE || e->limiter > TG_LIMITER_VENKATAKRISHNAN)
        return fail(TG_ERR_INVALID, "invalid limiter kind (%d)", e->limiter);
    if (e->source < TG_SOURCE_NONE || e->source > TG_SOURCE_DEVICE)
        return fail(TG_ERR_INVALID, "invalid source kind (%d)", e->source);
    if (e->source == TG_SOURCE_BULK_FORCING && !(e->source_parameter[1] != 0))
        return fail(TG_ERR_INVALID, "bulk forcing needs a nonzero time scale");
    int nb = m->off_boundary_entities - m->num_inner_entities;
    if (nb != e->num_boundaries)
        return fail(TG_ERR_INVALID, "boundary count %d does not match the mesh (%d)", e->num_boundaries, nb);
    for (int i = 0; i < nb; i++) {
        int k = e->boundary_kind ? e->boundary_kind[i] : 0;
        if (k < TG_BC_SYMMETRY || k > TG_BC_CUSTOM)
            return fail(TG_ERR_INVALID, "boundary %d has no device boundary condition", i);
        if (k == TG_BC_ADIABATIC_WALL && e->physics != TG_NAVIERSTOKES)
            return fail(TG_ERR_INVALID, "adiabatic wall needs the Navier-Stokes equations");
    }
    return TG_OK;
}

// boundary faces of one mesh -> its boundary index; boundary kinds and contexts
static int boundary_tables(const tg_mesh *m, const tg_equations *e, std::vector<int> &bent, std::vector<int> &bkind,
                           std::vector<double> &bctx)
{
    int F_in = m->num_inner_faces, F_bd = m->off_boundary_faces;
    bent.assign(F_bd - F_in, -1);
    bkind.resize(e->num_boundaries);
    bctx.assign(5 * (size_t)e->num_boundaries, 0.0);
    for (int i = 0; i < e->num_boundaries; i++) {
        bkind[i] = e->boundary_kind[i];
        for (int v = 0; v < 5; v++) bctx[5 * i + v] = e->boundary_context ? e->boundary_context[5 * i + v] : 0.0;
        int ent = m->num_inner_entities + i;
        int beg = m->entity_face_off[ent], end = m->entity_face_off[ent + 1];
        if (beg < F_in || end > F_bd || beg > end)
            return fail(TG_ERR_INVALID, "boundary entity %d face range [%d, %d) invalid", i, beg, end);
        for (int f = beg; f < end; f++) bent[f - F_in] = i;
    }
    for (size_t i = 0; i < bent.size(); i++) {
        if (bent[i] < 0) return fail(TG_ERR_INVALID, "boundary face %zu belongs to no boundary", i + F_in);
        int r = m->face_cell[2 * (F_in + i) + 1];
        if (r < m->num_inner_cells || r >= m->off_boundary_cells)
            return fail(TG_ERR_INVALID, "boundary face right cell out of range");
    }
    return TG_OK;
}

static void limiter_parameter(const tg_mesh *m, const tg_equations *e, double *eps2)
{
    for (int i = 0; i < m->num_inner_cells; i++) {
        if (e->limiter_parameter) {
            eps2[i] = e->limiter_parameter[i];
        }
        else {  // eps^2 = (K * V^(1/3))^3, src/equations/limiter.c:8-21
            double x = e->limiter_coefficient * cbrt(m->cell_volume[i]);
            eps2[i] = (x * x) * x;
        }
    }
}

static int single_input(const tg_mesh *m, const tg_equations *e, MeshInput &in)
{
    TRY(validate(m, e));
    in.m = *m;
    TRY(build_owner_map(m, in.owner));
    TRY(boundary_tables(m, e, in.bent, in.bkind, in.bctx));
    if (e->limiter == TG_LIMITER_VENKATAKRISHNAN) {
        in.eps2.resize(m->num_inner_cells);
        limiter_parameter(m, e, in.eps2.data());
    }
    in.inst_cell_off = {0, m->num_inner_cells};
    in.sum_volume = {m->sum_volume};
    in.inst_row_off = {0, m->num_cells};
    in.rowmap.resize(m->num_cells);
    for (int r = 0; r < m->num_cells; r++) {
        in.rowmap[r] = r < m->off_boundary_cells ? r : in.owner[r - m->off_boundary_cells];
    }
    return TG_OK;
}

// Pack several meshes into one arena: all inner cells (instance order), then all boundary ghosts,
// then all periodic ghosts; faces likewise (inner, boundary, periodic). Every kernel then runs over
// the arena as over one mesh whose instances are disconnected pieces.
static int merged_input(const tg_mesh *ms, const tg_equations *es, int num, MeshInput &in)
{
    if (num <= 0) return fail(TG_ERR_INVALID, "a batch needs at least one instance");
    const tg_equations &e0 = es[0];
    for (int i = 0; i < num; i++) {
        TRY(validate(&ms[i], &es[i]));
        const tg_equations &e = es[i];
        if (e.source == TG_SOURCE_DEVICE)
            return fail(TG_ERR_INVALID, "device source functions need a one-mesh context");
        for (int b = 0; b < e.num_boundaries; b++) {
            if (e.boundary_kind[b] == TG_BC_CUSTOM)
                return fail(TG_ERR_INVALID, "custom boundary functions need a one-mesh context");
        }
        if (e.physics != e0.physics || e.space_order != e0.space_order || e.convective != e0.convective ||
            e.viscous != e0.viscous || e.limiter != e0.limiter || e.property[0] != e0.property[0] ||
            e.property[1] != e0.property[1] || e.property[2] != e0.property[2] || e.source != e0.source ||
            memcmp(e.source_parameter, e0.source_parameter, sizeof(e.source_parameter)) != 0)
            return fail(TG_ERR_INVALID, "batch instance %d differs in equations, schemes or properties", i);
    }
    long C = 0, NB = 0, NP = 0, Fi = 0, Fb = 0, Fp = 0, nbnd = 0, rows = 0;
    for (int i = 0; i < num; i++) {
        const tg_mesh &m = ms[i];
        C += m.num_inner_cells;
        NB += m.off_boundary_cells - m.num_inner_cells;
        NP += m.num_cells - m.off_boundary_cells;
        Fi += m.num_inner_faces;
        Fb += m.off_boundary_faces - m.num_inner_faces;
        Fp += m.num_faces - m.off_boundary_faces;
        nbnd += es[i].num_boundaries;
        rows += m.num_cells;
    }
    if (C + NB + NP > 2000000000L || Fi + Fb + Fp > 2000000000L)
        return fail(TG_ERR_INVALID, "batch exceeds 2^31 cells or faces");
    const long F = Fi + Fb + Fp;
    in.face_cell.resize(2 * F);
    in.area.resize(F);
    in.basis.resize(9 * F);
    in.weight.resize(6 * F);
    in.offset.resize(6 * F);
    bool visc = e0.viscous == TG_VISCOUS_CENTRAL;
    if (visc) in.correction.resize(4 * F);
    in.volume.assign(C + NB + NP, 0.0);
    in.projection.assign(3 * (C + NB + NP), 0.0);
    in.owner.resize(NP);
    in.bent.resize(Fb);
    in.bkind.clear();
    in.bctx.clear();
    if (e0.limiter == TG_LIMITER_VENKATAKRISHNAN) in.eps2.resize(C);
    in.inst_cell_off.assign(1, 0);
    in.sum_volume.clear();
    in.inst_row_off.assign(1, 0);
    in.rowmap.resize(rows);

    long c0 = 0, b0 = 0, p0 = 0, fi0 = 0, fb0 = 0, fp0 = 0, bnd0 = 0, row0 = 0;
    for (int i = 0; i < num; i++) {
        const tg_mesh &m = ms[i];
        const tg_equations &e = es[i];
        std::vector<int> owner, bent, bkind;
        std::vector<double> bctx;
        TRY(build_owner_map(&m, owner));
        TRY(boundary_tables(&m, &e, bent, bkind, bctx));
        const int Ci = m.num_inner_cells, OBi = m.off_boundary_cells;
        auto cell = [&](int r) -> long {
            if (r < Ci) return c0 + r;
            if (r < OBi) return C + b0 + (r - Ci);
            return C + NB + p0 + (r - OBi);
        };
        auto copy_face = [&](int f, long g) {
            in.face_cell[2 * g] = (int)cell(m.face_cell[2 * f]);
            in.face_cell[2 * g + 1] = (int)cell(m.face_cell[2 * f + 1]);
            in.area[g] = m.face_area[f];
            memcpy(&in.basis[9 * g], m.face_basis + 9 * (size_t)f, 9 * sizeof(double));
            memcpy(&in.weight[6 * g], m.face_weight + 6 * (size_t)f, 6 * sizeof(double));
            memcpy(&in.offset[6 * g], m.face_offset + 6 * (size_t)f, 6 * sizeof(double));
            if (visc) memcpy(&in.correction[4 * g], m.face_correction + 4 * (size_t)f, 4 * sizeof(double));
        };
        for (int f = 0; f < m.num_inner_faces; f++) copy_face(f, fi0 + f);
        for (int f = m.num_inner_faces; f < m.off_boundary_faces; f++) {
            copy_face(f, Fi + fb0 + (f - m.num_inner_faces));
            in.bent[fb0 + (f - m.num_inner_faces)] = (int)(bnd0 + bent[f - m.num_inner_faces]);
        }
        for (int f = m.off_boundary_faces; f < m.num_faces; f++) copy_face(f, Fi + Fb + fp0 + (f - m.off_boundary_faces));
        for (int r = 0; r < m.num_cells; r++) {
            long a = cell(r);
            in.volume[a] = m.cell_volume[r];
            memcpy(&in.projection[3 * a], m.cell_projection + 3 * (size_t)r, 3 * sizeof(double));
        }
        for (int p = 0; p < m.num_cells - OBi; p++) in.owner[p0 + p] = (int)(c0 + owner[p]);
        in.bkind.insert(in.bkind.end(), bkind.begin(), bkind.end());
        in.bctx.insert(in.bctx.end(), bctx.begin(), bctx.end());
        if (!in.eps2.empty()) limiter_parameter(&m, &e, &in.eps2[c0]);
        for (int r = 0; r < m.num_cells; r++) {
            in.rowmap[row0 + r] = (int)(r < OBi ? cell(r) : c0 + owner[r - OBi]);
        }
        c0 += Ci;
        b0 += OBi - Ci;
        p0 += m.num_cells - OBi;
        fi0 += m.num_inner_faces;
        fb0 += m.off_boundary_faces - m.num_inner_faces;
        fp0 += m.num_faces - m.off_boundary_faces;
        bnd0 += e.num_boundaries;
        row0 += m.num_cells;
        in.inst_cell_off.push_back((int)c0);
        in.sum_volume.push_back(m.sum_volume);
        in.inst_row_off.push_back((int)row0);
    }
    tg_mesh &v = in.m;
    memset(&v, 0, sizeof(v));
    v.num_cells = (int)(C + NB + NP);
    v.num_inner_cells = (int)C;
    v.off_boundary_cells = (int)(C + NB);
    v.off_periodic_cells = v.num_cells;
    v.cell_volume = in.volume.data();
    v.cell_projection = in.projection.data();
    v.num_faces = (int)F;
    v.num_inner_faces = (int)Fi;
    v.off_boundary_faces = (int)(Fi + Fb);
    v.face_cell = in.face_cell.data();
    v.face_area = in.area.data();
    v.face_basis = in.basis.data();
    v.face_weight = in.weight.data();
    v.face_offset = in.offset.data();
    v.face_correction = visc ? in.correction.data() : nullptr;
    return TG_OK;
}

// ---- device upload ------------------------------------------------------------------------------

template <typename T>
static int upload(T **dst, const T *src, size_t n, cudaStream_t st)
{
    TRY(dalloc(dst, n));
    if (n) CU(cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return TG_OK;
}

static int alloc_geom32(tg_ctx *c)
{
    const Sizes &s = c->s;
    TRY(dalloc(&c->gb.area32, s.F));
    TRY(dalloc(&c->gb.basis32, 9 * (size_t)s.F));
    TRY(dalloc(&c->gb.offl32, 3 * (size_t)s.F));
    TRY(dalloc(&c->gb.offr32, 3 * (size_t)s.F));
    if (c->gb.corr) TRY(dalloc(&c->gb.corr32, 4 * (size_t)s.F));
    return TG_OK;
}

__global__ static void k_to_float(size_t n, const double *__restrict__ a, float *__restrict__ b)
{
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = float(a[i]);
}

static int to_float(const double *a, float *b, size_t n, cudaStream_t st)
{
    if (!a || !b || n == 0) return TG_OK;
    k_to_float<<<(unsigned)((n + BLOCK - 1) / BLOCK), BLOCK, 0, st>>>(n, a, b);
    CU(cudaGetLastError());
    return TG_OK;
}

// AoS host array [n][k] -> device SoA [k][n] through a device temporary
static int upload_soa(double **dst, const double *src, size_t n, int k, double *tmp, cudaStream_t st)
{
    TRY(dalloc(dst, (size_t)k * n));
    if (!n) return TG_OK;
    CU(cudaMemcpyAsync(tmp, src, (size_t)k * n * sizeof(double), cudaMemcpyHostToDevice, st));
    k_transpose<double><<<grid_of((long)n), BLOCK, 0, st>>>((int)n, k, tmp, *dst);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(st));  // tmp is reused by the next upload
    return TG_OK;
}

static int create_ctx(MeshInput &in, const tg_equations *e, int precision, tg_ctx **out)
{
    *out = nullptr;
    if (precision != TG_PRECISION_FP64 && precision != TG_PRECISION_FP32_FLUX && precision != TG_PRECISION_FP64_EXACT)
        return fail(TG_ERR_INVALID, "invalid precision %d", precision);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(TG_ERR_NO_DEVICE, "no CUDA device available");
    const tg_mesh *m = &in.m;

    tg_ctx *c = new tg_ctx();
    int rc = [&]() -> int {
        CU(cudaGetDevice(&c->device));
        CU(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
        c->stream = c->own_stream;
        cudaStream_t st = c->stream;

        Sizes &s = c->s;
        s.C = m->num_inner_cells;
        s.N = m->off_boundary_cells + in.halo;  // state rows: inner, boundary ghosts, halo (partitions)
        s.F = m->num_faces;
        s.F_in = m->num_inner_faces;
        s.F_bd = m->off_boundary_faces;
        s.SL = (s.C + 3) & ~3;
        c->num_periodic = m->num_cells - m->off_boundary_cells;
        c->physics = e->physics;
        c->order = e->space_order;
        c->flux = e->convective;
        c->viscous = e->viscous;
        c->limiter = e->limiter;
        c->precision = precision;
        for (int i = 0; i < 3; i++) c->prop[i] = e->property[i];
        c->source = e->source;
        for (int i = 0; i < 4; i++) c->src_par[i] = e->source_parameter[i];

        // instances and reduction pieces
        c->ninst = (int)in.inst_cell_off.size() - 1;
        c->inst_row_off = in.inst_row_off;
        c->h_inst_cell_off = in.inst_cell_off;
        std::vector<int> cell_inst(s.C), piece_beg, inst_piece_off(1, 0);
        for (int i = 0; i < c->ninst; i++) {
            for (int x = in.inst_cell_off[i]; x < in.inst_cell_off[i + 1]; x++) cell_inst[x] = i;
            for (int x = in.inst_cell_off[i]; x < in.inst_cell_off[i + 1]; x += PIECE) piece_beg.push_back(x);
            inst_piece_off.push_back((int)piece_beg.size());
        }
        c->npieces = (int)piece_beg.size();
        piece_beg.push_back(s.C);
        TRY(upload(&c->cell_inst, cell_inst.data(), cell_inst.size(), st));
        TRY(upload(&c->inst_cell_off, in.inst_cell_off.data(), in.inst_cell_off.size(), st));
        TRY(upload(&c->piece_beg, piece_beg.data(), piece_beg.size(), st));
        TRY(upload(&c->inst_piece_off, inst_piece_off.data(), inst_piece_off.size(), st));
        TRY(upload(&c->sum_volume, in.sum_volume.data(), in.sum_volume.size(), st));
        TRY(upload(&c->rowmap, in.rowmap.data(), in.rowmap.size(), st));
        c->seg = Segments{c->ninst, c->npieces, c->cell_inst, c->inst_cell_off, c->piece_beg, c->inst_piece_off,
                          c->sum_volume};

        // raw teal arrays -> device temporaries
        int *d_face_cell = nullptr, *d_err = nullptr, *d_cnt = nullptr;
        double *d_weight = nullptr, *d_offset = nullptr, *d_tmp = nullptr;
        auto cleanup = [&]() {
            cudaFree(d_face_cell);
            cudaFree(d_err);
            cudaFree(d_cnt);
            cudaFree(d_weight);
            cudaFree(d_offset);
            cudaFree(d_tmp);
        };
        int r2 = [&]() -> int {
            TRY(upload(&d_face_cell, m->face_cell, 2 * (size_t)s.F, st));
            TRY(upload(&c->owner, in.owner.data(), in.owner.size(), st));
            TRY(dalloc(&d_err, 1));
            CU(cudaMemsetAsync(d_err, 0, sizeof(int), st));
            TRY(dalloc(&c->lr, s.F));
            k_redirect<<<grid_of(s.F), BLOCK, 0, st>>>(s.F, s.F_bd, m->off_boundary_cells, d_face_cell, c->owner,
                                                       (int)in.owner.size(), c->lr, d_err);
            CU(cudaGetLastError());

            // per-cell slot lists: count, scatter, sort by face (integer work on the device)
            TRY(dalloc(&d_cnt, 2 * (size_t)s.C));
            CU(cudaMemsetAsync(d_cnt, 0, 2 * sizeof(int) * s.C, st));
            // slot rows are SL = C rounded up to 4 long (16-byte rows); the padding columns stay zero
            TRY(dalloc(&c->slot_face, MAX_SLOTS * (size_t)s.SL));
            TRY(dalloc(&c->slot_nbr, MAX_SLOTS * (size_t)s.SL));
            TRY(dalloc(&c->slot_cnt, s.C));
            TRY(dalloc(&c->gb.slot_w, 3 * MAX_SLOTS * (size_t)s.SL));
            TRY(dalloc(&c->gb.slot_off, 3 * MAX_SLOTS * (size_t)s.SL));
            CU(cudaMemsetAsync(c->slot_face, 0, MAX_SLOTS * sizeof(int) * (size_t)s.SL, st));
            CU(cudaMemsetAsync(c->slot_nbr, 0, MAX_SLOTS * sizeof(int) * (size_t)s.SL, st));
            CU(cudaMemsetAsync(c->gb.slot_w, 0, 3 * MAX_SLOTS * sizeof(double) * (size_t)s.SL, st));
            CU(cudaMemsetAsync(c->gb.slot_off, 0, 3 * MAX_SLOTS * sizeof(double) * (size_t)s.SL, st));
            k_slot_count<<<grid_of(s.F), BLOCK, 0, st>>>(s.F, s.F_in, s.C, c->lr, d_cnt);
            k_slot_fill<<<grid_of(s.F), BLOCK, 0, st>>>(s.F, s.F_in, s.C, s.SL, c->lr, d_cnt + s.C, c->slot_face);
            TRY(upload(&d_weight, m->face_weight, 6 * (size_t)s.F, st));
            TRY(upload(&d_offset, m->face_offset, 6 * (size_t)s.F, st));
            k_slot_finish<double><<<grid_of(s.C), BLOCK, 0, st>>>(s.C, s.SL, c->lr, d_cnt, d_weight, d_offset,
                                                                  c->slot_face, c->slot_nbr, c->slot_cnt,
                                                                  c->gb.slot_w, c->gb.slot_off, d_err);
            CU(cudaGetLastError());
            {
                // on meshes whose cells all have MAX_SLOTS faces (hexahedra) the gradient kernel
                // takes the slot count as a compile-time constant
                std::vector<uint8_t> cnt(s.C);
                CU(cudaMemcpyAsync(cnt.data(), c->slot_cnt, s.C, cudaMemcpyDeviceToHost, st));
                CU(cudaStreamSynchronize(st));
                c->full_slots = true;
                for (uint8_t k : cnt) c->full_slots = c->full_slots && k == MAX_SLOTS;

                // gradient tiles: the slot geometry of every 32 cells in one block, as many slots as
                // the block's cell with the most faces (FP64 always; FP32 for the FP32-flux form)
                const int ntiles = (s.C + GRAD_CELLS - 1) / GRAD_CELLS;
                std::vector<int> tj(ntiles, 0);
                for (int i = 0; i < s.C; i++) tj[i / GRAD_CELLS] = std::max(tj[i / GRAD_CELLS], int(cnt[i]));
                auto tiles = [&](auto zero, unsigned char **buf, long long **toff) -> int {
                    using G = decltype(zero);
                    std::vector<long long> off(ntiles + 1, 0);
                    for (int t = 0; t < ntiles; t++) off[t + 1] = off[t] + grad_tile_bytes<G>(tj[t]);
                    TRY(upload(toff, off.data(), off.size(), st));
                    TRY(dalloc(buf, (size_t)off[ntiles]));
                    if (ntiles > 0) {
                        k_grad_tiles<G><<<ntiles, GRAD_CELLS, 0, st>>>(s.C, s.SL, *toff, c->slot_nbr, c->gb.slot_w,
                                                                      c->gb.slot_off, *buf);
                    }
                    CU(cudaGetLastError());
                    return TG_OK;
                };
                TRY(tiles(double(0), &c->gb.tile64, &c->gb.toff64));
                if (precision == TG_PRECISION_FP32_FLUX) TRY(tiles(float(0), &c->gb.tile32, &c->gb.toff32));
                CU(cudaStreamSynchronize(st));
                cudaFree(c->gb.slot_w);
                cudaFree(c->gb.slot_off);
                c->gb.slot_w = c->gb.slot_off = nullptr;
            }

            // face geometry, structure of arrays
            TRY(upload(&c->gb.area, m->face_area, s.F, st));
            TRY(dalloc(&d_tmp, 9 * (size_t)s.F > 3 * (size_t)s.C ? 9 * (size_t)s.F : 3 * (size_t)s.C));
            TRY(upload_soa(&c->gb.basis, m->face_basis, s.F, 9, d_tmp, st));
            std::vector<double> ol(3 * (size_t)s.F), orr(3 * (size_t)s.F);
            for (int f = 0; f < s.F; f++) {
                for (int d = 0; d < 3; d++) {
                    ol[(size_t)f * 3 + d] = m->face_offset[(size_t)f * 6 + d];
                    orr[(size_t)f * 3 + d] = m->face_offset[(size_t)f * 6 + 3 + d];
                }
            }
            TRY(upload_soa(&c->gb.offl, ol.data(), s.F, 3, d_tmp, st));
            TRY(upload_soa(&c->gb.offr, orr.data(), s.F, 3, d_tmp, st));
            if (e->viscous == TG_VISCOUS_CENTRAL) {
                TRY(upload_soa(&c->gb.corr, m->face_correction, s.F, 4, d_tmp, st));
            }

            // cells and boundaries
            TRY(upload(&c->volume, m->cell_volume, s.C, st));
            TRY(upload_soa(&c->proj, m->cell_projection, s.C, 3, d_tmp, st));
            if (!in.eps2.empty()) TRY(upload(&c->eps2, in.eps2.data(), s.C, st));
            if (s.F_bd > s.F_in) {
                TRY(upload(&c->bface_ent, in.bent.data(), in.bent.size(), st));
                TRY(upload(&c->bkind, in.bkind.data(), in.bkind.size(), st));
                TRY(upload(&c->bctx, in.bctx.data(), in.bctx.size(), st));
            }
            CU(cudaGetLastError());

            int h_err = 0;
            CU(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
            CU(cudaStreamSynchronize(st));
            if (h_err == 1) return fail(TG_ERR_INVALID, "a cell has more than %d or no faces", MAX_SLOTS);
            if (h_err == 2) return fail(TG_ERR_INVALID, "periodic face right cell is not a periodic ghost");
            return TG_OK;
        }();
        cleanup();
        TRY(r2);

        // FP32 copies for the FP32 flux form
        if (precision == TG_PRECISION_FP32_FLUX) {
            TRY(alloc_geom32(c));
            TRY(to_float(c->gb.area, c->gb.area32, s.F, st));
            TRY(to_float(c->gb.basis, c->gb.basis32, 9 * (size_t)s.F, st));
            TRY(to_float(c->gb.offl, c->gb.offl32, 3 * (size_t)s.F, st));
            TRY(to_float(c->gb.offr, c->gb.offr32, 3 * (size_t)s.F, st));
            TRY(to_float(c->gb.corr, c->gb.corr32, 4 * (size_t)s.F, st));
        }
        c->g64 = Geometry<double>{c->lr,       c->gb.area,  c->gb.basis,   c->gb.offl,   c->gb.offr,   c->gb.corr,
                                  c->slot_nbr, c->slot_face, c->slot_cnt, c->gb.tile64, c->gb.toff64};
        c->g32 = Geometry<float>{c->lr,         c->gb.area32, c->gb.basis32, c->gb.offl32,   c->gb.offr32,
                                 c->gb.corr32, c->slot_nbr,  c->slot_face,  c->slot_cnt, c->gb.tile32,
                                 c->gb.toff32};

        // state
        // FP64 record size in every form: the FP32-flux form's implicit step evaluates its Newton
        // residuals with the FP64 kernels (enqueue_implicit_step)
        size_t rsz = sizeof(double);
        TRY(dalloc(&c->q, 5 * (size_t)s.N));
        CU(cudaMemsetAsync(c->q, 0, 5 * sizeof(double) * s.N, st));
        TRY(dalloc(&c->U0, 5 * (size_t)s.C));
        TRY(dalloc(&c->R, 5 * (size_t)s.C));
        CU(cudaMemsetAsync(c->R, 0, 5 * sizeof(double) * s.C, st));
        if (c->order == 2) {
            // records for every state row: a partition's halo rows receive their owners' records
            CU(cudaMalloc(&c->grad, 20 * rsz * s.N));
        }
        if (in.halo > 0 || !in.send_rows.empty()) {
            c->halo = in.halo;
            c->nsend = (int)in.send_rows.size();
            TRY(upload(&c->send_rows, in.send_rows.data(), in.send_rows.size(), st));
            TRY(dalloc(&c->send_q, 5 * (size_t)c->nsend));
            TRY(dalloc(&c->recv_q, 5 * (size_t)c->halo));
            CU(cudaMalloc(&c->send_rec, 20 * rsz * (size_t)(c->nsend > 0 ? c->nsend : 1)));
            CU(cudaMalloc(&c->recv_rec, 20 * rsz * (size_t)(c->halo > 0 ? c->halo : 1)));
        }
        // the exact form with a viscous flux keeps the viscous records apart (face.cuh)
        const bool two = precision == TG_PRECISION_FP64_EXACT && c->viscous == TG_VISCOUS_CENTRAL;
        const size_t nrec_elems = two ? flux_rec2_offset(s.F) + (size_t)FLUX_REC * s.F : (size_t)FLUX_REC * s.F;
        CU(cudaMalloc(&c->G, nrec_elems * rsz));
        TRY(dalloc(&c->dtc, s.C));
        if (precision == TG_PRECISION_FP32_FLUX) {
            TRY(dalloc(&c->pref, c->ninst));
            CU(cudaMemsetAsync(c->pref, 0, sizeof(double) * c->ninst, st));
            c->h_pref.assign(c->ninst, 0.0);
        }
        CU(cudaMemsetAsync(c->dtc, 0, sizeof(double) * s.C, st));
        TRY(dalloc(&c->part_min, c->npieces));
        TRY(dalloc(&c->part_sum, 5 * (size_t)c->npieces));
        TRY(dalloc(&c->src_avg, 5 * (size_t)c->ninst));
        TRY(dalloc(&c->sd, (size_t)SD_COUNT * c->ninst));
        TRY(dalloc(&c->si, (size_t)SI_COUNT * c->ninst + 2));
        CU(cudaMallocHost(&c->hd, sizeof(double) * SD_COUNT * c->ninst));
        CU(cudaMallocHost(&c->hi, sizeof(int) * (SI_COUNT * c->ninst + 2)));
        memset(c->hd, 0, sizeof(double) * SD_COUNT * c->ninst);
        memset(c->hi, 0, sizeof(int) * (SI_COUNT * c->ninst + 2));
        for (int i = 0; i < c->ninst; i++) {
            hd_at(c, SD_MAX_STEP, i) = DBL_MAX;
            hd_at(c, SD_MAX_TIME, i) = DBL_MAX;
            hi_at(c, SI_VARIABLE, i) = -1;
            hi_at(c, SI_MAX_ITER, i) = 0x7fffffff;
            hi_at(c, SI_ACTIVE, i) = 1;
        }
        // the device copy starts as the host mirror (error word clear)
        CU(cudaMemcpyAsync(c->sd, c->hd, sizeof(double) * SD_COUNT * c->ninst, cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(c->si, c->hi, sizeof(int) * (SI_COUNT * c->ninst + 2), cudaMemcpyHostToDevice, st));
        int n = c->ninst;
        c->st = Steps{c->sd + SD_TIME * n,     c->sd + SD_STEP * n,      c->sd + SD_STEP0 * n,
                      c->sd + SD_MAX_STEP * n, c->sd + SD_MAX_TIME * n,  c->sd + SD_THRESHOLD * n,
                      c->sd + SD_RESIDUAL * n, c->si + SI_VARIABLE * n,  c->si + SI_ITER * n,
                      c->si + SI_MAX_ITER * n, c->si + SI_ACTIVE * n,    c->si + SI_FAIL * n, c->si + SI_COUNT * n,
                      c->si + SI_COUNT * n + 1, 0};
        // the residual block is [ninst][5] inside the doubles: SD_RESIDUAL * n .. + 5 n
        c->aos_len = (size_t)15 * ((size_t)m->num_cells > (size_t)s.F ? (size_t)m->num_cells : (size_t)s.F);
        TRY(dalloc(&c->aos, c->aos_len));
        CU(cudaStreamSynchronize(st));
        return TG_OK;
    }();
    if (rc != TG_OK) {
        std::string msg = g_error;
        cudaDeviceSynchronize();
        free_ctx(c);
        g_error = msg;
        return rc;
    }
    *out = c;
    return TG_OK;
}

// Device data of the device functions: boundary ranges and ghost centres for custom boundaries,
// cell centres and the source buffer for a device source, the properties.
static int setup_functions(tg_ctx *c, const tg_mesh *m, const tg_equations *e)
{
    int nb = e->num_boundaries;
    c->bd_range.resize(nb);
    c->bd_kernel.assign(nb, nullptr);
    c->bd_kind.assign(e->boundary_kind, e->boundary_kind + nb);
    bool custom = false;
    for (int i = 0; i < nb; i++) {
        int ent = m->num_inner_entities + i;
        c->bd_range[i] = {m->entity_face_off[ent], m->entity_face_off[ent + 1]};
        custom = custom || e->boundary_kind[i] == TG_BC_CUSTOM;
    }
    cudaStream_t st = c->stream;
    if (custom || e->source == TG_SOURCE_DEVICE) {
        TRY(upload(&c->dprop, c->prop, 3, st));
    }
    if (custom) {
        int F_in = m->num_inner_faces, nbf = m->off_boundary_faces - F_in;
        std::vector<double> centre(3 * (size_t)std::max(nbf, 1));
        for (int i = 0; i < nbf; i++) {
            int r = m->face_cell[2 * (size_t)(F_in + i) + 1];
            for (int d = 0; d < 3; d++) centre[3 * (size_t)i + d] = m->cell_center[3 * (size_t)r + d];
        }
        TRY(upload(&c->bcenter, centre.data(), centre.size(), st));
    }
    if (e->source == TG_SOURCE_DEVICE) {
        TRY(upload(&c->ccenter, m->cell_center, 3 * (size_t)c->s.C, st));
        TRY(dalloc(&c->S, 5 * (size_t)c->s.C));
        CU(cudaMemsetAsync(c->S, 0, 5 * sizeof(double) * c->s.C, st));
    }
    CU(cudaStreamSynchronize(st));
    return TG_OK;
}

static void drop_graph(tg_ctx *c)
{
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    if (c->igraph) {
        cudaGraphExecDestroy(c->igraph);
        c->igraph = nullptr;
    }
}

extern "C" int tg_function_register(const char *name, int kind, const char *source, char *log, long log_size)
{
    std::string error;
    int rc = function_register(name, kind, source, log, log_size, error);
    if (rc == 1) return fail(TG_ERR_INVALID, "%s", error.c_str());
    if (rc != 0) return fail(TG_ERR_CUDA, "%s", error.c_str());
    return TG_OK;
}

extern "C" int tg_bind_boundary_function(tg_ctx *c, int boundary, const char *name)
{
    if (!c || !name) return fail(TG_ERR_INVALID, "null argument");
    if (c->ninst != 1) return fail(TG_ERR_INVALID, "device functions need a one-mesh context");
    if (boundary < 0 || boundary >= (int)c->bd_range.size())
        return fail(TG_ERR_INVALID, "boundary %d out of range", boundary);
    if (c->bd_kind[boundary] != TG_BC_CUSTOM)
        return fail(TG_ERR_INVALID, "boundary %d is not a custom boundary", boundary);
    std::string error;
    const void *k = nullptr;
    int rc = function_kernel(name, FUNCTION_BOUNDARY, &k, error);
    if (rc == 1) return fail(TG_ERR_INVALID, "%s", error.c_str());
    if (rc != 0) return fail(TG_ERR_CUDA, "%s", error.c_str());
    CU(cudaStreamSynchronize(c->stream));
    c->bd_kernel[boundary] = k;
    drop_graph(c);  // captured steps launch the previous binding
    return TG_OK;
}

extern "C" int tg_bind_source_function(tg_ctx *c, const char *name)
{
    if (!c || !name) return fail(TG_ERR_INVALID, "null argument");
    if (c->ninst != 1) return fail(TG_ERR_INVALID, "device functions need a one-mesh context");
    if (c->source != TG_SOURCE_DEVICE) return fail(TG_ERR_INVALID, "the equations' source is not a device function");
    std::string error;
    const void *k = nullptr;
    int rc = function_kernel(name, FUNCTION_SOURCE, &k, error);
    if (rc == 1) return fail(TG_ERR_INVALID, "%s", error.c_str());
    if (rc != 0) return fail(TG_ERR_CUDA, "%s", error.c_str());
    CU(cudaStreamSynchronize(c->stream));
    c->src_kernel = k;
    drop_graph(c);
    return TG_OK;
}

extern "C" int tg_bind_source_prepare(tg_ctx *c, int prepare)
{
    if (!c) return fail(TG_ERR_INVALID, "null argument");
    if (c->source != TG_SOURCE_DEVICE) return fail(TG_ERR_INVALID, "the equations' source is not a device function");
    if (prepare != TG_PREPARE_NONE && prepare != TG_PREPARE_AVERAGE)
        return fail(TG_ERR_INVALID, "unknown source prepare %d", prepare);
    CU(cudaStreamSynchronize(c->stream));
    c->src_prepare = prepare;
    drop_graph(c);
    return TG_OK;
}

extern "C" int tg_create(const tg_mesh *m, const tg_equations *e, int precision, tg_ctx **out)
{
    if (!out) return fail(TG_ERR_INVALID, "null output pointer");
    *out = nullptr;
    MeshInput in;
    TRY(single_input(m, e, in));
    TRY(create_ctx(in, e, precision, out));
    int rc = setup_functions(*out, m, e);
    if (rc != TG_OK) {
        std::string msg = g_error;
        tg_destroy(*out);
        *out = nullptr;
        return fail(rc, "%s", msg.c_str());
    }
    return TG_OK;
}

// ---- partitions: one rank's share of a mesh (multi-GPU) ------------------------------------------
//
// A partition is uploaded like a one-process mesh whose faces may reference halo rows: state rows
// after the boundary ghosts that hold inner cells of other ranks. Its faces are the global mesh's
// faces that touch its own inner cells, in global order and orientation, so every own cell sums
// its faces in the global order; faces between an own cell and a halo cell are computed on both
// ranks from the same exchanged inputs. The periodic ghosts of its periodic faces map through
// `owner` to state rows (own inner cells or halo rows).

extern "C" int tg_create_partition(const tg_mesh *m, const tg_equations *e, int precision, const int *owner,
                                   int num_halo, const int *send_rows, int num_send, tg_ctx **out)
{
    if (!out) return fail(TG_ERR_INVALID, "null output pointer");
    *out = nullptr;
    TRY(validate(m, e));
    if (num_halo < 0 || num_send < 0 || (num_send > 0 && !send_rows))
        return fail(TG_ERR_INVALID, "invalid halo sizes");
    if (e->source != TG_SOURCE_NONE)
        return fail(TG_ERR_INVALID, "source terms are not supported in a partition (their prepare pass is global)");
    MeshInput in;
    in.m = *m;
    const int C = m->num_inner_cells, OB = m->off_boundary_cells, rows = OB + num_halo;
    const int np = m->num_cells - OB;
    if (np > 0 && !owner) return fail(TG_ERR_INVALID, "periodic ghosts need their owner rows");
    in.owner.assign(owner, owner + np);
    for (int r : in.owner) {
        if (r < 0 || r >= rows || (r >= C && r < OB))
            return fail(TG_ERR_INVALID, "periodic ghost owner row %d is neither an inner cell nor a halo row", r);
    }
    in.send_rows.assign(send_rows, send_rows + num_send);
    for (int r : in.send_rows) {
        if (r < 0 || r >= C) return fail(TG_ERR_INVALID, "send row %d is not an inner cell", r);
    }
    for (int f = 0; f < m->off_boundary_faces; f++) {
        const int l = m->face_cell[2 * f], r = m->face_cell[2 * f + 1];
        const bool inner = f < m->num_inner_faces;
        const bool l_ok = (l >= 0 && l < C) || (inner && l >= OB && l < rows);
        const bool r_ok = inner ? ((r >= 0 && r < C) || (r >= OB && r < rows)) : (r >= C && r < OB);
        if (!l_ok || !r_ok || (inner && l >= C && r >= C))
            return fail(TG_ERR_INVALID, "face %d references rows (%d, %d) outside the partition", f, l, r);
    }
    TRY(boundary_tables(m, e, in.bent, in.bkind, in.bctx));
    for (int k : in.bkind) {
        if (k == TG_BC_CUSTOM) return fail(TG_ERR_INVALID, "custom boundaries are not supported in a partition");
    }
    if (e->limiter == TG_LIMITER_VENKATAKRISHNAN) {
        in.eps2.resize(C);
        limiter_parameter(m, e, in.eps2.data());
    }
    in.inst_cell_off = {0, C};
    in.sum_volume = {m->sum_volume};
    in.inst_row_off = {0, m->num_cells};
    in.rowmap.resize(m->num_cells);
    for (int r = 0; r < m->num_cells; r++) in.rowmap[r] = r < OB ? r : in.owner[r - OB];
    in.halo = num_halo;
    return create_ctx(in, e, precision, out);
}

extern "C" int tg_batch_create(const tg_mesh *meshes, const tg_equations *eqns, int num, int precision,
                               tg_ctx **out)
{
    if (!out || !meshes || !eqns) return fail(TG_ERR_INVALID, "null argument");
    *out = nullptr;
    MeshInput in;
    TRY(merged_input(meshes, eqns, num, in));
    TRY(create_ctx(in, &eqns[0], precision, out));
    (*out)->batch = true;
    return TG_OK;
}

extern "C" int tg_batch_status(tg_ctx *c, int *status)
{
    if (!c || !status) return fail(TG_ERR_INVALID, "null argument");
    for (int i = 0; i < c->ninst; i++) status[i] = hi_at(c, SI_FAIL, i) ? TG_ERR_NONFINITE : TG_OK;
    return TG_OK;
}

extern "C" int tg_batch_size(tg_ctx *c, int *num)
{
    if (!c || !num) return fail(TG_ERR_INVALID, "null argument");
    *num = c->ninst;
    return TG_OK;
}

extern "C" int tg_destroy(tg_ctx *c)
{
    if (!c) return TG_OK;
    cudaStreamSynchronize(c->stream);
    free_ctx(c);
    return TG_OK;
}

extern "C" int tg_set_stream(tg_ctx *c, void *stream)
{
    if (!c) return fail(TG_ERR_INVALID, "null context");
    CU(cudaStreamSynchronize(c->stream));
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    drop_graph(c);
    c->graph_method = -1;
    return TG_OK;
}

extern "C" int tg_set_wait_limit(tg_ctx *c, int polls)
{
    if (!c) return fail(TG_ERR_INVALID, "null context");
    if (polls < 0) return fail(TG_ERR_INVALID, "the poll limit must be >= 0");
    c->wait_polls = polls > MBAR_POLLS ? MBAR_POLLS : polls;
    drop_graph(c);  // the limit is a kernel argument baked into the step graph
    return TG_OK;
}

// ---- host transfers --------------------------------------------------------------------------

static int ensure_pinned(tg_ctx *c, size_t n)
{
    if (c->pinned_len >= n) return TG_OK;
    if (c->pinned) cudaFreeHost(c->pinned);
    c->pinned = nullptr;
    c->pinned_len = 0;
    CU(cudaMallocHost(&c->pinned, n * sizeof(double)));
    c->pinned_len = n;
    return TG_OK;
}

// host AoS -> device (through pinned staging when the source is pageable)
static int h2d(tg_ctx *c, double *dst, const double *src, size_t n)
{
    cudaPointerAttributes at;
    bool pinned = cudaPointerGetAttributes(&at, src) == cudaSuccess && at.type == cudaMemoryTypeHost;
    cudaGetLastError();
    if (pinned) {
        CU(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        return TG_OK;
    }
    TRY(ensure_pinned(c, n));
    memcpy(c->pinned, src, n * sizeof(double));
    CU(cudaMemcpyAsync(dst, c->pinned, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return TG_OK;
}

static int d2h(tg_ctx *c, double *dst, const double *src, size_t n)
{
    cudaPointerAttributes at;
    bool pinned = cudaPointerGetAttributes(&at, dst) == cudaSuccess && at.type == cudaMemoryTypeHost;
    cudaGetLastError();
    if (pinned) {
        CU(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CU(cudaStreamSynchronize(c->stream));
        return TG_OK;
    }
    TRY(ensure_pinned(c, n));
    CU(cudaMemcpyAsync(c->pinned, src, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    memcpy(dst, c->pinned, n * sizeof(double));
    return TG_OK;
}

static int set_rows(tg_ctx *c, int inst, const double *prim, double *q)
{
    if (inst < 0 || inst >= c->ninst) return fail(TG_ERR_INVALID, "invalid instance %d", inst);
    int row0 = c->h_inst_cell_off[inst];
    int n = c->h_inst_cell_off[inst + 1] - row0;
    TRY(h2d(c, c->aos, prim, 5 * (size_t)n));
    k_rows_aos_to_soa<<<grid_of(n), BLOCK, 0, c->stream>>>(n, row0, c->s.N, c->aos, q);
    CU(cudaGetLastError());
    if (q == c->q && c->pref && n > 0) {
        // the FP32-flux form's reference pressure: the instance's first cell (any constant cancels
        // over closed cells; a representative one keeps the relative pressures small)
        double p0 = prim[4];
        c->h_pref[inst] = std::isfinite(p0) ? p0 : 0.0;
        CU(cudaMemcpyAsync(c->pref + inst, &c->h_pref[inst], sizeof(double), cudaMemcpyHostToDevice, c->stream));
    }
    return TG_OK;
}

extern "C" int tg_batch_set_primitive(tg_ctx *c, int inst, const double *prim)
{
    if (!c || !prim) return fail(TG_ERR_INVALID, "null argument");
    TRY(set_rows(c, inst, prim, c->q));
    hi_at(c, SI_FAIL, inst) = 0;  // a new state: the instance may run again
    c->prepared = false;
    return TG_OK;
}

extern "C" int tg_batch_get_primitive(tg_ctx *c, int inst, double *prim)
{
    if (!c || !prim) return fail(TG_ERR_INVALID, "null argument");
    if (inst < 0 || inst >= c->ninst) return fail(TG_ERR_INVALID, "invalid instance %d", inst);
    int r0 = c->inst_row_off[inst];
    int n = c->inst_row_off[inst + 1] - r0;
    k_rows_gather<<<grid_of(n), BLOCK, 0, c->stream>>>(n, c->rowmap + r0, c->s.N, c->q, c->aos);
    CU(cudaGetLastError());
    TRY(d2h(c, prim, c->aos, 5 * (size_t)n));
    return TG_OK;
}

extern "C" int tg_set_primitive(tg_ctx *c, const double *prim)
{
    if (c && c->ninst != 1) return fail(TG_ERR_INVALID, "a batch takes its state per instance");
    return tg_batch_set_primitive(c, 0, prim);
}

extern "C" int tg_get_primitive(tg_ctx *c, double *prim)
{
    if (c && c->ninst != 1) return fail(TG_ERR_INVALID, "a batch gives its state per instance");
    return tg_batch_get_primitive(c, 0, prim);
}

// ---- kernel sequencing -----------------------------------------------------------------------

static Props props_of(const tg_ctx *c)
{
    Props p;
    for (int i = 0; i < 3; i++) p.v[i] = c->prop[i];
    return p;
}

static bool is_ns(const tg_ctx *c)
{
    return c->physics == TG_NAVIERSTOKES;
}

// FP64 records and geometry (the plain and the exact FP64 forms)
static bool is_fp64(const tg_ctx *c)
{
    return c->precision != TG_PRECISION_FP32_FLUX;
}

static bool is_exact(const tg_ctx *c)
{
    return c->precision == TG_PRECISION_FP64_EXACT;
}

// teal's O2 path keeps the unlimited gradient only when a viscous flux needs it
static bool fold_psi(const tg_ctx *c)
{
    return !(c->viscous == TG_VISCOUS_CENTRAL) || c->limiter == TG_LIMITER_NONE;
}

// `masked`: inside a step sequence, where instances that have stopped keep their ghost rows
static int run_boundary(tg_ctx *c, double *q, bool masked = false)
{
    int nbf = c->s.F_bd - c->s.F_in;
    if (nbf <= 0) return TG_OK;
    Launch l(c, TG_PROF_BOUNDARY);
    if (is_exact(c)) {
        BoundaryLaunch a{c->s,   c->lr,      c->gb.basis, c->bface_ent, c->bkind, c->bctx, q,
                         c->prop[0], c->cell_inst, masked ? c->st.active : nullptr};
        CU(launch_boundary_exact(a, c->stream));
    }
    else {
        k_boundary<false><<<grid_of(nbf), BLOCK, 0, c->stream>>>(c->s, c->lr, c->gb.basis, c->bface_ent, c->bkind,
                                                                 c->bctx, q, c->prop[0], c->cell_inst,
                                                                 masked ? c->st.active : nullptr);
    }
    CU(cudaGetLastError());
    // custom boundaries: their device functions, face by face of each boundary
    for (size_t b = 0; b < c->bd_kernel.size(); b++) {
        if (!c->bd_kernel[b]) continue;
        int n = c->bd_range[b].second - c->bd_range[b].first, f0 = c->bd_range[b].first;
        if (n <= 0) continue;
        Launch lc(c, TG_PROF_BOUNDARY);
        const int *lr = reinterpret_cast<const int *>(c->lr);
        const double *centre = c->bcenter + 3 * (size_t)(f0 - c->s.F_in);
        long N = c->s.N;
        const int *active = masked ? c->st.active : nullptr;
        void *args[] = {&n, &f0, &lr, &centre, &q, &N, &c->dprop, &c->t_time, &c->t_step, &c->t_coef, &c->t_host,
                        &active};
        CU(cudaLaunchKernel(c->bd_kernel[b], dim3((n + 127) / 128), dim3(128), args, 0, c->stream));
    }
    return TG_OK;
}

// the context's sizes with the work range of its next cell-wise or face-wise launch
static Sizes cell_sizes(const tg_ctx *c)
{
    Sizes s = c->s;
    s.lo = c->cell_lo;
    s.hi = c->cell_hi < 0 ? c->s.C : c->cell_hi;
    return s;
}

static Sizes face_sizes(const tg_ctx *c)
{
    Sizes s = c->s;
    s.lo = c->face_lo;
    s.hi = c->face_hi < 0 ? c->s.F : c->face_hi;
    return s;
}

template <typename R, bool MIXED>
static void launch_gradient_s(tg_ctx *c, const Geometry<R> &g, bool fold, const double *q)
{
    const Sizes s = cell_sizes(c);
    if (s.hi <= s.lo) return;
    dim3 grid((s.hi - s.lo + GRAD_CELLS - 1) / GRAD_CELLS);
    R *rec = (R *)c->grad;
    switch (c->limiter) {
        case TG_LIMITER_NONE:
            k_gradient<R, 0, true, MIXED, false><<<grid, GRAD_THREADS, 0, c->stream>>>(s, g, c->eps2, q, rec, c->st.error, c->wait_polls);
            break;
        case TG_LIMITER_BARTH_JESPERSEN:
            if (fold)
                k_gradient<R, 1, true, MIXED, false><<<grid, GRAD_THREADS, 0, c->stream>>>(s, g, c->eps2, q, rec, c->st.error, c->wait_polls);
            else
                k_gradient<R, 1, false, MIXED, false><<<grid, GRAD_THREADS, 0, c->stream>>>(s, g, c->eps2, q, rec, c->st.error, c->wait_polls);
            break;
        default:
            if (fold)
                k_gradient<R, 2, true, MIXED, false><<<grid, GRAD_THREADS, 0, c->stream>>>(s, g, c->eps2, q, rec, c->st.error, c->wait_polls);
            else
                k_gradient<R, 2, false, MIXED, false><<<grid, GRAD_THREADS, 0, c->stream>>>(s, g, c->eps2, q, rec, c->st.error, c->wait_polls);
            break;
    }
}

template <typename R>
static void launch_gradient(tg_ctx *c, const Geometry<R> &g, bool fold, const double *q)
{
    if (c->full_slots)
        launch_gradient_s<R, false>(c, g, fold, q);
    else
        launch_gradient_s<R, true>(c, g, fold, q);
}

// gradient with an explicit limiter choice (tg_gradient reports the unlimited one on request)
static int run_gradient(tg_ctx *c, const double *q, int limiter_override = -1)
{
    int saved = c->limiter;
    if (limiter_override >= 0) c->limiter = limiter_override;
    bool fold = fold_psi(c);
    Launch l(c, TG_PROF_GRADIENT);
    if (is_exact(c)) {
        GradientLaunch a{cell_sizes(c), c->g64, c->eps2,  q, (double *)c->grad, c->limiter, fold, !c->full_slots,
                         c->st.error, c->wait_polls};
        cudaError_t e = launch_gradient_exact(a, c->stream);
        c->limiter = saved;
        CU(e);
        return TG_OK;
    }
    if (c->precision == TG_PRECISION_FP64)
        launch_gradient<double>(c, c->g64, fold, q);
    else
        launch_gradient<float>(c, c->g32, fold, q);
    c->limiter = saved;
    CU(cudaGetLastError());
    return TG_OK;
}

static int run_face(tg_ctx *c, const double *q)
{
    FaceLaunch a;
    a.s = face_sizes(c);
    a.geom = is_fp64(c) ? (const void *)&c->g64 : (const void *)&c->g32;
    a.q = q;
    a.rec = c->grad;
    a.gamma = c->prop[0];
    a.mu = c->prop[1];
    a.prandtl = c->prop[2];
    a.G = c->G;
    a.err = c->st.error;
    a.pr_ref = PressureRef{c->precision == TG_PRECISION_FP32_FLUX ? c->pref : nullptr, c->cell_inst};
    a.polls = c->wait_polls;
    bool ns = c->viscous == TG_VISCOUS_CENTRAL;
    bool fold = fold_psi(c);
    Launch l(c, TG_PROF_FACE);
    cudaError_t e;
    if (is_exact(c)) {
        switch (c->flux) {
            case TG_FLUX_ROE: e = launch_face_exact<FK_ROE>(ns, c->order, fold, a, c->stream); break;
            case TG_FLUX_HLL: e = launch_face_exact<FK_HLL>(ns, c->order, fold, a, c->stream); break;
            case TG_FLUX_HLLC: e = launch_face_exact<FK_HLLC>(ns, c->order, fold, a, c->stream); break;
            case TG_FLUX_HLLE: e = launch_face_exact<FK_HLLE>(ns, c->order, fold, a, c->stream); break;
            case TG_FLUX_AUSMD: e = launch_face_exact<FK_AUSMD>(ns, c->order, fold, a, c->stream); break;
            case TG_FLUX_AUSMDV: e = launch_face_exact<FK_AUSMDV>(ns, c->order, fold, a, c->stream); break;
            case TG_FLUX_LXF: e = launch_face_exact<FK_LXF>(ns, c->order, fold, a, c->stream); break;
            case TG_FLUX_CENTRAL: e = launch_face_exact<FK_CENTRAL>(ns, c->order, fold, a, c->stream); break;
            default: e = launch_face_exact<FK_NONE>(ns, c->order, fold, a, c->stream); break;
        }
        CU(e);
        return TG_OK;
    }
    switch (c->flux) {
        case TG_FLUX_ROE: e = launch_face<FK_ROE>(c->precision, ns, c->order, fold, a, c->stream); break;
        case TG_FLUX_HLL: e = launch_face<FK_HLL>(c->precision, ns, c->order, fold, a, c->stream); break;
        case TG_FLUX_HLLC: e = launch_face<FK_HLLC>(c->precision, ns, c->order, fold, a, c->stream); break;
        case TG_FLUX_HLLE: e = launch_face<FK_HLLE>(c->precision, ns, c->order, fold, a, c->stream); break;
        case TG_FLUX_AUSMD: e = launch_face<FK_AUSMD>(c->precision, ns, c->order, fold, a, c->stream); break;
        case TG_FLUX_AUSMDV: e = launch_face<FK_AUSMDV>(c->precision, ns, c->order, fold, a, c->stream); break;
        case TG_FLUX_LXF: e = launch_face<FK_LXF>(c->precision, ns, c->order, fold, a, c->stream); break;
        case TG_FLUX_CENTRAL: e = launch_face<FK_CENTRAL>(c->precision, ns, c->order, fold, a, c->stream); break;
        default: e = launch_face<FK_NONE>(c->precision, ns, c->order, fold, a, c->stream); break;
    }
    CU(e);
    return TG_OK;
}

template <int MODE, bool NS, typename GT, int SRC>
static void launch_cell_s(tg_ctx *c, double alpha, int last, double *q, double *Rout)
{
    CellData cd{c->volume, c->proj, c->eps2};
    Source src{{c->src_par[0], c->src_par[1], c->src_par[2], c->src_par[3]},
               c->source == TG_SOURCE_DEVICE ? c->S : c->src_avg};
    const Sizes s = cell_sizes(c);
    if (s.hi <= s.lo) return;
    k_cell<MODE, NS, GT, SRC, false><<<(s.hi - s.lo + CELL_BLOCK - 1) / CELL_BLOCK, CELL_BLOCK, 0, c->stream>>>(
        s, c->slot_face, c->slot_cnt, cd, (const GT *)c->G, c->U0, q, Rout, c->seg, c->st, alpha, last,
        props_of(c), c->dtc, src, 0);
}

template <int MODE, bool NS, typename GT>
static void launch_cell_t(tg_ctx *c, double alpha, int last, double *q, double *Rout)
{
    switch (c->source) {
        case TG_SOURCE_BODY_FORCE: launch_cell_s<MODE, NS, GT, 1>(c, alpha, last, q, Rout); break;
        case TG_SOURCE_BULK_FORCING: launch_cell_s<MODE, NS, GT, 2>(c, alpha, last, q, Rout); break;
        case TG_SOURCE_DEVICE: launch_cell_s<MODE, NS, GT, 3>(c, alpha, last, q, Rout); break;
        default: launch_cell_s<MODE, NS, GT, 0>(c, alpha, last, q, Rout); break;
    }
}

template <int MODE>
static int launch_cell(tg_ctx *c, double alpha, int last, double *q, double *Rout)
{
    Launch l(c, TG_PROF_CELL);
    bool ns = is_ns(c);
    if (is_exact(c)) {
        CellLaunch a;
        a.mode = MODE;
        a.ns = ns;
        a.source = c->source;
        a.two = (c->viscous == TG_VISCOUS_CENTRAL && c->order == 2) ? 1 : 0;
        a.s = cell_sizes(c);
        a.slot_face = c->slot_face;
        a.slot_cnt = c->slot_cnt;
        a.cd = CellData{c->volume, c->proj, c->eps2};
        a.G = (const double *)c->G;
        a.U0 = c->U0;
        a.q = q;
        a.Rout = Rout;
        a.seg = c->seg;
        a.st = c->st;
        a.alpha = alpha;
        a.last = last;
        a.prop = props_of(c);
        a.dtc = c->dtc;
        a.src = Source{{c->src_par[0], c->src_par[1], c->src_par[2], c->src_par[3]},
                       c->source == TG_SOURCE_DEVICE ? c->S : c->src_avg};
        CU(launch_cell_exact(a, c->stream));
        return TG_OK;
    }
    if (c->precision == TG_PRECISION_FP64) {
        if (ns)
            launch_cell_t<MODE, true, double>(c, alpha, last, q, Rout);
        else
            launch_cell_t<MODE, false, double>(c, alpha, last, q, Rout);
    }
    else {
        if (ns)
            launch_cell_t<MODE, true, float>(c, alpha, last, q, Rout);
        else
            launch_cell_t<MODE, false, float>(c, alpha, last, q, Rout);
    }
    CU(cudaGetLastError());
    return TG_OK;
}

// what a residual needs before its gradients: the sources' Prepare pass and values, the boundary pass
static int run_fluxes_pre(tg_ctx *c, double *q, bool masked)
{
    for (size_t b = 0; b < c->bd_kernel.size(); b++) {
        if (!c->bd_kernel[b] && c->bd_kind[b] == TG_BC_CUSTOM)
            return fail(TG_ERR_INVALID, "custom boundary %d has no device function (tg_bind_boundary_function)",
                        (int)b);
    }
    bool prepare_average = c->source == TG_SOURCE_BULK_FORCING ||
                           (c->source == TG_SOURCE_DEVICE && c->src_prepare == TG_PREPARE_AVERAGE);
    if (c->source == TG_SOURCE_DEVICE && !c->src_kernel)
        return fail(TG_ERR_INVALID, "the device source has no function (tg_bind_source_function)");
    if (prepare_average) {
        // the Prepare pass: volume averages of the state being differentiated, per instance
        Launch l(c, TG_PROF_REDUCE);
        k_piece_average<<<c->npieces, BLOCK, 0, c->stream>>>(c->seg, c->s.N, q, c->volume, c->part_sum);
        k_inst_average<<<(c->ninst + 127) / 128, 128, 0, c->stream>>>(c->seg, c->part_sum, c->src_avg);
        CU(cudaGetLastError());
    }
    if (c->source == TG_SOURCE_DEVICE) {
        // the source of every cell from the state being differentiated, added by the cell gather
        Launch l(c, TG_PROF_CELL);
        int C = c->s.C;
        long N = c->s.N;
        const double *qc = q;
        const double *avg = prepare_average ? c->src_avg : nullptr;
        void *args[] = {&C,         &c->ccenter, &qc,       &N,     &c->dprop, &c->t_time,
                        &c->t_step, &c->t_coef,  &c->t_host, &c->S, &avg};
        CU(cudaLaunchKernel(c->src_kernel, dim3((C + 127) / 128), dim3(128), args, 0, c->stream));
    }
    TRY(run_boundary(c, q, masked));
    return TG_OK;
}

// boundary pass, gradient + limiter, face fluxes: everything of a residual before the gather
static int run_fluxes(tg_ctx *c, double *q, bool masked = false)
{
    TRY(run_fluxes_pre(c, q, masked));
    if (c->order == 2) TRY(run_gradient(c, q));
    TRY(run_face(c, q));
    return TG_OK;
}

// per-piece reductions of the cell steps (and of V R^2 with `res`)
static int run_pieces(tg_ctx *c, int res)
{
    Launch l(c, TG_PROF_REDUCE);
    k_piece_reduce<<<c->npieces, BLOCK, 0, c->stream>>>(c->seg, c->s.C, c->dtc, c->R, c->volume, res, c->part_min,
                                                        c->part_sum);
    CU(cudaGetLastError());
    return TG_OK;
}

static int run_prepare(tg_ctx *c)
{
    CellData cd{c->volume, c->proj, c->eps2};
    if (is_exact(c))
        CU(launch_prepare_exact(is_ns(c), c->s, cd, c->q, c->U0, props_of(c), c->dtc, c->stream));
    else if (is_ns(c))
        k_prepare<true, false><<<grid_of(c->s.C), BLOCK, 0, c->stream>>>(c->s, cd, c->q, c->U0, props_of(c), c->dtc);
    else
        k_prepare<false, false><<<grid_of(c->s.C), BLOCK, 0, c->stream>>>(c->s, cd, c->q, c->U0, props_of(c), c->dtc);
    CU(cudaGetLastError());
    TRY(run_pieces(c, 0));
    c->prepared = true;
    return TG_OK;
}

// ---- step bookkeeping transfers ---------------------------------------------------------------

static int read_steps(tg_ctx *c)
{
    CU(cudaMemcpyAsync(c->hd, c->sd, sizeof(double) * SD_COUNT * c->ninst, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaMemcpyAsync(c->hi, c->si, sizeof(int) * (SI_COUNT * c->ninst + 2), cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return TG_OK;
}

static int write_steps(tg_ctx *c)
{
    CU(cudaMemcpyAsync(c->sd, c->hd, sizeof(double) * SD_COUNT * c->ninst, cudaMemcpyHostToDevice, c->stream));
    CU(cudaMemcpyAsync(c->si, c->hi, sizeof(int) * (SI_COUNT * c->ninst + 2), cudaMemcpyHostToDevice, c->stream));
    return TG_OK;
}

static int check_error(tg_ctx *c)
{
    int e = hi_error(c);
    if (e) {
        hi_error(c) = 0;
        write_steps(c);
        if (e & ERR_TIMEOUT) return fail(TG_ERR_TIMEOUT, "a device-side wait for staged face geometry gave up");
        if (e & ERR_LOOP_LIMIT)
            return fail(TG_ERR_TIMEOUT, "an implicit step reached the device limit of %d Newton iterations",
                        NEWTON_LOOP_LIMIT);
        // an instance of a batch whose state went non-finite has stopped on its own (tg_batch_status);
        // the other instances go on
        if (c->batch) return TG_OK;
        return fail(TG_ERR_NONFINITE, "non-finite time step or residual");
    }
    return TG_OK;
}

// residual[5] of instance i from the host mirror
static void residual_of(tg_ctx *c, int i, double *out)
{
    for (int v = 0; v < 5; v++) out[v] = c->hd[(size_t)SD_RESIDUAL * c->ninst + 5 * i + v];
}

// ---- public single-evaluation entry points ----------------------------------------------------

extern "C" int tg_derivative(tg_ctx *c, const double *prim, double *deriv, double time)
{
    if (!c || !deriv) return fail(TG_ERR_INVALID, "null argument");
    c->t_time = c->t_step = nullptr, c->t_host = time;  // time reaches the device functions only
    if (c->ninst != 1) return fail(TG_ERR_INVALID, "tg_derivative takes a single-mesh context");
    double *q = c->q;
    if (prim) {  // evaluate a host-given state in scratch memory; the resident state stays as it is
        if (!c->qs) {
            TRY(dalloc(&c->qs, 5 * (size_t)c->s.N));
            CU(cudaMemsetAsync(c->qs, 0, 5 * sizeof(double) * c->s.N, c->stream));
        }
        q = c->qs;
        TRY(set_rows(c, 0, prim, q));
    }
    TRY(run_fluxes(c, q));
    TRY(launch_cell<0>(c, 0.0, 0, q, c->R));
    k_soa5_to_aos<<<grid_of(c->s.C), BLOCK, 0, c->stream>>>(c->s.C, c->R, c->aos);
    CU(cudaGetLastError());
    TRY(d2h(c, deriv, c->aos, 5 * (size_t)c->s.C));
    TRY(read_steps(c));
    TRY(check_error(c));
    return TG_OK;
}

extern "C" int tg_gradient(tg_ctx *c, double time, int limited, double *gradient)
{
    if (!c || !gradient) return fail(TG_ERR_INVALID, "null argument");
    c->t_time = c->t_step = nullptr, c->t_host = time;  // for custom boundaries
    if (c->order != 2) return fail(TG_ERR_INVALID, "gradients exist only at space order 2");
    TRY(run_boundary(c, c->q));
    int lim = limited ? c->limiter : TG_LIMITER_NONE;
    TRY(run_gradient(c, c->q, lim));
    // a folded record already carries psi (or none was applied); an unfolded one gets it
    // multiplied in here
    const bool folded = lim == TG_LIMITER_NONE || c->viscous != TG_VISCOUS_CENTRAL;
    int limit = (limited && lim != TG_LIMITER_NONE && !folded) ? 1 : 0;
    if (is_fp64(c))
        k_grad_to_aos<double><<<grid_of(c->s.C), BLOCK, 0, c->stream>>>(c->s.C, (const double *)c->grad, limit,
                                                                        c->aos);
    else
        k_grad_to_aos<float><<<grid_of(c->s.C), BLOCK, 0, c->stream>>>(c->s.C, (const float *)c->grad, limit,
                                                                       c->aos);
    CU(cudaGetLastError());
    TRY(d2h(c, gradient, c->aos, 15 * (size_t)c->s.C));
    return TG_OK;
}

extern "C" int tg_timestep(tg_ctx *c, double *step)
{
    if (!c || !step) return fail(TG_ERR_INVALID, "null argument");
    TRY(run_prepare(c));
    TRY(read_steps(c));
    for (int i = 0; i < c->ninst; i++) {
        hd_at(c, SD_MAX_STEP, i) = DBL_MAX;
        hi_at(c, SI_ACTIVE, i) = 1;
    }
    c->st.use_max_time = 0;
    TRY(write_steps(c));
    k_inst_begin<<<c->ninst, INST_BLOCK, 0, c->stream>>>(c->seg, c->part_min, 1.0, c->st);
    CU(cudaGetLastError());
    TRY(read_steps(c));
    *step = hd_at(c, SD_STEP0, 0);
    return TG_OK;
}

extern "C" int tg_residual(tg_ctx *c, const double *deriv, double *residual)
{
    if (!c || !deriv || !residual) return fail(TG_ERR_INVALID, "null argument");
    if (c->ninst != 1) return fail(TG_ERR_INVALID, "tg_residual takes a single-mesh context");
    TRY(h2d(c, c->aos, deriv, 5 * (size_t)c->s.C));
    k_aos5_to_soa<<<grid_of(c->s.C), BLOCK, 0, c->stream>>>(c->s.C, c->aos, c->R);
    CU(cudaGetLastError());
    TRY(run_pieces(c, 1));
    k_inst_end<<<c->ninst, INST_BLOCK, 0, c->stream>>>(c->seg, c->part_sum, 0, c->st);
    CU(cudaGetLastError());
    TRY(read_steps(c));
    residual_of(c, 0, residual);
    c->prepared = false;  // the piece minima were recomputed from stale cell steps
    return TG_OK;
}

// ---- explicit steps --------------------------------------------------------------------------

static int rk_params(const tg_ctx *c, int method, const void *context, int *stages, const double **alpha)
{
    static const double euler_alpha[2] = {0.0, 1.0};
    if (method == TG_ADVANCE_EULER) {
        *stages = 1;
        *alpha = euler_alpha;
        return TG_OK;
    }
    int order = c->order, ns = c->order + 1;  // teal's default (src/simulation/set.c:88-96)
    if (context) {
        const tg_runge_kutta *rk = (const tg_runge_kutta *)context;
        order = rk->time_order;
        ns = rk->num_stages;
    }
    if (order < 1 || order > 3) return fail(TG_ERR_INVALID, "invalid time order (%d)", order);
    if (ns < 1 || ns > 6) return fail(TG_ERR_INVALID, "invalid number of stages (%d)", ns);
    *stages = ns;
    *alpha = LSERK_ALPHA[order - 1][ns - 1];
    return TG_OK;
}

// one explicit step of every active instance (U0 and the piece minima must be current)
static int enqueue_explicit_step(tg_ctx *c, int stages, const double *alpha, double courant)
{
    {
        Launch l(c, TG_PROF_REDUCE);
        k_inst_begin<<<c->ninst, INST_BLOCK, 0, c->stream>>>(c->seg, c->part_min, courant, c->st);
    }
    CU(cudaGetLastError());
    for (int i = 0; i < stages; i++) {
        // the residual of stage i at time + alpha_i step (advance.c:100)
        c->t_time = c->st.time, c->t_step = c->st.step, c->t_coef = alpha[i];
        TRY(run_fluxes(c, c->q, true));
        TRY(launch_cell<1>(c, alpha[i + 1], i == stages - 1, c->q, c->R));
    }
    TRY(run_pieces(c, 1));
    {
        Launch l(c, TG_PROF_REDUCE);
        k_inst_end<<<c->ninst, INST_BLOCK, 0, c->stream>>>(c->seg, c->part_sum, 1, c->st);
    }
    {
        Launch l(c, TG_PROF_REDUCE);
        k_count_active<<<1, 256, 0, c->stream>>>(c->ninst, c->st);
    }
    CU(cudaGetLastError());
    return TG_OK;
}

// one explicit step: a replay of the step's CUDA graph, or plain launches while events time them
static int launch_step(tg_ctx *c, int stages, const double *alpha, double courant)
{
    if (c->prof_on) return enqueue_explicit_step(c, stages, alpha, courant);
    CU(cudaGraphLaunch(c->graph, c->stream));
    c->launches += c->graph_kernels;
    return TG_OK;
}

static int step_graph(tg_ctx *c, int method, int stages, const double *alpha, double courant, int use_max_time)
{
    c->st.use_max_time = use_max_time;
    if (c->graph && c->graph_method == method && c->graph_stages == stages && c->graph_courant == courant &&
        c->graph_use_max_time == use_max_time) {
        return TG_OK;
    }
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    cudaGraph_t g;
    CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    long before = c->launches;
    bool prof = c->prof_on;
    c->prof_on = false;
    int rc = enqueue_explicit_step(c, stages, alpha, courant);
    c->prof_on = prof;
    c->graph_kernels = c->launches - before;
    c->launches = before;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (rc != TG_OK) {
        if (e == cudaSuccess) cudaGraphDestroy(g);
        return rc;
    }
    CU(e);
    cudaError_t e2 = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    CU(e2);
    c->graph_method = method;
    c->graph_stages = stages;
    c->graph_courant = courant;
    c->graph_use_max_time = use_max_time;
    return TG_OK;
}

static int implicit_step_all(tg_ctx *c, const void *context, double courant);
static int implicit_run(tg_ctx *c, const void *context, double courant, int most);

// one implicit step of a single mesh with the Advance semantics (time advanced by the step clipped
// to max_step; residual and unclipped step returned)
static int implicit_advance(tg_ctx *c, const void *context, double courant, double *time, double max_step,
                            double *residual, double *step0)
{
    hd_at(c, SD_TIME, 0) = *time;
    hd_at(c, SD_MAX_STEP, 0) = max_step;
    hd_at(c, SD_THRESHOLD, 0) = 0.0;
    hi_at(c, SI_ITER, 0) = 0;
    hi_at(c, SI_MAX_ITER, 0) = 0x7fffffff;
    hi_at(c, SI_ACTIVE, 0) = 1;
    hi_error(c) = 0;
    c->st.use_max_time = 0;
    TRY(write_steps(c));
    TRY(implicit_step_all(c, context, courant));
    TRY(read_steps(c));
    TRY(check_error(c));
    *time = hd_at(c, SD_TIME, 0);
    if (residual) residual_of(c, 0, residual);
    if (step0) *step0 = hd_at(c, SD_STEP0, 0);
    return TG_OK;
}

extern "C" int tg_advance(tg_ctx *c, int method, const void *context, double courant, double *time,
                          double max_step, double *residual, double *step0)
{
    if (!c || !time) return fail(TG_ERR_INVALID, "null argument");
    if (c->ninst != 1) return fail(TG_ERR_INVALID, "tg_advance takes a single-mesh context (batches: tg_batch_run)");
    if (!(courant > 0)) return fail(TG_ERR_INVALID, "invalid courant number (%g)", courant);
    if (method == TG_ADVANCE_IMPLICIT_EULER) {
        return implicit_advance(c, context, courant, time, max_step, residual, step0);
    }
    if (method != TG_ADVANCE_EULER && method != TG_ADVANCE_LSERK)
        return fail(TG_ERR_INVALID, "invalid advance method (%d)", method);
    int stages;
    const double *alpha;
    TRY(rk_params(c, method, context, &stages, &alpha));
    if (!c->prepared) TRY(run_prepare(c));
    hd_at(c, SD_TIME, 0) = *time;
    hd_at(c, SD_MAX_STEP, 0) = max_step;
    hd_at(c, SD_THRESHOLD, 0) = 0;
    hi_at(c, SI_ITER, 0) = 0;
    hi_at(c, SI_MAX_ITER, 0) = 0x7fffffff;
    hi_at(c, SI_ACTIVE, 0) = 1;
    hi_error(c) = 0;
    TRY(write_steps(c));
    TRY(step_graph(c, method, stages, alpha, courant, 0));
    TRY(launch_step(c, stages, alpha, courant));
    TRY(read_steps(c));
    TRY(check_error(c));
    *time = hd_at(c, SD_TIME, 0);
    if (residual) residual_of(c, 0, residual);
    if (step0) *step0 = hd_at(c, SD_STEP0, 0);
    return TG_OK;
}

// ---- steps with overlapped host copies ----------------------------------------------------------
//
// tg_advance_host takes one step from a host state to a host state. The new state goes down chunk
// by chunk while the last stage runs: that stage's face fluxes and cell updates run in chunks of
// consecutive cells, and each chunk's rows are copied to the host (copy stream) as soon as they are
// final. Every element is computed by the same kernel with the same operations as in an unsplit
// step, so the results are the same bits. (The first stage split the same way behind a chunked
// upload gained nothing: in teal's breadth-first cell order periodic links join cells far apart,
// so most chunks' gradients wait for chunks that arrive late, and each chunk costs a kernel tail.)

#ifndef TG_IO_CHUNKS
#define TG_IO_CHUNKS 8
#endif
constexpr int IO_CHUNKS = TG_IO_CHUNKS;

static uint64_t io_bit(int k) { return uint64_t(1) << k; }

static int build_io_plan(tg_ctx *c)
{
    const int C = c->s.C, F = c->s.F, Fin = c->s.F_in;
    std::unique_ptr<IoPlan> p(new IoPlan);
    // chunks of at least 64 gradient tiles
    int K = std::max(1, std::min(IO_CHUNKS, C / (64 * GRAD_CELLS)));
    const int per = ((C + K - 1) / K + GRAD_CELLS - 1) / GRAD_CELLS * GRAD_CELLS;
    K = (C + per - 1) / per;
    std::vector<int2> lr(F);
    if (F > 0) {
        CU(cudaMemcpyAsync(lr.data(), c->lr, sizeof(int2) * F, cudaMemcpyDeviceToHost, c->stream));
        CU(cudaStreamSynchronize(c->stream));
    }
    bool sorted = true;
    for (int f = 1; f < Fin && sorted; f++) sorted = lr[f].x >= lr[f - 1].x;
    if (!sorted) K = 1;  // face chunks need inner faces ordered by their left cell
    const int step = (K == 1) ? C : per;
    p->K = K;
    p->cell_off.resize(K + 1);
    p->face_off.resize(K + 1);
    for (int k = 0; k <= K; k++) p->cell_off[k] = std::min(C, k * step);
    for (int k = 0; k < K; k++) {
        int lo = 0, hi = Fin;  // first inner face whose left cell is >= cell_off[k]
        while (lo < hi) {
            int mid = lo + (hi - lo) / 2;
            if (lr[mid].x < p->cell_off[k]) lo = mid + 1;
            else hi = mid;
        }
        p->face_off[k] = lo;
    }
    p->face_off[0] = 0;
    p->face_off[K] = Fin;
    auto chunk = [&](int cell) { return std::min(K - 1, cell / step); };
    p->cell_face.assign(K, 0);
    for (int f = 0; f < Fin; f++) {
        const int kl = chunk(lr[f].x), kr = chunk(lr[f].y);
        p->cell_face[kl] |= io_bit(kl);
        p->cell_face[kr] |= io_bit(kl);
    }
    CU(cudaStreamCreateWithFlags(&p->copy, cudaStreamNonBlocking));
    p->ev.resize(K + 1, nullptr);
    for (int k = 0; k <= K; k++) CU(cudaEventCreateWithFlags(&p->ev[k], cudaEventDisableTiming));
    c->io = p.release();
    return TG_OK;
}

static bool host_pinned(const void *ptr)
{
    cudaPointerAttributes at;
    bool pinned = cudaPointerGetAttributes(&at, ptr) == cudaSuccess && at.type == cudaMemoryTypeHost;
    cudaGetLastError();
    return pinned;
}

// the step with its last stage in chunks, each chunk's rows copied into the pinned host array `out`
// (or none with out == null); on return the copy stream has finished (also after an error)
static int advance_chunked(tg_ctx *c, int stages, const double *alpha, double courant, double *out)
{
    IoPlan &p = *c->io;
    const int K = p.K, C = c->s.C, Fin = c->s.F_in, F = c->s.F;
    const long N = c->s.N;
    const int rows = c->inst_row_off[1];
    std::vector<char> fl(K, 0);
    {
        Launch l(c, TG_PROF_REDUCE);
        k_inst_begin<<<c->ninst, INST_BLOCK, 0, c->stream>>>(c->seg, c->part_min, courant, c->st);
    }
    CU(cudaGetLastError());
    // the stages before the last one as in an unsplit step
    int i = 0;
    for (; i < stages - 1; i++) {
        c->t_time = c->st.time, c->t_step = c->st.step, c->t_coef = alpha[i];
        TRY(run_fluxes(c, c->q, true));
        TRY(launch_cell<1>(c, alpha[i + 1], 0, c->q, c->R));
    }
    // the last stage: sources, boundary ghosts, gradients and the boundary and periodic faces whole,
    // then the inner faces and the cell updates chunk by chunk
    c->t_time = c->st.time, c->t_step = c->st.step, c->t_coef = alpha[i];
    TRY(run_fluxes_pre(c, c->q, true));
    if (c->order == 2) TRY(run_gradient(c, c->q));
    c->face_lo = Fin, c->face_hi = F;
    TRY(run_face(c, c->q));
    for (int k = 0; k < K; k++) {
        for (int j = 0; j < K; j++) {
            if (!fl[j] && (p.cell_face[k] & io_bit(j))) {
                c->face_lo = p.face_off[j], c->face_hi = p.face_off[j + 1];
                TRY(run_face(c, c->q));
                fl[j] = 1;
            }
        }
        c->cell_lo = p.cell_off[k], c->cell_hi = p.cell_off[k + 1];
        TRY(launch_cell<1>(c, alpha[i + 1], 1, c->q, c->R));
        c->cell_lo = 0, c->cell_hi = -1;
        if (out) {
            const int r0 = p.cell_off[k], n = p.cell_off[k + 1] - r0;
            k_rows_gather<<<grid_of(n), BLOCK, 0, c->stream>>>(n, c->rowmap + r0, (int)N, c->q, c->aos + 5 * (size_t)r0);
            CU(cudaGetLastError());
            CU(cudaEventRecord(p.ev[k], c->stream));
            CU(cudaStreamWaitEvent(p.copy, p.ev[k], 0));
            CU(cudaMemcpyAsync(out + 5 * (size_t)r0, c->aos + 5 * (size_t)r0, sizeof(double) * 5 * (size_t)n,
                               cudaMemcpyDeviceToHost, p.copy));
        }
    }
    c->face_lo = 0, c->face_hi = -1;
    // ghost rows (boundary ghosts as the last boundary pass left them, periodic ghosts from their owners)
    if (out && rows > C) {
        const int n = rows - C;
        k_rows_gather<<<grid_of(n), BLOCK, 0, c->stream>>>(n, c->rowmap + C, (int)N, c->q, c->aos + 5 * (size_t)C);
        CU(cudaGetLastError());
        CU(cudaEventRecord(p.ev[K], c->stream));
        CU(cudaStreamWaitEvent(p.copy, p.ev[K], 0));
        CU(cudaMemcpyAsync(out + 5 * (size_t)C, c->aos + 5 * (size_t)C, sizeof(double) * 5 * (size_t)n,
                           cudaMemcpyDeviceToHost, p.copy));
    }
    TRY(run_pieces(c, 1));
    {
        Launch l(c, TG_PROF_REDUCE);
        k_inst_end<<<c->ninst, INST_BLOCK, 0, c->stream>>>(c->seg, c->part_sum, 1, c->st);
    }
    {
        Launch l(c, TG_PROF_REDUCE);
        k_count_active<<<1, 256, 0, c->stream>>>(c->ninst, c->st);
    }
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(p.copy));
    return TG_OK;
}

extern "C" int tg_advance_host(tg_ctx *c, int method, const void *context, double courant, double *time,
                               double max_step, const double *prim_in, double *prim_out, double *residual,
                               double *step0)
{
    if (!c || !time) return fail(TG_ERR_INVALID, "null argument");
    if (c->ninst != 1)
        return fail(TG_ERR_INVALID, "tg_advance_host takes a single-mesh context (batches: tg_batch_run)");
    if (prim_in) TRY(tg_set_primitive(c, prim_in));
    // the last stage runs in chunks when the new state goes to pinned host memory (pageable memory
    // goes through the staging buffer in one piece)
    const bool chunked = (method == TG_ADVANCE_EULER || method == TG_ADVANCE_LSERK) && c->halo == 0 &&
                         c->nsend == 0 && !c->prof_on && prim_out && host_pinned(prim_out);
    if (!chunked) {
        TRY(tg_advance(c, method, context, courant, time, max_step, residual, step0));
        if (prim_out) TRY(tg_get_primitive(c, prim_out));
        return TG_OK;
    }
    if (!(courant > 0)) return fail(TG_ERR_INVALID, "invalid courant number (%g)", courant);
    int stages;
    const double *alpha;
    TRY(rk_params(c, method, context, &stages, &alpha));
    if (!c->io) TRY(build_io_plan(c));
    if (!c->prepared) TRY(run_prepare(c));
    hd_at(c, SD_TIME, 0) = *time;
    hd_at(c, SD_MAX_STEP, 0) = max_step;
    hd_at(c, SD_THRESHOLD, 0) = 0;
    hi_at(c, SI_ITER, 0) = 0;
    hi_at(c, SI_MAX_ITER, 0) = 0x7fffffff;
    hi_at(c, SI_ACTIVE, 0) = 1;
    hi_error(c) = 0;
    TRY(write_steps(c));
    const int rc = advance_chunked(c, stages, alpha, courant, prim_out);
    c->cell_lo = 0, c->cell_hi = -1, c->face_lo = 0, c->face_hi = -1;
    if (rc != TG_OK) {
        // nothing may still write into the caller's buffer once this returns
        cudaStreamSynchronize(c->stream);
        cudaStreamSynchronize(c->io->copy);
        return rc;
    }
    TRY(read_steps(c));
    TRY(check_error(c));
    *time = hd_at(c, SD_TIME, 0);
    if (residual) residual_of(c, 0, residual);
    if (step0) *step0 = hd_at(c, SD_STEP0, 0);
    return TG_OK;
}

// run loop over every instance: each stops on its own limits; the host replays the step graph
// and checks the number of active instances every `every` steps
static int run_instances(tg_ctx *c, int method, const void *context, double courant, int max_launch, int every)
{
    int stages;
    const double *alpha;
    TRY(rk_params(c, method, context, &stages, &alpha));
    if (!c->prepared) TRY(run_prepare(c));
    TRY(write_steps(c));
    TRY(step_graph(c, method, stages, alpha, courant, 1));
    for (int it = 0; it < max_launch;) {
        int n = (max_launch - it < every) ? max_launch - it : every;
        for (int k = 0; k < n; k++) TRY(launch_step(c, stages, alpha, courant));
        it += n;
        TRY(read_steps(c));
        TRY(check_error(c));
        if (hi_num_active(c) == 0) break;
    }
    TRY(read_steps(c));
    TRY(check_error(c));
    c->prepared = false;  // cells of stopped instances carry no current step estimate
    return TG_OK;
}

extern "C" int tg_run(tg_ctx *c, int method, const void *context, double courant, int max_iter,
                      double max_time, int variable, double threshold, double *time, int *iter,
                      double *residual)
{
    if (!c || !time || !iter) return fail(TG_ERR_INVALID, "null argument");
    if (c->ninst != 1) return fail(TG_ERR_INVALID, "tg_run takes a single-mesh context (batches: tg_batch_run)");
    if (variable < -1 || variable > 4) return fail(TG_ERR_INVALID, "invalid termination variable");
    if (!(courant > 0)) return fail(TG_ERR_INVALID, "invalid courant number (%g)", courant);
    if (method != TG_ADVANCE_EULER && method != TG_ADVANCE_LSERK && method != TG_ADVANCE_IMPLICIT_EULER)
        return fail(TG_ERR_INVALID, "invalid advance method (%d)", method);
    if (max_iter <= 0) {
        *iter = 0;
        return TG_OK;
    }
    hd_at(c, SD_TIME, 0) = *time;
    hd_at(c, SD_MAX_TIME, 0) = max_time;
    hd_at(c, SD_THRESHOLD, 0) = threshold;
    hi_at(c, SI_VARIABLE, 0) = variable;
    hi_at(c, SI_ITER, 0) = 0;
    hi_at(c, SI_MAX_ITER, 0) = max_iter;
    hi_at(c, SI_ACTIVE, 0) = 1;
    hi_error(c) = 0;
    if (method == TG_ADVANCE_IMPLICIT_EULER) {
        // implicit steps synchronise inside the Newton loop anyway; the stop tests run every step
        c->st.use_max_time = 1;
        TRY(implicit_run(c, context, courant, max_iter));
    }
    else {
        // stop tests that can end the run early are polled every step, a fixed count only at the end
        int every = (threshold > 0 || max_time < DBL_MAX) ? 1 : max_iter;
        TRY(run_instances(c, method, context, courant, max_iter, every));
    }
    *time = hd_at(c, SD_TIME, 0);
    *iter = hi_at(c, SI_ITER, 0);
    if (residual) residual_of(c, 0, residual);
    return TG_OK;
}

extern "C" int tg_last_step(tg_ctx *c, int instance, double *step0)
{
    if (!c || !step0) return fail(TG_ERR_INVALID, "null argument");
    if (instance < 0 || instance >= c->ninst) return fail(TG_ERR_INVALID, "invalid instance (%d)", instance);
    TRY(read_steps(c));
    *step0 = hd_at(c, SD_STEP0, instance);
    return TG_OK;
}

extern "C" int tg_batch_run(tg_ctx *c, int method, const void *context, double courant, const int *max_iter,
                            const double *max_time, const int *variable, const double *threshold, double *time,
                            int *iter, double *residual)
{
    if (!c || !max_iter || !time || !iter) return fail(TG_ERR_INVALID, "null argument");
    if (method != TG_ADVANCE_EULER && method != TG_ADVANCE_LSERK && method != TG_ADVANCE_IMPLICIT_EULER)
        return fail(TG_ERR_INVALID, "invalid advance method (%d)", method);
    if (!(courant > 0)) return fail(TG_ERR_INVALID, "invalid courant number (%g)", courant);
    int most = 0;
    bool early = false;
    for (int i = 0; i < c->ninst; i++) {
        int var = variable ? variable[i] : -1;
        if (var < -1 || var > 4) return fail(TG_ERR_INVALID, "invalid termination variable of instance %d", i);
        hd_at(c, SD_TIME, i) = time[i];
        hd_at(c, SD_MAX_TIME, i) = max_time ? max_time[i] : DBL_MAX;
        hd_at(c, SD_THRESHOLD, i) = threshold ? threshold[i] : 0.0;
        hi_at(c, SI_VARIABLE, i) = var;
        hi_at(c, SI_ITER, i) = 0;
        hi_at(c, SI_MAX_ITER, i) = max_iter[i];
        hi_at(c, SI_ACTIVE, i) = max_iter[i] > 0 && !hi_at(c, SI_FAIL, i);  // failed instances stay stopped
        most = max_iter[i] > most ? max_iter[i] : most;
        early = early || hd_at(c, SD_THRESHOLD, i) > 0 || hd_at(c, SD_MAX_TIME, i) < DBL_MAX;
    }
    hi_error(c) = 0;
    if (most > 0 && method == TG_ADVANCE_IMPLICIT_EULER) {
        c->st.use_max_time = 1;
        TRY(implicit_run(c, context, courant, most));
    }
    else if (most > 0) {
        TRY(run_instances(c, method, context, courant, most, early ? 8 : most));
    }
    for (int i = 0; i < c->ninst; i++) {
        time[i] = hd_at(c, SD_TIME, i);
        iter[i] = hi_at(c, SI_ITER, i);
        if (residual) residual_of(c, i, residual + 5 * i);
    }
    return TG_OK;
}

// ---- implicit Euler with Jacobian-free Newton-GMRES (advance.c:119-195, gmres.c:52-149) --------
//
// Every instance of the arena takes its own implicit step at once: its own CFL step, Newton and
// Arnoldi iterations that stop on their own tests, masked out of the vector updates once done.
// The host loops over Newton and Arnoldi iterations and reads, once per iteration, how many
// instances go on.

static int gm_alloc(tg_ctx *c, int dim)
{
    Gmres &g = c->gm;
    if (g.V && g.dim >= dim) return TG_OK;
    void *old[] = {g.U, g.Ustart, g.r, g.delta, g.V, g.w, g.q1, g.R1, g.part, g.sc, g.flag, g.count, g.ctl, g.Rm};
    for (void *p : old) {
        if (p) cudaFree(p);
    }
    g = Gmres{};
    size_t n = 5 * (size_t)c->s.C;
    TRY(dalloc(&g.U, n));
    TRY(dalloc(&g.Ustart, n));
    TRY(dalloc(&g.r, n));
    TRY(dalloc(&g.delta, n));
    TRY(dalloc(&g.V, (size_t)(dim + 1) * n));
    TRY(dalloc(&g.w, n));
    TRY(dalloc(&g.q1, 5 * (size_t)c->s.N));
    CU(cudaMemset(g.q1, 0, 5 * sizeof(double) * c->s.N));
    TRY(dalloc(&g.R1, n));
    TRY(dalloc(&g.part, (size_t)c->npieces));
    TRY(dalloc(&g.sc, (size_t)c->ninst * gmres_scn(dim)));
    TRY(dalloc(&g.flag, (size_t)GF_COUNT * c->ninst));
    CU(cudaMemset(g.flag, 0, sizeof(int) * GF_COUNT * c->ninst));
    TRY(dalloc(&g.count, 2));
    TRY(dalloc(&g.ctl, GC_COUNT));
    CU(cudaMemset(g.ctl, 0, sizeof(int) * GC_COUNT));
    if (c->precision == TG_PRECISION_FP32_FLUX) TRY(dalloc(&g.Rm, n));
    g.dim = dim;
    drop_graph(c);  // a captured implicit step refers to the old workspace
    return TG_OK;
}

static GmresBatch gm_batch(tg_ctx *c, int dim)
{
    return GmresBatch{dim, gmres_scn(dim), c->ninst, c->cell_inst, c->gm.sc, c->gm.flag, c->gm.count, c->gm.ctl};
}

// sc[instance][slot] = x . y (or its square root) for the instances whose flag `which` is set
static int gm_dot(tg_ctx *c, const GmresBatch &gb, const double *x, const double *y, int which, int slot,
                  int take_sqrt)
{
    k_piece_dot<<<c->npieces, BLOCK, 0, c->stream>>>(c->seg, c->s.C, x, y, gb, which, c->gm.part);
    k_inst_dot<<<c->ninst, GM_INST_BLOCK, 0, c->stream>>>(c->seg, c->gm.part, gb, which, slot, take_sqrt);
    CU(cudaGetLastError());
    return TG_OK;
}

static int inst_grid(const tg_ctx *c)
{
    return (c->ninst + 127) / 128;
}

// ---- device-driven loops of a captured graph ---------------------------------------------------
//
// A loop whose trip count only the device knows becomes a conditional WHILE node of the graph
// being captured on c->stream: while_begin creates the node's condition handle in that graph,
// enqueues `init` (a kernel that sets the condition before the node runs, every time the node is
// reached), appends the node and captures its body on a side stream until while_end. The body's
// last kernel sets the condition for the next round.

struct WhileLoop {
    cudaStream_t outer = nullptr;
    cudaGraphConditionalHandle h = 0;
};

template <typename Init>
static int while_begin(tg_ctx *c, WhileLoop &w, int depth, Init init)
{
    cudaStreamCaptureStatus status;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    CU(cudaStreamGetCaptureInfo(c->stream, &status, nullptr, &graph, &deps, &ndeps));
    if (status != cudaStreamCaptureStatusActive) return fail(TG_ERR_INVALID, "device loops need a stream capture");
    CU(cudaGraphConditionalHandleCreate(&w.h, graph, 0, 0));
    init(w.h);
    CU(cudaGetLastError());
    CU(cudaStreamGetCaptureInfo(c->stream, &status, nullptr, &graph, &deps, &ndeps));
    cudaGraphNodeParams params = {};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = w.h;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    CU(cudaGraphAddNode(&node, graph, deps, ndeps, &params));
    CU(cudaStreamUpdateCaptureDependencies(c->stream, &node, 1, cudaStreamSetCaptureDependencies));
    if (!c->cap_stream[depth]) CU(cudaStreamCreateWithFlags(&c->cap_stream[depth], cudaStreamNonBlocking));
    w.outer = c->stream;
    c->stream = c->cap_stream[depth];
    cudaError_t e = cudaStreamBeginCaptureToGraph(c->stream, params.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        c->stream = w.outer;
        CU(e);
    }
    return TG_OK;
}

static int while_end(tg_ctx *c, WhileLoop &w)
{
    cudaGraph_t body = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &body);
    c->stream = w.outer;
    CU(e);
    return TG_OK;
}

// derivative of a primitive state q (boundary rows refreshed) into Rout, with the kernels of
// `precision` (the context's own, or FP64 for the FP32-flux form's Newton residuals)
static int gm_derivative(tg_ctx *c, double *q, double *Rout, int precision)
{
    // implicit Euler evaluates every residual at the end of the step, time + step (advance.c:144)
    c->t_time = c->st.time, c->t_step = c->st.step, c->t_coef = 1.0;
    const int own = c->precision;
    c->precision = precision;
    int rc = run_fluxes(c, q);
    if (rc == TG_OK) rc = launch_cell<0>(c, 0.0, 0, q, Rout);
    c->precision = own;
    return rc;
}

// the Newton residual's precision: FP64 in the FP32-flux form, whose FP32 fluxes serve the matvec
// only ("FP64 Arnoldi, FP32 matvec flux": the Newton iteration then converges to the FP64 state)
static int newton_precision(const tg_ctx *c)
{
    return c->precision == TG_PRECISION_FP32_FLUX ? TG_PRECISION_FP64 : c->precision;
}

// one GMRES cycle for the increment of every Newton instance (gmres.c:52-149): the Arnoldi
// iterations and each column's Gram-Schmidt rows are device loops (a finished instance is masked
// out of every vector update); each Gram-Schmidt dot is fused with the update of the row before it
static int gm_solve(tg_ctx *c, const GmresBatch &gb, double krylov_tol)
{
    Gmres &g = c->gm;
    const int C = c->s.C, cb = grid_of(C), ib = inst_grid(c);
    k_gmres_begin<<<ib, 128, 0, c->stream>>>(gb, krylov_tol);
    k_gmres_start<<<cb, BLOCK, 0, c->stream>>>(C, g.r, gb, g.V, g.delta);
    CU(cudaGetLastError());
    c->launches += 2;
    WhileLoop arnoldi;
    TRY(while_begin(c, arnoldi, 1, [&](cudaGraphConditionalHandle h) {
        k_arnoldi_enter<<<1, 256, 0, c->stream>>>(gb, h);
        c->launches += 1;
    }));
    {
        // matvec (gmres.c:12-50)
        k_piece_vnorm<<<c->npieces, BLOCK, 0, c->stream>>>(c->seg, C, g.V, gb, g.part);
        k_inst_dot_at<<<c->ninst, GM_INST_BLOCK, 0, c->stream>>>(c->seg, g.part, gb, 2);
        k_perturb_at<<<cb, BLOCK, 0, c->stream>>>(C, c->s.N, g.U, g.V, gb, c->prop[0], g.q1);
        CU(cudaGetLastError());
        c->launches += 3;
        TRY(gm_derivative(c, g.q1, g.R1, c->precision));
        // the matvec differences two residuals of the same precision (gmres.c:41-46)
        k_matvec_finish_at<<<cb, BLOCK, 0, c->stream>>>(C, g.V, g.R1, g.Rm ? g.Rm : c->R, gb, g.w);
        CU(cudaGetLastError());
        c->launches += 1;
        // modified Gram-Schmidt rows 0..k
        WhileLoop mgs;
        TRY(while_begin(c, mgs, 2, [&](cudaGraphConditionalHandle h) {
            k_mgs_enter<<<1, 1, 0, c->stream>>>(gb, h);
            c->launches += 1;
        }));
        k_mgs_piece<<<c->npieces, BLOCK, 0, c->stream>>>(c->seg, C, g.V, gb, 0, g.w, g.part);
        k_inst_dot_at<<<c->ninst, GM_INST_BLOCK, 0, c->stream>>>(c->seg, g.part, gb, 0);
        k_mgs_next<<<1, 1, 0, c->stream>>>(gb, mgs.h);
        CU(cudaGetLastError());
        c->launches += 3;
        TRY(while_end(c, mgs));
        // the last row's update and the norm of w
        k_mgs_piece<<<c->npieces, BLOCK, 0, c->stream>>>(c->seg, C, g.V, gb, 1, g.w, g.part);
        k_inst_dot_at<<<c->ninst, GM_INST_BLOCK, 0, c->stream>>>(c->seg, g.part, gb, 1);
        CU(cudaMemsetAsync(g.count + 1, 0, sizeof(int), c->stream));
        k_givens_at<<<ib, 128, 0, c->stream>>>(gb);
        k_normalize_at<<<cb, BLOCK, 0, c->stream>>>(C, g.w, gb, g.V);
        k_arnoldi_next<<<1, 1, 0, c->stream>>>(gb, arnoldi.h);
        CU(cudaGetLastError());
        c->launches += 5;
    }
    TRY(while_end(c, arnoldi));
    k_backsolve<<<ib, 128, 0, c->stream>>>(gb);
    k_accumulate<<<cb, BLOCK, 0, c->stream>>>(C, g.V, gb, g.delta);
    CU(cudaGetLastError());
    c->launches += 2;
    return TG_OK;
}

static int newton_params(const void *context, double *newton_tol, double *krylov_tol, int *dim)
{
    *newton_tol = 0.1, *krylov_tol = 0.3, *dim = 32;  // teal's defaults (src/simulation/set.c:113-115)
    if (context) {
        const tg_newton_krylov *nk = (const tg_newton_krylov *)context;
        *newton_tol = nk->newton_tolerance;
        *krylov_tol = nk->krylov_tolerance;
        *dim = nk->krylov_dimension;
    }
    if (!(*newton_tol > 0)) return fail(TG_ERR_INVALID, "invalid newton tolerance (%g)", *newton_tol);
    if (!(*krylov_tol > 0)) return fail(TG_ERR_INVALID, "invalid krylov tolerance (%g)", *krylov_tol);
    if (*dim <= 0) return fail(TG_ERR_INVALID, "invalid krylov dimension (%d)", *dim);
    return TG_OK;
}

// One implicit Euler step of every active instance (advance.c:119-195), enqueued on a capturing
// stream: CFL step, Newton iterations (a device loop) with a GMRES solve each, then the residual
// norm and the run loop's time / iteration / stop bookkeeping (k_inst_end). The device step arrays
// must be current when the graph runs.
static int enqueue_implicit_step(tg_ctx *c, double courant, double newton_tol, double krylov_tol, int dim)
{
    Gmres &g = c->gm;
    const GmresBatch gb = gm_batch(c, dim);
    const int C = c->s.C, cb = grid_of(C), ib = inst_grid(c);
    const size_t n = 5 * (size_t)C;
    // finite-difference perturbation relative to the state: teal's 1e-6 (advance.c:157) in FP64;
    // the FP32-flux form's residual carries ~1e-7 relative rounding, so it perturbs by 3e-4
    const double fd_rel = is_fp64(c) ? 1e-6 : 3e-4;

    // step from the CFL condition; U = cons(q) (advance.c:136-143)
    TRY(run_prepare(c));
    {
        Launch l(c, TG_PROF_REDUCE);
        k_inst_begin<<<c->ninst, INST_BLOCK, 0, c->stream>>>(c->seg, c->part_min, courant, c->st);
    }
    k_newton_begin<<<ib, 128, 0, c->stream>>>(gb, c->st);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(g.U, c->U0, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    CU(cudaMemcpyAsync(g.Ustart, c->U0, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    c->prepared = false;

    TRY(gm_derivative(c, c->q, c->R, newton_precision(c)));
    if (g.Rm) TRY(gm_derivative(c, c->q, g.Rm, c->precision));
    k_newton_init<<<cb, BLOCK, 0, c->stream>>>(C, c->R, gb, g.r);
    CU(cudaGetLastError());
    TRY(gm_dot(c, gb, g.r, g.r, GF_NEWTON, GS_NORM, 1));
    TRY(gm_dot(c, gb, g.U, g.U, GF_NEWTON, GS_CONS_NORM, 1));
    k_fd_scale<<<ib, 128, 0, c->stream>>>(gb, fd_rel, newton_tol, 1);
    CU(cudaGetLastError());
    c->launches += 4;
    auto newton_check = [&](cudaGraphConditionalHandle h, int enter) {
        cudaMemsetAsync(g.count, 0, sizeof(int), c->stream);
        k_newton_check<<<ib, 128, 0, c->stream>>>(gb, c->seg, c->st);
        k_newton_next<<<1, 1, 0, c->stream>>>(gb, h, enter, c->st.error);
        c->launches += 2;
    };
    WhileLoop newton;
    TRY(while_begin(c, newton, 0, [&](cudaGraphConditionalHandle h) { newton_check(h, 1); }));
    {
        TRY(gm_solve(c, gb, krylov_tol));
        k_newton_update<<<cb, BLOCK, 0, c->stream>>>(C, c->s.N, g.U, g.delta, gb, c->prop[0], c->q);
        CU(cudaGetLastError());
        TRY(gm_derivative(c, c->q, c->R, newton_precision(c)));
        if (g.Rm) TRY(gm_derivative(c, c->q, g.Rm, c->precision));
        k_newton_residual<<<cb, BLOCK, 0, c->stream>>>(C, g.U, g.Ustart, c->R, gb, g.r);
        CU(cudaGetLastError());
        TRY(gm_dot(c, gb, g.r, g.r, GF_NEWTON, GS_NORM, 1));
        TRY(gm_dot(c, gb, g.U, g.U, GF_NEWTON, GS_CONS_NORM, 1));
        k_fd_scale<<<ib, 128, 0, c->stream>>>(gb, fd_rel, newton_tol, 0);
        CU(cudaGetLastError());
        c->launches += 3;
        newton_check(newton.h, 0);
        CU(cudaGetLastError());
    }
    TRY(while_end(c, newton));
    // residual of the last derivative (advance.c:188), time, iteration and the run loop's tests
    TRY(run_pieces(c, 1));
    {
        Launch l(c, TG_PROF_REDUCE);
        k_inst_end<<<c->ninst, INST_BLOCK, 0, c->stream>>>(c->seg, c->part_sum, 1, c->st);
        k_count_active<<<1, 256, 0, c->stream>>>(c->ninst, c->st);
    }
    CU(cudaGetLastError());
    return TG_OK;
}

// One implicit Euler step of every active instance: a replay of the step's graph, captured on first
// use for these parameters. The host waits for nothing inside the step.
static int implicit_step_all(tg_ctx *c, const void *context, double courant)
{
    double newton_tol, krylov_tol;
    int dim;
    TRY(newton_params(context, &newton_tol, &krylov_tol, &dim));
    TRY(gm_alloc(c, dim));
    if (!(c->igraph && c->ig_courant == courant && c->ig_newton_tol == newton_tol &&
          c->ig_krylov_tol == krylov_tol && c->ig_dim == dim && c->ig_use_max_time == c->st.use_max_time)) {
        if (c->igraph) {
            cudaGraphExecDestroy(c->igraph);
            c->igraph = nullptr;
        }
        cudaGraph_t graph;
        CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const long before = c->launches;
        const bool prof = c->prof_on;
        c->prof_on = false;  // no event records inside the graph
        cudaStream_t outer = c->stream;
        int rc = enqueue_implicit_step(c, courant, newton_tol, krylov_tol, dim);
        c->stream = outer;  // restored even when a loop body's capture failed half way
        c->prof_on = prof;
        if (rc != TG_OK) {  // close loop-body captures left open by the failure
            for (cudaStream_t side : c->cap_stream) {
                cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
                if (side && cudaStreamIsCapturing(side, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
                    cudaGraph_t body = nullptr;
                    cudaStreamEndCapture(side, &body);
                }
            }
            cudaGetLastError();
        }
        c->igraph_kernels = c->launches - before;
        c->launches = before;
        cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
        if (rc != TG_OK) {
            if (e == cudaSuccess) cudaGraphDestroy(graph);
            return rc;
        }
        CU(e);
        cudaError_t e2 = cudaGraphInstantiate(&c->igraph, graph, 0);
        cudaGraphDestroy(graph);
        CU(e2);
        c->ig_courant = courant, c->ig_newton_tol = newton_tol, c->ig_krylov_tol = krylov_tol;
        c->ig_dim = dim, c->ig_use_max_time = c->st.use_max_time;
    }
    CU(cudaGraphLaunch(c->igraph, c->stream));
    c->launches += c->igraph_kernels;
    c->prepared = false;
    return TG_OK;
}

// implicit steps of every instance until each one stops (iterations, residual threshold, end time)
static int implicit_run(tg_ctx *c, const void *context, double courant, int most)
{
    TRY(write_steps(c));
    // stopped instances sit out the following steps on the device, so the host looks in only every
    // 8 steps (and at the end)
    for (int it = 0; it < most;) {
        const int n = most - it < 8 ? most - it : 8;
        for (int k = 0; k < n; k++) TRY(implicit_step_all(c, context, courant));
        it += n;
        TRY(read_steps(c));
        TRY(check_error(c));
        if (hi_num_active(c) == 0) break;
    }
    return TG_OK;
}

// ---- profiling ---------------------------------------------------------------------------------

extern "C" int tg_profile(tg_ctx *c, int enable)
{
    if (!c) return fail(TG_ERR_INVALID, "null context");
    CU(cudaStreamSynchronize(c->stream));
    for (auto &p : c->prof_open) {
        c->prof_pool.push_back(p.second.first);
        c->prof_pool.push_back(p.second.second);
    }
    c->prof_open.clear();
    for (int i = 0; i < TG_PROF_CATEGORIES; i++) {
        c->prof_ms[i] = 0;
        c->prof_n[i] = 0;
    }
    c->prof_on = enable != 0;
    return TG_OK;
}

extern "C" int tg_profile_read(tg_ctx *c, double *ms, long *launches)
{
    if (!c) return fail(TG_ERR_INVALID, "null context");
    CU(cudaStreamSynchronize(c->stream));
    for (auto &p : c->prof_open) {
        float t = 0;
        CU(cudaEventElapsedTime(&t, p.second.first, p.second.second));
        c->prof_ms[p.first] += t;
        c->prof_n[p.first] += 1;
        c->prof_pool.push_back(p.second.first);
        c->prof_pool.push_back(p.second.second);
    }
    c->prof_open.clear();
    for (int i = 0; i < TG_PROF_CATEGORIES; i++) {
        if (ms) ms[i] = c->prof_ms[i];
        if (launches) launches[i] = c->prof_n[i];
    }
    return TG_OK;
}

extern "C" int tg_launch_count(tg_ctx *c, long *count)
{
    if (!c || !count) return fail(TG_ERR_INVALID, "null argument");
    *count = c->launches;
    return TG_OK;
}

// ---- layout introspection --------------------------------------------------------------------

extern "C" int tg_layout(tg_ctx *c, const char *name, void *out, long count)
{
    if (!c || !name || !out) return fail(TG_ERR_INVALID, "null argument");
    const void *src = nullptr;
    size_t bytes = 0, pitch = 0;  // pitch: row length of a pitched [6][SL] slot array
    long expect = 0;
    if (!strcmp(name, "face_lr")) {
        src = c->lr, expect = 2L * c->s.F, bytes = sizeof(int);
    }
    else if (!strcmp(name, "slot_face")) {
        src = c->slot_face, expect = (long)MAX_SLOTS * c->s.C, bytes = sizeof(int), pitch = c->s.SL;
    }
    else if (!strcmp(name, "slot_nbr")) {
        src = c->slot_nbr, expect = (long)MAX_SLOTS * c->s.C, bytes = sizeof(int), pitch = c->s.SL;
    }
    else if (!strcmp(name, "slot_cnt")) {
        src = c->slot_cnt, expect = c->s.C, bytes = 1;
    }
    else if (!strcmp(name, "owner")) {
        src = c->owner, expect = c->num_periodic, bytes = sizeof(int);
    }
    else if (!strcmp(name, "tile_slots")) {
        // slots of each gradient tile (32 cells), from the tiles' byte offsets
        const long ntiles = (c->s.C + GRAD_CELLS - 1) / GRAD_CELLS;
        if (count != ntiles) return fail(TG_ERR_INVALID, "layout array %s has %ld elements, not %ld", name, ntiles, count);
        std::vector<long long> off(ntiles + 1);
        CU(cudaMemcpyAsync(off.data(), c->gb.toff64, sizeof(long long) * (ntiles + 1), cudaMemcpyDeviceToHost,
                           c->stream));
        CU(cudaStreamSynchronize(c->stream));
        int *o = static_cast<int *>(out);
        for (long t = 0; t < ntiles; t++) o[t] = int((off[t + 1] - off[t]) / grad_tile_bytes<double>(1));
        return TG_OK;
    }
    else {
        return fail(TG_ERR_INVALID, "unknown layout array (%s)", name);
    }
    if (count != expect) return fail(TG_ERR_INVALID, "layout array %s has %ld elements, not %ld", name, expect, count);
    if (count == 0) return TG_OK;
    if (pitch) {
        // returned unpitched, [6][C]
        CU(cudaMemcpy2DAsync(out, bytes * c->s.C, src, bytes * pitch, bytes * c->s.C, MAX_SLOTS,
                             cudaMemcpyDeviceToHost, c->stream));
    }
    else {
        CU(cudaMemcpyAsync(out, src, bytes * count, cudaMemcpyDeviceToHost, c->stream));
    }
    CU(cudaStreamSynchronize(c->stream));
    return TG_OK;
}

// ---- drop-in Advance methods ------------------------------------------------------------------

struct Binding {
    tg_ctx *ctx;
    double *host_primitive;
    bool registered;  // page-locked in place by tg_bind (the step's copies then reach it directly)
};
static std::map<const void *, Binding> g_bindings;
static std::mutex g_bind_mutex;

extern "C" int tg_bind(const void *eqns, tg_ctx *c, double *host_primitive)
{
    if (!eqns || !c || !host_primitive) return fail(TG_ERR_INVALID, "null argument");
    if (c->ninst != 1) return fail(TG_ERR_INVALID, "tg_bind takes a single-mesh context");
    TRY(tg_set_primitive(c, host_primitive));
    std::lock_guard<std::mutex> lock(g_bind_mutex);
    auto old = g_bindings.find(eqns);
    if (old != g_bindings.end() && old->second.registered) cudaHostUnregister(old->second.host_primitive);
    // teal's primitive array (teal_calloc, pageable) is page-locked in place, so each step's state
    // goes down into it by DMA, chunk by chunk while the last stage runs; where that is refused the
    // copies go through the context's pinned staging buffer
    const size_t bytes = sizeof(double) * 5 * (size_t)c->inst_row_off[1];
    bool reg = !host_pinned(host_primitive) &&
               cudaHostRegister(host_primitive, bytes, cudaHostRegisterDefault) == cudaSuccess;
    cudaGetLastError();
    g_bindings[eqns] = Binding{c, host_primitive, reg};
    return TG_OK;
}

extern "C" int tg_unbind(const void *eqns)
{
    std::lock_guard<std::mutex> lock(g_bind_mutex);
    auto it = g_bindings.find(eqns);
    if (it != g_bindings.end()) {
        if (it->second.registered) cudaHostUnregister(it->second.host_primitive);
        g_bindings.erase(it);
    }
    return TG_OK;
}

static double dropin(int method, const void *eqns, double *time, void *residual, double max_step,
                     double courant, const void *context)
{
    Binding b{nullptr, nullptr, false};
    {
        std::lock_guard<std::mutex> lock(g_bind_mutex);
        auto it = g_bindings.find(eqns);
        if (it != g_bindings.end()) b = it->second;
    }
    double step0 = 0;
    int rc = b.ctx ? TG_OK : fail(TG_ERR_INVALID, "equations are not bound to a device context");
    // the step, with the new state copied into teal's array while the last stage runs
    if (rc == TG_OK)
        rc = tg_advance_host(b.ctx, method, context, courant, time, max_step, nullptr, b.host_primitive,
                             (double *)residual, &step0);
    if (rc != TG_OK) {
        fprintf(stderr, "[0] ERROR: %s\n", tg_last_error());
        fflush(stderr);
        exit(EXIT_FAILURE);
    }
    return step0;
}

extern "C" double tg_teal_euler(const void *eqns, double *time, void *residual, double max_step,
                                double courant, const void *context)
{
    return dropin(TG_ADVANCE_EULER, eqns, time, residual, max_step, courant, context);
}

extern "C" double tg_teal_lserk(const void *eqns, double *time, void *residual, double max_step,
                                double courant, const void *context)
{
    return dropin(TG_ADVANCE_LSERK, eqns, time, residual, max_step, courant, context);
}

extern "C" double tg_teal_implicit_euler(const void *eqns, double *time, void *residual, double max_step,
                                         double courant, const void *context)
{
    return dropin(TG_ADVANCE_IMPLICIT_EULER, eqns, time, residual, max_step, courant, context);
}

// ---- partitions: the phases of an RK stage around the caller's halo exchange --------------------

// device pointers of the exchange buffers: states [send][5] / [halo][5] (FP64) and gradient records
// [send][20] / [halo][20] of `record_bytes` / 20 bytes each
extern "C" int tg_part_buffers(tg_ctx *c, void **send_q, void **recv_q, void **send_rec, void **recv_rec,
                               long *record_bytes)
{
    if (!c) return fail(TG_ERR_INVALID, "null context");
    if (send_q) *send_q = c->send_q;
    if (recv_q) *recv_q = c->recv_q;
    if (send_rec) *send_rec = c->send_rec;
    if (recv_rec) *recv_rec = c->recv_rec;
    if (record_bytes) *record_bytes = 20 * (long)(is_fp64(c) ? sizeof(double) : sizeof(float));
    return TG_OK;
}

// the cells' stable steps of the current state (U0 refreshed first when the state changed) and
// their minimum over this partition's cells, in piece order
extern "C" int tg_part_step_begin(tg_ctx *c, double *local_min)
{
    if (!c || !local_min) return fail(TG_ERR_INVALID, "null argument");
    if (!c->prepared) TRY(run_prepare(c));
    else TRY(run_pieces(c, 0));
    std::vector<double> part(c->npieces);
    CU(cudaMemcpyAsync(part.data(), c->part_min, sizeof(double) * c->npieces, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    double m = DBL_MAX;
    for (double v : part) m = fmin(m, v);
    *local_min = m;
    return TG_OK;
}

// the step every rank takes (courant times the minimum over all ranks, clipped) and the time
extern "C" int tg_part_set_step(tg_ctx *c, double step, double time)
{
    if (!c) return fail(TG_ERR_INVALID, "null context");
    if (!(step > 0) || !std::isfinite(step)) return fail(TG_ERR_NONFINITE, "non-finite time step");
    hd_at(c, SD_STEP, 0) = step;
    hd_at(c, SD_STEP0, 0) = step;
    hd_at(c, SD_TIME, 0) = time;
    hi_at(c, SI_ACTIVE, 0) = 1;
    TRY(write_steps(c));
    return TG_OK;
}

// One RK stage in three phases, with the halo exchange between them done by the caller:
//   0  boundary states, then pack the sent rows' states into send_q
//   1  unpack recv_q into the halo rows, gradients and limiter, pack the sent rows' records
//   2  unpack recv_rec into the halo records, face fluxes, cell gather and the stage update
//      U = U0 + alpha step R (the last stage also refreshes U0 and the cells' stable steps)
extern "C" int tg_part_phase(tg_ctx *c, int phase, double alpha, int last)
{
    if (!c) return fail(TG_ERR_INVALID, "null context");
    const int N = c->s.N, h0 = N - c->halo;
    const bool f64 = is_fp64(c);
    if (phase == 0) {
        TRY(run_boundary(c, c->q));
        if (c->nsend) k_halo_pack_q<<<grid_of(c->nsend), BLOCK, 0, c->stream>>>(c->nsend, c->send_rows, N, c->q, c->send_q);
    }
    else if (phase == 1) {
        if (c->halo) k_halo_unpack_q<<<grid_of(c->halo), BLOCK, 0, c->stream>>>(c->halo, h0, N, c->recv_q, c->q);
        CU(cudaGetLastError());
        if (c->order == 2) {
            TRY(run_gradient(c, c->q));
            if (c->nsend && f64)
                k_halo_pack_rec<double><<<grid_of(c->nsend), BLOCK, 0, c->stream>>>(
                    c->nsend, c->send_rows, (const double *)c->grad, (double *)c->send_rec);
            else if (c->nsend)
                k_halo_pack_rec<float><<<grid_of(c->nsend), BLOCK, 0, c->stream>>>(
                    c->nsend, c->send_rows, (const float *)c->grad, (float *)c->send_rec);
        }
    }
    else if (phase == 2) {
        if (c->order == 2 && c->halo) {
            if (f64)
                k_halo_unpack_rec<double><<<grid_of(c->halo), BLOCK, 0, c->stream>>>(
                    c->halo, h0, (const double *)c->recv_rec, (double *)c->grad);
            else
                k_halo_unpack_rec<float><<<grid_of(c->halo), BLOCK, 0, c->stream>>>(
                    c->halo, h0, (const float *)c->recv_rec, (float *)c->grad);
        }
        CU(cudaGetLastError());
        TRY(run_face(c, c->q));
        TRY(launch_cell<1>(c, alpha, last, c->q, c->R));
        c->prepared = last != 0;  // the last stage leaves U0 and the cells' steps current
    }
    else {
        return fail(TG_ERR_INVALID, "invalid phase %d", phase);
    }
    CU(cudaGetLastError());
    return TG_OK;
}

// sums of volume * R^2 per variable over this partition's cells (the last stage's derivative), in
// piece order; the norm is sqrt(sum over all ranks / total volume)
extern "C" int tg_part_residual_sums(tg_ctx *c, double *sums)
{
    if (!c || !sums) return fail(TG_ERR_INVALID, "null argument");
    TRY(run_pieces(c, 1));
    std::vector<double> part(5 * (size_t)c->npieces);
    CU(cudaMemcpyAsync(part.data(), c->part_sum, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    for (int k = 0; k < 5; k++) {
        double t = 0;
        for (int p = 0; p < c->npieces; p++) t += part[5 * (size_t)p + k];
        sums[k] = t;
    }
    return TG_OK;
}

// teal's low-storage RK coefficients alpha[0..stages] of (order, stages) (advance.c:50-75)
extern "C" int tg_lserk_alpha(int order, int stages, double *alpha)
{
    if (!alpha || order < 1 || order > 3 || stages < 1 || stages > 6)
        return fail(TG_ERR_INVALID, "invalid lserk order %d / stages %d", order, stages);
    for (int i = 0; i <= stages; i++) alpha[i] = LSERK_ALPHA[order - 1][stages - 1][i];
    return TG_OK;
}

extern "C" int tg_stream_of(tg_ctx *c, void **stream)
{
    if (!c || !stream) return fail(TG_ERR_INVALID, "null argument");
    *stream = (void *)c->stream;
    return TG_OK;
}
