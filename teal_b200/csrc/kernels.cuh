// Kernels of the residual / time-integration path. One thread per cell or per face; every sum over
// a cell's faces runs through that cell's slot list in face order, so results are deterministic
// and need no floating-point atomics.
#pragma once

#include "common.cuh"
#include "tma.cuh"

namespace tg {

// ---- boundary pass (src/equations/boundary.c:5-43) -------------------------------------------

// With `active` (inside a step sequence), faces of instances that have stopped keep their ghost
// rows: a stopped instance's state, ghosts included, is what it was when it stopped.
// X (here and in the kernels below): the instantiation of the exact translation units.
template <bool X>
__global__ void k_boundary(Sizes s, const int2 *__restrict__ lr, const double *__restrict__ basis,
                           const int *__restrict__ bface_ent, const int *__restrict__ bkind,
                           const double *__restrict__ bctx, double *q, double gamma,
                           const int *__restrict__ cell_inst, const int *__restrict__ active)
{
    static_assert(X == kExact, "exact kernels live in the exact translation units only");
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int f = s.F_in + i;
    if (f >= s.F_bd) {
        return;
    }
    int2 c = lr[f];
    if (active && !active[cell_inst[c.x]]) {
        return;
    }
    int e = bface_ent[i];
    const int kind = bkind[e];
    if (kind == BC_CUSTOM) {  // written by the boundary's device function
        return;
    }
    Prim<double> in = load_prim<double>(q, s.N, c.x);
    Basis<double> b = load_basis(basis, s.F, f);
    Prim<double> ctx = prim_from(bctx + 5 * e);
    Prim<double> out = boundary_state(kind, in, ctx, gamma, b);
    store_prim(q, s.N, c.y, out);
}

// ---- least-squares gradient + limiter (src/equations/gradient.c:7-58, limiter.c:23-113) -------
//
// One thread per (cell, variable): a block of 5 x 32 threads covers 32 consecutive cells, warp w
// handling variable w, so each warp reads one contiguous row of the state. The mesh upload packed
// the slot geometry of every 32 cells (neighbour rows, least-squares weights, face offsets) into one
// contiguous tile with as many slots as the tile's cell with the most faces (grad_tile_bytes; no
// padding slots beyond that on mixed meshes). One thread stages the block's tile with bulk
// asynchronous copies completing on an mbarrier (a bounded wait: a block that gives up sets
// ERR_TIMEOUT in the error word and ends); the five variable warps then read it from shared memory.
// On meshes of hexahedra the threads read their neighbour rows from the tile in global memory and
// gather the neighbours' states while the weights and offsets are still on their way. Each
// gradient component is summed over the cell's slots in face order, as teal's face loop adds it.
// Output: one gradient record per cell, (gx, gy, gz, psi) per variable (grad_rec_store); FOLD
// multiplies psi in (Euler: only the limited gradient is used), otherwise the record keeps the
// unlimited gradient for the viscous flux.
constexpr int GRAD_CELLS = 32;
constexpr int GRAD_THREADS = 5 * GRAD_CELLS;

template <typename R, int LIM, bool FOLD, bool MIXED, bool X>
__global__ void __launch_bounds__(GRAD_THREADS, GRAD_MINB) k_gradient(Sizes s, Geometry<R> g,
                                                           const double *__restrict__ eps2,
                                                           const double *__restrict__ q,
                                                           R *__restrict__ rec, int *err, int polls)
{
    static_assert(X == kExact, "exact kernels live in the exact translation units only");
    __shared__ __align__(16) int s_nbr[MIXED ? MAX_SLOTS : 1][GRAD_CELLS];
    __shared__ __align__(16) R s_w[3 * MAX_SLOTS][GRAD_CELLS];
    __shared__ __align__(16) R s_off[(LIM != 0) ? 3 * MAX_SLOTS : 1][GRAD_CELLS];
    __shared__ int s_cnt[MIXED ? GRAD_CELLS : 1];
    __shared__ uint64_t bar;
    __shared__ int s_J;
    const int tile = s.lo / GRAD_CELLS + blockIdx.x;
    const int base = tile * GRAD_CELLS;
    const int ncell = min(GRAD_CELLS, s.hi - base);
    const int v = threadIdx.x / GRAD_CELLS;  // variable of this warp
    const int l = threadIdx.x % GRAD_CELLS;
    const int c = base + min(l, ncell - 1);
    const double *qv = q + (size_t)v * s.N;
    double qn[MAX_SLOTS];
    if constexpr (MIXED) {
        // the whole tile by bulk copies; its slot count is the tile's largest, so a warp of
        // tetrahedra stops after 4
        if (threadIdx.x == 0) {
            const long long t0 = __ldg(g.gtile_off + tile);
            const int J = int((__ldg(g.gtile_off + tile + 1) - t0) / grad_tile_bytes<R>(1));
            s_J = J;
            const unsigned char *tile_p = g.gtile + t0;
            const uint32_t nb = uint32_t(grad_tile_nbr_bytes<R>(J)), vb = uint32_t(grad_tile_vec_bytes<R>(J));
            mbar_init(&bar, 1);
            mbar_arrive_expect_tx(&bar, nb + vb + (LIM != 0 ? vb : 0u));
            bulk_g2s(&s_nbr[0][0], tile_p, nb, &bar);
            bulk_g2s(&s_w[0][0], tile_p + nb, vb, &bar);
            if (LIM != 0) {
                bulk_g2s(&s_off[0][0], tile_p + nb + vb, vb, &bar);
            }
        }
        if (threadIdx.x < GRAD_CELLS) {
            s_cnt[threadIdx.x] = (threadIdx.x < ncell) ? int(g.slot_cnt[base + threadIdx.x]) : 0;
        }
    }
    else {
        // hexahedra only: every tile has MAX_SLOTS slots (the slot tests below fold away). The weights
        // and offsets come by bulk copies; meanwhile the threads read their neighbour rows from the
        // tile's first part themselves and gather the neighbours' states (padding slots name the
        // cell itself), so the gathers overlap the copies
        const unsigned char *tile_p = g.gtile + (size_t)tile * (size_t)grad_tile_bytes<R>(MAX_SLOTS);
        constexpr uint32_t nb = uint32_t(grad_tile_nbr_bytes<R>(MAX_SLOTS));
        constexpr uint32_t vb = uint32_t(grad_tile_vec_bytes<R>(MAX_SLOTS));
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            mbar_arrive_expect_tx(&bar, vb + (LIM != 0 ? vb : 0u));
            bulk_g2s(&s_w[0][0], tile_p + nb, vb, &bar);
            if (LIM != 0) {
                bulk_g2s(&s_off[0][0], tile_p + nb + vb, vb, &bar);
            }
        }
        const int *nbr = reinterpret_cast<const int *>(tile_p);
#pragma unroll
        for (int j = 0; j < MAX_SLOTS; j++) {
            qn[j] = __ldg(qv + __ldg(nbr + j * GRAD_CELLS + l));
        }
    }
    // the cell's own state does not depend on the tile: its load overlaps the copies
    const double qc = __ldg(qv + c);
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0, polls);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) {
            atomicOr(err, ERR_TIMEOUT);
        }
        mbar_wait_bounded(&bar, 0, MBAR_POLLS);  // let copies still in flight land before the block exits
        return;
    }
    if (l >= ncell) {
        return;
    }
    const int cnt = MIXED ? s_cnt[l] : MAX_SLOTS;
    const int jmax = MIXED ? s_J : MAX_SLOTS;
    if constexpr (MIXED) {
#pragma unroll
        for (int j = 0; j < MAX_SLOTS; j++) {
            if (j >= jmax) break;
            qn[j] = __ldg(qv + ((j < cnt) ? s_nbr[j][l] : c));
        }
    }
    R gx = R(0), gy = R(0), gz = R(0);
    double mn = qc, mx = qc;
#pragma unroll
    for (int j = 0; j < MAX_SLOTS; j++) {
        if (j >= jmax) break;
        if (j < cnt) {
            R d = R(qn[j] - qc);
            gx += d * s_w[3 * j + 0][l];
            gy += d * s_w[3 * j + 1][l];
            gz += d * s_w[3 * j + 2][l];
            mn = fmin(mn, qn[j]);
            mx = fmax(mx, qn[j]);
        }
    }

    // limiter factor: the minimum over the cell's faces of teal's candidate ratios. Each candidate
    // is a fraction num / den with num >= 0 and den > 0 (delta1 has delta2's sign or is zero):
    //   Barth-Jespersen  min(1, delta1 / delta2) = |delta1| / |delta2|, the 1 by psi's start value
    //                    (limiter.c:54-58);
    //   Venkatakrishnan  top / bot / delta2 (limiter.c:100-106) with delta2 divided out of top:
    //                    (d1 (d1 + 2 d2) + eps2) / (d1 (d1 + d2) + 2 d2^2 + eps2), every term >= 0.
    // The running minimum stays a fraction compared by cross multiplication and is divided once:
    // one division per thread instead of one or two per face, within a few ulps of teal's per-face
    // quotients (FP32: a product underflows only for candidates below about 1e-30, where a fraction
    // of 0 and its rounding do not change the minimum; FP32 ramp-batch gradient 0.626 -> 0.517 ms).
    R psi = R(1);
    if (X && LIM != 0) {
        // teal's own candidates, one quotient per face (limiter.c:54-58, :100-106)
        const R e2 = (LIM == 2) ? R(__ldg(eps2 + c)) : R(0);
#pragma unroll
        for (int j = 0; j < MAX_SLOTS; j++) {
            if (j >= jmax) break;
            if (j < cnt) {
                R d2 = ((gx * s_off[3 * j + 0][l]) + (gy * s_off[3 * j + 1][l])) + (gz * s_off[3 * j + 2][l]);
                if (!is_close_zero(d2)) {
                    const R d1 = ((d2 > R(0)) ? R(mx) : R(mn)) - R(qc);
                    if (LIM == 1) {
                        psi = fmin(psi, fmin(R(1), d1 / d2));
                    }
                    else {
                        const R top = (((d1 * d1) + e2) * d2) + ((R(2) * (d2 * d2)) * d1);
                        const R bot = (((d1 * d1) + (R(2) * (d2 * d2))) + (d1 * d2)) + e2;
                        psi = fmin(psi, (top / bot) / d2);
                    }
                }
            }
        }
    }
    else if (LIM != 0) {
        const R e2 = (LIM == 2) ? R(__ldg(eps2 + c)) : R(0);
        const R dmx = R(mx - qc), dmn = R(mn - qc);
        R best_n = R(1), best_d = R(1);
#pragma unroll
        for (int j = 0; j < MAX_SLOTS; j++) {
            if (j >= jmax) break;
            if (j < cnt) {
                R d2 = ((gx * s_off[3 * j + 0][l]) + (gy * s_off[3 * j + 1][l])) + (gz * s_off[3 * j + 2][l]);
                if (!is_close_zero(d2)) {
                    const R d1 = (d2 > R(0)) ? dmx : dmn;
                    R num, den;
                    if (LIM == 1) {
                        num = fabs(d1);
                        den = fabs(d2);
                    }
                    else {
                        num = fma(d1, fma(R(2), d2, d1), e2);
                        den = fma(d1, d1 + d2, fma(d2 + d2, d2, e2));
                    }
                    if (num * best_d < best_n * den) {
                        best_n = num;
                        best_d = den;
                    }
                }
            }
        }
        psi = best_n / best_d;
    }
    if (FOLD && LIM != 0) {
        gx *= psi;
        gy *= psi;
        gz *= psi;
    }
    grad_rec_store(rec, c, v, gx, gy, gz, psi);
}

// per-cell time step of the equations' Timestep plugin
template <bool NS>
__device__ __forceinline__ double cell_timestep(const Prim<double> &p, const double *prop,
                                                const CellData &cd, int C, int c)
{
    double vol = __ldg(cd.volume + c);
    V3<double> proj = load_v3(cd.projection, C, c);
    if (NS) {
        return navierstokes_timestep(p, prop[0], prop[1], prop[2], vol, proj);
    }
    return euler_timestep(p, prop[0], vol, proj);
}

struct Props {
    double v[3];
};

// ---- cell gather, finalize and stage update (derivative.c:229-267, advance.c:96-108) ---------
//
// MODE 0: R = -sum / V (equations_derivative); MODE 1: one low-storage RK stage
// U = U0 + R * alpha * step, q = prim(U), with the step of the cell's instance (cells of inactive
// instances keep their state). With `last`, also: R kept, U0 <- cons(q) for the next step and the
// cell's stable time step of the new state.
// Device source terms in place of teal's Compute / Prepare callbacks (src/equations.h:27-41):
// kind TG_SOURCE_BODY_FORCE (p = acceleration) or TG_SOURCE_BULK_FORCING (p = target x velocity,
// time scale; avg = per-instance volume average of the primitive state being differentiated)
struct Source {
    double p[4];
    const double *avg;  // [ninst][5] volume averages (bulk forcing), or [5][C] values (device source)
};

// R += S(q) as teal's finalize_derivative adds source[j] to -sum / V (derivative.c:260-265)
template <int SRC>
__device__ __forceinline__ void add_source(const Source &src, const Prim<double> &q, int inst, double (&r)[5])
{
    double sv[5] = {0, 0, 0, 0, 0};
    if (SRC == 1) {  // body force (run/rayleigh_taylor_instability/run.c:17-24)
        sv[1] = src.p[0] * q.rho;
        sv[2] = src.p[1] * q.rho;
        sv[3] = src.p[2] * q.rho;
        sv[4] = ((sv[1] * q.u.x) + (sv[2] * q.u.y)) + (sv[3] * q.u.z);
    }
    else if (SRC == 2) {  // bulk forcing (run/periodic_hill/run.c:8-21)
        const double s1 = (q.rho * (src.p[0] - src.avg[5 * inst + 1])) / src.p[1];
        sv[1] = s1;
        sv[4] = q.u.x * s1;
    }
#pragma unroll
    for (int v = 0; v < 5; v++) {
        r[v] = r[v] + sv[v];
    }
}

// X (exact translation units): with `two` (a viscous flux), the viscous records (second set) are summed
// before the convective ones, the order of teal's two face loops, and R = -sum / V is a quotient.
template <int MODE, bool NS, typename GT, int SRC, bool X>
__global__ void __launch_bounds__(CELL_BLOCK, CELL_MINB) k_cell(Sizes s, const int *__restrict__ slot_face,
                                                const uint8_t *__restrict__ slot_cnt, CellData cd,
                                                const GT *__restrict__ G, double *__restrict__ U0,
                                                double *__restrict__ q, double *__restrict__ Rout,
                                                Segments seg, Steps st, double alpha, int last, Props prop,
                                                double *__restrict__ dtc, Source src, int two)
{
    static_assert(X == kExact, "exact kernels live in the exact translation units only");
    const int C = s.C, N = s.N;
    int c = s.lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= s.hi) {
        return;
    }
    // the stage update's inputs do not depend on the face records: their loads are issued first so
    // that their latency overlaps the record gathers
    int inst = 0, act = 1;
    double step = 0.0;
    if (MODE != 0) {
        inst = __ldg(seg.cell_inst + c);
        act = st.active[inst];
        step = st.step[inst];
    }
    double r[5];
    if constexpr (X) {
        double acc[5] = {0, 0, 0, 0, 0};
        const int cnt = slot_cnt[c];
        int sf[MAX_SLOTS];
#pragma unroll
        for (int j = 0; j < MAX_SLOTS; j++) {
            sf[j] = (j < cnt) ? __ldg(slot_face + j * s.SL + c) : 0;
        }
        if (two) {  // viscous terms: subtracted on the left, added on the right (derivative.c:91-156)
            const GT *Gv = G + flux_rec2_offset(s.F);
#pragma unroll
            for (int j = 0; j < MAX_SLOTS; j++) {
                if (j < cnt) {
                    double gv[5];
                    flux_rec_load(Gv, s.F, sf[j] >= 0 ? sf[j] : ~sf[j], gv);
#pragma unroll
                    for (int v = 0; v < 5; v++) {
                        acc[v] = (sf[j] >= 0) ? (acc[v] - gv[v]) : (acc[v] + gv[v]);
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < MAX_SLOTS; j++) {
            if (j < cnt) {
                double gv[5];
                flux_rec_load(G, s.F, sf[j] >= 0 ? sf[j] : ~sf[j], gv);
#pragma unroll
                for (int v = 0; v < 5; v++) {
                    acc[v] = (sf[j] >= 0) ? (acc[v] + gv[v]) : (acc[v] - gv[v]);
                }
            }
        }
        const double vol = __ldg(cd.volume + c);
#pragma unroll
        for (int v = 0; v < 5; v++) {
            r[v] = -acc[v] / vol;
        }
    }
    else {
        // all slot indices first, then every face record in flight at once; sums in slot order
        double acc[5] = {0, 0, 0, 0, 0};
        const int cnt = slot_cnt[c];
        int sf[MAX_SLOTS];
#pragma unroll
        for (int j = 0; j < MAX_SLOTS; j++) {
            sf[j] = (j < cnt) ? __ldg(slot_face + j * s.SL + c) : 0;
        }
        double gv[MAX_SLOTS][5];
#pragma unroll
        for (int j = 0; j < MAX_SLOTS; j++) {
            flux_rec_load(G, s.F, (j < cnt) ? (sf[j] >= 0 ? sf[j] : ~sf[j]) : 0, gv[j]);
        }
#pragma unroll
        for (int j = 0; j < MAX_SLOTS; j++) {
            if (j < cnt) {
#pragma unroll
                for (int v = 0; v < 5; v++) {
                    acc[v] = (sf[j] >= 0) ? (acc[v] + gv[j][v]) : (acc[v] - gv[j][v]);
                }
            }
        }
        const double ivol = 1.0 / __ldg(cd.volume + c);  // one reciprocal for the five components
#pragma unroll
        for (int v = 0; v < 5; v++) {
            r[v] = -acc[v] * ivol;
        }
    }
    if (SRC == 3) {
        // device source function: its values for this residual, [5][C] (derivative.c:262)
#pragma unroll
        for (int v = 0; v < 5; v++) {
            r[v] += src.avg[(size_t)v * C + c];
        }
    }
    else if (SRC != 0) {
        // the state being differentiated (plain loads: this kernel writes q afterwards)
        Prim<double> qc{q[c], v3(q[N + c], q[2 * N + c], q[3 * N + c]), q[4 * N + c]};
        add_source<SRC>(src, qc, __ldg(seg.cell_inst + c), r);
    }
    if (MODE == 0 || last) {
#pragma unroll
        for (int v = 0; v < 5; v++) {
            Rout[v * C + c] = r[v];
        }
    }
    if (MODE == 0) {
        return;
    }
    if (!act) {
        if (last) {
            dtc[c] = DBL_MAX;
        }
        return;
    }
    Cons<double> u;
    u.rho = __ldg(U0 + c) + ((r[0] * alpha) * step);
    u.m.x = __ldg(U0 + C + c) + ((r[1] * alpha) * step);
    u.m.y = __ldg(U0 + 2 * C + c) + ((r[2] * alpha) * step);
    u.m.z = __ldg(U0 + 3 * C + c) + ((r[3] * alpha) * step);
    u.e = __ldg(U0 + 4 * C + c) + ((r[4] * alpha) * step);
    Prim<double> p = cons_to_prim(u, prop.v[0]);
    store_prim(q, N, c, p);
    if (last) {
        Cons<double> u0 = prim_to_cons(p, prop.v[0]);
        U0[c] = u0.rho;
        U0[C + c] = u0.m.x;
        U0[2 * C + c] = u0.m.y;
        U0[3 * C + c] = u0.m.z;
        U0[4 * C + c] = u0.e;
        dtc[c] = cell_timestep<NS>(p, prop.v, cd, C, c);
    }
}

// U0 = cons(q) and the stable time step of every cell (start of a run / after the host changed
// the state)
template <bool NS, bool X>
__global__ void __launch_bounds__(BLOCK) k_prepare(Sizes s, CellData cd, const double *__restrict__ q,
                                                   double *__restrict__ U0, Props prop, double *__restrict__ dtc)
{
    static_assert(X == kExact, "exact kernels live in the exact translation units only");
    const int C = s.C;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) {
        return;
    }
    Prim<double> p = load_prim<double>(q, s.N, c);
    Cons<double> u0 = prim_to_cons(p, prop.v[0]);
    U0[c] = u0.rho;
    U0[C + c] = u0.m.x;
    U0[2 * C + c] = u0.m.y;
    U0[3 * C + c] = u0.m.z;
    U0[4 * C + c] = u0.e;
    dtc[c] = cell_timestep<NS>(p, prop.v, cd, C, c);
}

// ---- launchers of the exact translation unit (stage_exact.cu) ----------------------------------
//
// FP64 stage kernels with teal's exact arithmetic. The context's own translation unit launches the
// fast instantiations directly; these take the same arguments as plain structs.

struct GradientLaunch {
    Sizes s;
    Geometry<double> g;
    const double *eps2;
    const double *q;
    double *rec;
    int limiter;  // TG_LIMITER_*
    bool fold;    // multiply psi into the record
    bool mixed;   // cells with fewer than MAX_SLOTS faces exist
    int *err;     // device error word (a staging wait that gives up sets ERR_TIMEOUT)
    int polls;    // limit of the staging wait (MBAR_POLLS unless a test lowers it)
};

struct CellLaunch {
    int mode;    // 0: derivative, 1: RK stage
    bool ns;     // Navier-Stokes time step
    int source;  // 0 none, 1 body force, 2 bulk forcing, 3 device function
    int two;     // viscous records before the convective ones
    Sizes s;
    const int *slot_face;
    const uint8_t *slot_cnt;
    CellData cd;
    const double *G;
    double *U0, *q, *Rout;
    Segments seg;
    Steps st;
    double alpha;
    int last;
    Props prop;
    double *dtc;
    Source src;
};

struct BoundaryLaunch {
    Sizes s;
    const int2 *lr;
    const double *basis;
    const int *bface_ent, *bkind;
    const double *bctx;
    double *q;
    double gamma;
    const int *cell_inst, *active;
};

cudaError_t launch_gradient_exact(const GradientLaunch &a, cudaStream_t st);
cudaError_t launch_cell_exact(const CellLaunch &a, cudaStream_t st);
cudaError_t launch_prepare_exact(bool ns, Sizes s, CellData cd, const double *q, double *U0, Props prop, double *dtc,
                                 cudaStream_t st);
cudaError_t launch_boundary_exact(const BoundaryLaunch &a, cudaStream_t st);

}  // namespace tg
