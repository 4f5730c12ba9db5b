// Kernels of the host-driven bookkeeping around the stage kernels: per-piece and per-instance
// reductions (time-step minima, residual norms, volume averages), the step's instance bookkeeping,
// and the device mesh upload / teal-layout transfers. Included only by the context's translation
// unit.
#pragma once

#include "kernels.cuh"

namespace tg {

// per-piece volume-weighted sums of the primitive state (the Prepare of the bulk forcing:
// equations_average over the inner cells, src/equations/average.c:8-40)
__global__ void __launch_bounds__(BLOCK) k_piece_average(Segments seg, int N, const double *__restrict__ q,
                                                         const double *__restrict__ volume,
                                                         double *__restrict__ part)
{
    __shared__ double sh[BLOCK / 32];
    const int beg = seg.piece_beg[blockIdx.x], end = seg.piece_beg[blockIdx.x + 1];
    double t[5] = {0, 0, 0, 0, 0};
    for (int c = beg + threadIdx.x; c < end; c += BLOCK) {
        const double v = volume[c];
#pragma unroll
        for (int k = 0; k < 5; k++) {
            t[k] += v * q[(size_t)k * N + c];
        }
    }
#pragma unroll
    for (int k = 0; k < 5; k++) {
        double sum = block_sum<BLOCK>(t[k], sh);
        if (threadIdx.x == 0) {
            part[5 * blockIdx.x + k] = sum;
        }
    }
}

// avg[i] = sum of instance i's piece sums / its volume
__global__ void k_inst_average(Segments seg, const double *__restrict__ part, double *__restrict__ avg)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= seg.ninst) {
        return;
    }
    for (int k = 0; k < 5; k++) {
        double t = 0;
        for (int p = seg.inst_piece_off[i]; p < seg.inst_piece_off[i + 1]; p++) {
            t += part[5 * p + k];
        }
        avg[5 * i + k] = t / seg.sum_volume[i];
    }
}

// ---- per-instance reductions (deterministic: fixed pieces, fixed order) ---------------------

// per piece: minimum cell time step and (with `res`) the sums of V * R^2 per variable
__global__ void __launch_bounds__(BLOCK) k_piece_reduce(Segments seg, int C, const double *__restrict__ dtc,
                                                        const double *__restrict__ R,
                                                        const double *__restrict__ volume, int res,
                                                        double *__restrict__ part_min,
                                                        double *__restrict__ part_sum)
{
    __shared__ double sh[BLOCK / 32];
    const int beg = seg.piece_beg[blockIdx.x], end = seg.piece_beg[blockIdx.x + 1];
    double m = DBL_MAX;
    double t[5] = {0, 0, 0, 0, 0};
    for (int c = beg + threadIdx.x; c < end; c += BLOCK) {
        m = fmin(m, dtc[c]);
        if (res) {
            double v = volume[c];
#pragma unroll
            for (int k = 0; k < 5; k++) {
                double r = R[k * C + c];
                t[k] += v * (r * r);
            }
        }
    }
    m = block_min<BLOCK>(m, sh);
    if (threadIdx.x == 0) {
        part_min[blockIdx.x] = m;
    }
    if (res) {
#pragma unroll
        for (int k = 0; k < 5; k++) {
            double sum = block_sum<BLOCK>(t[k], sh);
            if (threadIdx.x == 0) {
                part_sum[5 * blockIdx.x + k] = sum;
            }
        }
    }
}

constexpr int INST_BLOCK = 128;

// start of a step, one block per instance: step0 = courant * min, step = min(step0, clip)
__global__ void __launch_bounds__(INST_BLOCK) k_inst_begin(Segments seg, const double *__restrict__ part_min,
                                                           double courant, Steps st)
{
    __shared__ double sh[INST_BLOCK / 32];
    const int i = blockIdx.x;
    double m = DBL_MAX;
    for (int p = seg.inst_piece_off[i] + threadIdx.x; p < seg.inst_piece_off[i + 1]; p += INST_BLOCK) {
        m = fmin(m, part_min[p]);
    }
    m = block_min<INST_BLOCK>(m, sh);
    if (threadIdx.x == 0 && st.active[i]) {
        double step0 = courant * m;
        double clip = st.use_max_time ? (st.max_time[i] - st.time[i]) : st.max_step[i];
        st.step0[i] = step0;
        st.step[i] = fmin(step0, clip);
        if (!isfinite(step0) || !(step0 > 0)) {  // the instance stops; the others go on
            atomicOr(st.error, ERR_NONFINITE);
            st.fail[i] = 1;
            st.active[i] = 0;
        }
    }
}

// is_close of src/core/utils.c:29-34
__device__ __forceinline__ bool is_close(double a, double b)
{
    return fabs(a - b) <= fmax(1e-8, 1e-5 * fmax(fabs(a), fabs(b)));
}

// end of a step (or a bare residual), one block per instance: residual = sqrt(sum / sum_volume);
// with `advance`: time += step, iteration count, and the run loop's stop tests
// (src/simulation/run.c:68-83): iterations, residual threshold, end time
__global__ void __launch_bounds__(INST_BLOCK) k_inst_end(Segments seg, const double *__restrict__ part_sum,
                                                         int advance, Steps st)
{
    __shared__ double sh[INST_BLOCK / 32];
    const int i = blockIdx.x;
    const bool was_active = st.active[i] != 0;
    double res[5];
    for (int k = 0; k < 5; k++) {
        double t = 0;
        for (int p = seg.inst_piece_off[i] + threadIdx.x; p < seg.inst_piece_off[i + 1]; p += INST_BLOCK) {
            t += part_sum[5 * p + k];
        }
        res[k] = block_sum<INST_BLOCK>(t, sh);
    }
    if (threadIdx.x != 0 || (advance && !was_active)) {
        return;
    }
    double mx = 0;
    bool finite = true;
    for (int k = 0; k < 5; k++) {
        res[k] = sqrt(res[k] / seg.sum_volume[i]);
        st.residual[5 * i + k] = res[k];
        mx = (res[k] > mx) ? res[k] : mx;
        finite = finite && isfinite(res[k]);
    }
    if (!finite) {
        atomicOr(st.error, ERR_NONFINITE);
    }
    if (!advance) {
        return;
    }
    if (!finite) {  // the instance stops with its step counted; the others go on
        st.fail[i] = 1;
        st.active[i] = 0;
    }
    double t = st.time[i] + st.step[i];
    st.time[i] = t;
    int it = st.iter[i] + 1;
    st.iter[i] = it;
    bool stop = it >= st.max_iter[i];
    if (st.threshold[i] > 0) {
        int v = st.variable[i];
        stop = stop || (((v >= 0) ? res[v] : mx) < st.threshold[i]);
    }
    if (st.use_max_time) {
        double tm = st.max_time[i];
        stop = stop || !((t < tm) && !is_close(t, tm));
    }
    if (stop) {
        st.active[i] = 0;
    }
}

// number of active instances after a step
__global__ void k_count_active(int ninst, Steps st)
{
    __shared__ int sh;
    if (threadIdx.x == 0) {
        sh = 0;
    }
    __syncthreads();
    int n = 0;
    for (int i = threadIdx.x; i < ninst; i += blockDim.x) {
        n += st.active[i] != 0;
    }
    atomicAdd(&sh, n);
    __syncthreads();
    if (threadIdx.x == 0) {
        *st.num_active = sh;
    }
}

// ---- device mesh upload: per-cell slot lists (integer work, checked against a host recompute) --

// count faces per inner cell; a partition's halo rows (>= C) sit on faces but own no slots
__global__ void k_slot_count(int F, int F_in, int C, const int2 *__restrict__ lr, int *__restrict__ cnt)
{
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) {
        return;
    }
    int2 c = lr[f];
    if (c.x < C) {
        atomicAdd(cnt + c.x, 1);
    }
    if (f < F_in && c.y < C) {
        atomicAdd(cnt + c.y, 1);
    }
}

// scatter face references into the ELL slots (arbitrary order; sorted afterwards)
__global__ void k_slot_fill(int F, int F_in, int C, int SL, const int2 *__restrict__ lr, int *__restrict__ cursor,
                            int *__restrict__ slot_face)
{
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) {
        return;
    }
    int2 c = lr[f];
    if (c.x < C) {
        int j = atomicAdd(cursor + c.x, 1);
        if (j < MAX_SLOTS) {
            slot_face[j * SL + c.x] = f;
        }
    }
    if (f < F_in && c.y < C) {
        int k = atomicAdd(cursor + c.y, 1);
        if (k < MAX_SLOTS) {
            slot_face[k * SL + c.y] = ~f;
        }
    }
}

__device__ __forceinline__ int face_of(int sf)
{
    return sf >= 0 ? sf : ~sf;
}

// sort each cell's slots by face index, then fill neighbour, weight and offset of each slot
template <typename G>
__global__ void k_slot_finish(int C, int SL, const int2 *__restrict__ lr, const int *__restrict__ cnt_in,
                              const double *__restrict__ weight_aos, const double *__restrict__ offset_aos,
                              int *__restrict__ slot_face, int *__restrict__ slot_nbr,
                              uint8_t *__restrict__ slot_cnt, G *__restrict__ slot_w,
                              G *__restrict__ slot_off, int *__restrict__ error)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) {
        return;
    }
    int cnt = cnt_in[c];
    if (cnt > MAX_SLOTS || cnt < 1) {
        atomicExch(error, 1);
        cnt = cnt > MAX_SLOTS ? MAX_SLOTS : cnt;
    }
    int sf[MAX_SLOTS];
    for (int j = 0; j < cnt; j++) {
        sf[j] = slot_face[j * SL + c];
    }
    for (int i = 1; i < cnt; i++) {  // insertion sort by face index
        int key = sf[i];
        int j = i - 1;
        while (j >= 0 && face_of(sf[j]) > face_of(key)) {
            sf[j + 1] = sf[j];
            j -= 1;
        }
        sf[j + 1] = key;
    }
    slot_cnt[c] = (uint8_t)cnt;
    for (int j = 0; j < MAX_SLOTS; j++) {
        if (j < cnt) {
            int f = face_of(sf[j]);
            int side = sf[j] >= 0 ? 0 : 1;
            int2 p = lr[f];
            slot_face[j * SL + c] = sf[j];
            slot_nbr[j * SL + c] = side == 0 ? p.y : p.x;
            for (int d = 0; d < 3; d++) {
                slot_w[(size_t)(d * MAX_SLOTS + j) * SL + c] = G(weight_aos[(size_t)f * 6 + side * 3 + d]);
                slot_off[(size_t)(d * MAX_SLOTS + j) * SL + c] = G(offset_aos[(size_t)f * 6 + side * 3 + d]);
            }
        }
        else {  // padding: a self-reference with zero weight and offset
            slot_face[j * SL + c] = 0;
            slot_nbr[j * SL + c] = c;
            for (int d = 0; d < 3; d++) {
                slot_w[(size_t)(d * MAX_SLOTS + j) * SL + c] = G(0);
                slot_off[(size_t)(d * MAX_SLOTS + j) * SL + c] = G(0);
            }
        }
    }
}

// Gradient tiles (grad_tile_bytes) from the pitched slot arrays: block t fills tile t, lane l the
// column of cell 32 t + l; columns past the last cell hold zeros (their threads never read them)
template <typename G>
__global__ void k_grad_tiles(int C, int SL, const long long *__restrict__ toff, const int *__restrict__ slot_nbr,
                             const double *__restrict__ slot_w, const double *__restrict__ slot_off,
                             unsigned char *__restrict__ tiles)
{
    const int t = blockIdx.x, l = threadIdx.x, c = t * 32 + l;
    const long long o = toff[t];
    const int J = int((toff[t + 1] - o) / grad_tile_bytes<G>(1));
    int *nbr = reinterpret_cast<int *>(tiles + o);
    G *w = reinterpret_cast<G *>(tiles + o + grad_tile_nbr_bytes<G>(J));
    G *off = reinterpret_cast<G *>(tiles + o + grad_tile_nbr_bytes<G>(J) + grad_tile_vec_bytes<G>(J));
    for (int j = 0; j < J; j++) {
        nbr[j * 32 + l] = c < C ? slot_nbr[(size_t)j * SL + c] : 0;
        for (int d = 0; d < 3; d++) {
            const size_t src = (size_t)(d * MAX_SLOTS + j) * SL + c;
            w[(3 * j + d) * 32 + l] = c < C ? G(slot_w[src]) : G(0);
            off[(3 * j + d) * 32 + l] = c < C ? G(slot_off[src]) : G(0);
        }
    }
}

// AoS [n][k] -> SoA [k][n] with an element type change
template <typename T>
__global__ void k_transpose(int n, int k, const double *__restrict__ aos, T *__restrict__ soa)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    for (int j = 0; j < k; j++) {
        soa[(size_t)j * n + i] = T(aos[(size_t)i * k + j]);
    }
}

// periodic faces: redirect the ghost right cell to its owner
__global__ void k_redirect(int F, int F_bd, int off_periodic_ghost, const int *__restrict__ face_cell,
                           const int *__restrict__ owner, int num_owner, int2 *__restrict__ lr,
                           int *__restrict__ error)
{
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) {
        return;
    }
    int l = face_cell[2 * f], r = face_cell[2 * f + 1];
    if (f >= F_bd) {
        int g = r - off_periodic_ghost;
        if (g < 0 || g >= num_owner) {
            atomicExch(error, 2);
            r = l;
        }
        else {
            r = owner[g];
        }
    }
    lr[f] = make_int2(l, r);
}

// teal AoS rows [n][5] -> state rows [row0, row0 + n) of the SoA state
__global__ void k_rows_aos_to_soa(int n, int row0, int N, const double *__restrict__ aos, double *__restrict__ q)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
#pragma unroll
    for (int v = 0; v < 5; v++) {
        q[(size_t)v * N + row0 + i] = aos[(size_t)i * 5 + v];
    }
}

// teal AoS rows [n][5] gathered from the state rows `rowmap` (periodic ghosts map to their owners)
__global__ void k_rows_gather(int n, const int *__restrict__ rowmap, int N, const double *__restrict__ q,
                              double *__restrict__ aos)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    int src = rowmap[i];
#pragma unroll
    for (int v = 0; v < 5; v++) {
        aos[(size_t)i * 5 + v] = q[(size_t)v * N + src];
    }
}

// SoA [5][C] -> AoS [C][5] (derivative) and back
__global__ void k_soa5_to_aos(int C, const double *__restrict__ soa, double *__restrict__ aos)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C) {
        return;
    }
#pragma unroll
    for (int v = 0; v < 5; v++) {
        aos[(size_t)i * 5 + v] = soa[v * C + i];
    }
}

__global__ void k_aos5_to_soa(int C, const double *__restrict__ aos, double *__restrict__ soa)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C) {
        return;
    }
#pragma unroll
    for (int v = 0; v < 5; v++) {
        soa[v * C + i] = aos[(size_t)i * 5 + v];
    }
}

// gradient records -> teal's [C][5][3] (limited when `limit` and the record is not folded)
template <typename R>
__global__ void k_grad_to_aos(int C, const R *__restrict__ rec, int limit, double *__restrict__ aos)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C) {
        return;
    }
    for (int v = 0; v < 5; v++) {
        R gx, gy, gz, psi;
        grad_rec_load(rec, i, v, gx, gy, gz, psi);
        if (limit) {
            gx *= psi, gy *= psi, gz *= psi;
        }
        aos[(size_t)i * 15 + 3 * v] = double(gx);
        aos[(size_t)i * 15 + 3 * v + 1] = double(gy);
        aos[(size_t)i * 15 + 3 * v + 2] = double(gz);
    }
}

// ---- halo of a partition (one rank's share of a mesh) ---------------------------------------------
//
// A partition's state has, after its inner cells and boundary ghosts, one row per halo cell (an
// inner cell of another rank on a face of this rank's cells). Before the gradient the halo rows
// receive their owners' states, before the face fluxes their gradient records: packed by the owner
// from its `send` rows, moved by the caller, unpacked here in halo order.

// buf[i][v] = q[v][rows[i]]
__global__ void k_halo_pack_q(int n, const int *__restrict__ rows, int N, const double *__restrict__ q,
                              double *__restrict__ buf)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const int r = rows[i];
#pragma unroll
    for (int v = 0; v < 5; v++) {
        buf[(size_t)i * 5 + v] = q[(size_t)v * N + r];
    }
}

// q[v][row0 + i] = buf[i][v]
__global__ void k_halo_unpack_q(int n, int row0, int N, const double *__restrict__ buf, double *__restrict__ q)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
#pragma unroll
    for (int v = 0; v < 5; v++) {
        q[(size_t)v * N + row0 + i] = buf[(size_t)i * 5 + v];
    }
}

// gradient records (20 values of type R per row): buf[i] = rec[rows[i]], and back into rows row0 + i
template <typename R>
__global__ void k_halo_pack_rec(int n, const int *__restrict__ rows, const R *__restrict__ rec, R *__restrict__ buf)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const R *src = rec + (size_t)rows[i] * 20;
#pragma unroll
    for (int k = 0; k < 20; k++) {
        buf[(size_t)i * 20 + k] = src[k];
    }
}

template <typename R>
__global__ void k_halo_unpack_rec(int n, int row0, const R *__restrict__ buf, R *__restrict__ rec)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    R *dst = rec + (size_t)(row0 + i) * 20;
#pragma unroll
    for (int k = 0; k < 20; k++) {
        dst[k] = buf[(size_t)i * 20 + k];
    }
}

}  // namespace tg
