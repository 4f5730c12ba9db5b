// Host mesh generation for one process: teal's Cartesian box (src/mesh/create.c:509-544) and its
// connectivity / geometry generation (src/mesh/generate.c:779-815), producing teal's arrays in
// teal's order so a device context built from them matches a context built from teal's own Mesh.
// Floating-point expressions keep teal's evaluation order; this file is compiled without
// floating-point contraction so the geometry is bit-identical to teal's (-std=c99) build.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/teal_b200.h"

namespace {

struct Vec {
    double x, y, z;
};

inline Vec vadd(Vec a, Vec b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec vsub(Vec a, Vec b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec vmul(double s, Vec a) { return {s * a.x, s * a.y, s * a.z}; }
inline Vec vdiv(Vec a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double vdot(Vec a, Vec b) { return ((a.x * b.x) + (a.y * b.y)) + (a.z * b.z); }
inline double vnorm(Vec a) { return std::sqrt(vdot(a, a)); }
inline Vec vabs(Vec a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline Vec vcross(Vec a, Vec b)
{
    return {(a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x)};
}

inline bool is_close(double a, double b)  // src/core/utils.c:29-34
{
    return std::fabs(a - b) <= std::fmax(1e-8, 1e-5 * std::fmax(std::fabs(a), std::fabs(b)));
}

// Host threads for the loops of mesh generation whose iterations are independent: every element
// gets the same arithmetic as in a serial loop, so results do not depend on the split.

// parts for n items: at most 16 and the host's cores, at least 32768 items each
int num_parts(int n)
{
    unsigned hw = std::thread::hardware_concurrency();
    return std::max(1, std::min<int>(hw ? (int)hw : 1, std::min(16, n / 32768)));
}

// body(p) for p in [0, parts), part 0 on the calling thread
template <class Body>
void run_parts(int parts, const Body &body)
{
    std::vector<std::thread> pool;
    for (int p = 1; p < parts; p++) {
        try {
            pool.emplace_back([&body, p] { body(p); });
        }
        catch (...) {
            body(p);  // no thread to be had: this part runs here
        }
    }
    body(0);
    for (auto &th : pool) th.join();
}

// body(beg, end) over [0, n) in contiguous chunks
template <class Body>
void parallel_for(int n, const Body &body)
{
    int parts = num_parts(n), chunk = (n + parts - 1) / parts;
    run_parts(parts, [&](int p) { body(std::min(n, p * chunk), std::min(n, (p + 1) * chunk)); });
}

struct Entity {
    std::string name;
    double rotation[9];
    Vec translation;
};

}  // namespace

struct tg_host_mesh {
    // nodes
    std::vector<Vec> coord;
    // cells: node CSR, neighbour CSR
    int num_cells = 0, num_inner = 0, off_boundary = 0, off_periodic = 0;
    std::vector<int> node_off, node_idx;
    std::vector<int> cell_off, cell_idx;
    std::vector<double> volume;
    double sum_volume = 0;
    std::vector<Vec> center, projection, offset;
    // faces
    int num_faces = 0, num_inner_faces = 0, off_boundary_faces = 0;
    std::vector<int> fnode_off, fnode_idx;
    std::vector<int> face_cell;  // [F][2]
    std::vector<double> area;
    std::vector<Vec> fcenter;
    std::vector<double> basis;       // [F][9]
    std::vector<double> weight;      // [F][6]
    std::vector<double> foffset;     // [F][6]
    std::vector<double> correction;  // [F][4]
    // entities
    int num_inner_entities = 0, off_boundary_entities = 0;
    std::vector<Entity> entities;
    std::vector<int> ent_cell_off, ent_face_off;
    // periodic self-exchange
    std::vector<int> tag, recv_off, send_off, send_idx;
};

namespace {

// ---- Cartesian box (create.c) ------------------------------------------------------------------

int side_count(const int n[3], int side)
{
    switch (side / 2) {
        case 0: return n[1] * n[2];
        case 1: return n[2] * n[0];
        default: return n[0] * n[1];
    }
}

void append_side_cells(std::vector<int> &out, const int n[3], int side)
{
    if (side / 2 == 0) {
        int i = (side % 2 == 0) ? 0 : (n[0] - 1);
        for (int j = 0; j < n[1]; j++)
            for (int k = 0; k < n[2]; k++) out.push_back(i + (n[0] * (j + (n[1] * k))));
    }
    else if (side / 2 == 1) {
        int j = (side % 2 == 0) ? 0 : (n[1] - 1);
        for (int k = 0; k < n[2]; k++)
            for (int i = 0; i < n[0]; i++) out.push_back(i + (n[0] * (j + (n[1] * k))));
    }
    else {
        int k = (side % 2 == 0) ? 0 : (n[2] - 1);
        for (int i = 0; i < n[0]; i++)
            for (int j = 0; j < n[1]; j++) out.push_back(i + (n[0] * (j + (n[1] * k))));
    }
}

int cartesian(tg_host_mesh &m, const double *lo_in, const double *hi_in, const int *num, const int *periodic,
              const double *displacement)
{
    int n[3] = {num[0], num[1], num[2]};
    for (int d = 0; d < 3; d++) {
        if (n[d] < 1) return TG_ERR_INVALID;
    }
    int ndims = (n[0] > 1) + (n[1] > 1) + (n[2] > 1);
    // the axes with more than one cell must come first (the Cartesian communicator has ndims axes)
    for (int d = 0; d < 3; d++) {
        if ((d < ndims) != (n[d] > 1)) return TG_ERR_INVALID;
    }
    double lo[3] = {lo_in[0], lo_in[1], lo_in[2]}, hi[3] = {hi_in[0], hi_in[1], hi_in[2]};
    Vec extent = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    for (int d = 0; d < 3; d++) {  // split_bounds on one process (create.c:75-94)
        if (d < ndims) {
            double width = (hi[d] - lo[d]) / n[d];
            hi[d] = lo[d] + (n[d] * width);
        }
        else {
            n[d] = 1;
            if (is_close(lo[d], hi[d])) hi[d] = lo[d] + 1;
        }
    }
    int per[3] = {periodic[0] != 0, periodic[1] != 0, periodic[2] != 0};

    // nodes (create.c:130-160)
    int nnx = n[0] + 1, nny = n[1] + 1, nnz = n[2] + 1;
    Vec del = {(hi[0] - lo[0]) / n[0], (hi[1] - lo[1]) / n[1], (hi[2] - lo[2]) / n[2]};
    m.coord.resize((size_t)nnx * nny * nnz);
    size_t id = 0;
    for (int k = 0; k < nnz; k++)
        for (int j = 0; j < nny; j++)
            for (int i = 0; i < nnx; i++) {
                m.coord[id] = {lo[0] + (i * del.x), lo[1] + (j * del.y), lo[2] + (k * del.z)};
                if (displacement) {  // mesh_modify (src/mesh/modify.c:5-11)
                    m.coord[id].x += displacement[3 * id + 0];
                    m.coord[id].y += displacement[3 * id + 1];
                    m.coord[id].z += displacement[3 * id + 2];
                }
                id++;
            }

    // cells (create.c:180-277): inner hexes, then face cells per side
    int num_inner = n[0] * n[1] * n[2];
    int num_boundary = 0, num_periodic = 0;
    for (int s = 0; s < 2 * ndims; s++) {
        if (per[s / 2])
            num_periodic += side_count(n, s);
        else
            num_boundary += side_count(n, s);
    }
    int num_cells = num_inner + num_boundary + num_periodic;
    std::vector<int> off(num_cells + 1, 0), idx;
    idx.reserve((size_t)num_inner * 8 + (size_t)(num_boundary + num_periodic) * 4);
    auto node = [&](int i, int j, int k) { return i + (nnx * (j + (nny * k))); };
    int c = 0;
    for (int k = 0; k < n[2]; k++)
        for (int j = 0; j < n[1]; j++)
            for (int i = 0; i < n[0]; i++) {
                int v[8] = {node(i, j, k),         node(i + 1, j, k),     node(i + 1, j + 1, k),
                            node(i, j + 1, k),     node(i, j, k + 1),     node(i + 1, j, k + 1),
                            node(i + 1, j + 1, k + 1), node(i, j + 1, k + 1)};
                idx.insert(idx.end(), v, v + 8);
                off[++c] = (int)idx.size();
            }
    std::vector<int> side_of_cell;  // side index of each face cell, in creation order
    if (ndims >= 1)
        for (int i = 0; i <= n[0]; i += n[0])
            for (int j = 0; j < n[1]; j++)
                for (int k = 0; k < n[2]; k++) {
                    int v[4] = {node(i, j, k), node(i, j + 1, k), node(i, j + 1, k + 1), node(i, j, k + 1)};
                    idx.insert(idx.end(), v, v + 4);
                    off[++c] = (int)idx.size();
                    side_of_cell.push_back(i == 0 ? 0 : 1);
                }
    if (ndims >= 2)
        for (int j = 0; j <= n[1]; j += n[1])
            for (int k = 0; k < n[2]; k++)
                for (int i = 0; i < n[0]; i++) {
                    int v[4] = {node(i, j, k), node(i + 1, j, k), node(i + 1, j, k + 1), node(i, j, k + 1)};
                    idx.insert(idx.end(), v, v + 4);
                    off[++c] = (int)idx.size();
                    side_of_cell.push_back(j == 0 ? 2 : 3);
                }
    if (ndims >= 3)
        for (int k = 0; k <= n[2]; k += n[2])
            for (int i = 0; i < n[0]; i++)
                for (int j = 0; j < n[1]; j++) {
                    int v[4] = {node(i, j, k), node(i + 1, j, k), node(i + 1, j + 1, k), node(i, j + 1, k)};
                    idx.insert(idx.end(), v, v + 4);
                    off[++c] = (int)idx.size();
                    side_of_cell.push_back(k == 0 ? 4 : 5);
                }

    // entities (create.c:289-338): domain, boundary sides, periodic sides
    const char *names[] = {"domain", "left", "right", "bottom", "top", "back", "front"};
    m.entities.clear();
    m.ent_cell_off.assign(1, 0);
    Entity dom{};
    dom.name = names[0];
    m.entities.push_back(dom);
    m.ent_cell_off.push_back(num_inner);
    for (int s = 0; s < 2 * ndims; s++) {
        if (!per[s / 2]) {
            Entity e{};
            e.name = names[s + 1];
            m.entities.push_back(e);
            m.ent_cell_off.push_back(m.ent_cell_off.back() + side_count(n, s));
        }
    }
    int off_boundary_entities = (int)m.entities.size();
    for (int s = 0; s < 2 * ndims; s++) {
        if (per[s / 2]) {
            Entity e{};
            e.name = names[s + 1];
            e.rotation[0] = e.rotation[4] = e.rotation[8] = 1;
            double sign = (s % 2 == 0) ? -1 : +1;
            e.translation = {0, 0, 0};
            if (s / 2 == 0) e.translation.x = sign * extent.x;
            if (s / 2 == 1) e.translation.y = sign * extent.y;
            if (s / 2 == 2) e.translation.z = sign * extent.z;
            m.entities.push_back(e);
            m.ent_cell_off.push_back(m.ent_cell_off.back() + side_count(n, s));
        }
    }
    m.num_inner_entities = 1;
    m.off_boundary_entities = off_boundary_entities;

    // periodic self-exchange tables (create.c:388-440)
    m.tag.clear();
    m.recv_off.assign(1, num_inner + num_boundary);
    m.send_off.assign(1, 0);
    m.send_idx.clear();
    for (int s = 0; s < 2 * ndims; s++) {
        if (per[s / 2]) {
            m.tag.push_back(s);
            m.tag.push_back((s % 2 == 0) ? (s + 1) : (s - 1));
            m.recv_off.push_back(m.recv_off.back() + side_count(n, s));
            append_side_cells(m.send_idx, n, s);
            m.send_off.push_back((int)m.send_idx.size());
        }
    }

    // order the face cells: boundary sides first, periodic sides after (create.c:470-507)
    std::vector<int> map(num_cells);
    for (int i = 0; i < num_inner; i++) map[i] = i;
    int nb = 0, np = 0;
    for (int i = num_inner; i < num_cells; i++) {
        int s = side_of_cell[i - num_inner];
        map[i] = per[s / 2] ? (num_inner + num_boundary + np++) : (num_inner + nb++);
    }
    std::vector<int> off2(num_cells + 1, 0), idx2(idx.size());
    std::vector<int> inv(num_cells);
    for (int i = 0; i < num_cells; i++) inv[map[i]] = i;
    for (int i = 0; i < num_cells; i++) {
        int src = inv[i];
        int len = off[src + 1] - off[src];
        std::copy(idx.begin() + off[src], idx.begin() + off[src + 1], idx2.begin() + off2[i]);
        off2[i + 1] = off2[i] + len;
    }
    m.node_off.swap(off2);
    m.node_idx.swap(idx2);
    m.num_cells = num_cells;
    m.num_inner = num_inner;
    m.off_boundary = num_inner + num_boundary;
    m.off_periodic = num_cells;
    return TG_OK;
}

// ---- generation (generate.c) --------------------------------------------------------------------

// dual graph: cells sharing >= 3 nodes, or all but one node of either cell; face cells carry one
// extra private node so two face cells never pair up through a shared edge (generate.c:15-66 with
// METIS 5's MeshToDual rule). Neighbours are listed in order of first encounter.
void connect_cells(tg_host_mesh &m)
{
    int nn = (int)m.coord.size();
    int ne = m.num_cells;
    std::vector<int> eoff(ne + 1, 0), eind;
    eind.reserve(m.node_idx.size() + (size_t)(ne - m.num_inner));
    int extra = nn;
    for (int i = 0; i < ne; i++) {
        for (int j = m.node_off[i]; j < m.node_off[i + 1]; j++) eind.push_back(m.node_idx[j]);
        if (i >= m.num_inner) eind.push_back(extra++);
        eoff[i + 1] = (int)eind.size();
    }
    int total_nodes = extra;
    std::vector<int> noff(total_nodes + 1, 0), nind(eind.size());
    for (int v : eind) noff[v + 1]++;
    for (int v = 0; v < total_nodes; v++) noff[v + 1] += noff[v];
    std::vector<int> cur(noff.begin(), noff.end() - 1);
    for (int e = 0; e < ne; e++)
        for (int k = eoff[e]; k < eoff[e + 1]; k++) nind[cur[eind[k]]++] = e;

    // each cell's neighbour list depends only on the node lists: chunks of cells are listed
    // independently and concatenated in cell order
    m.cell_off.assign(ne + 1, 0);
    int parts = num_parts(ne), chunk = (ne + parts - 1) / parts;
    std::vector<std::vector<int>> part(parts);
    run_parts(parts, [&](int p) {
        std::vector<int> mark(ne, 0), nbrs;
        std::vector<int> &out = part[p];
        for (int e = p * chunk; e < std::min(ne, (p + 1) * chunk); e++) {
            nbrs.clear();
            int len_e = eoff[e + 1] - eoff[e];
            for (int k = eoff[e]; k < eoff[e + 1]; k++) {
                int v = eind[k];
                for (int t = noff[v]; t < noff[v + 1]; t++) {
                    int o = nind[t];
                    if (o == e) continue;
                    if (mark[o] == 0) nbrs.push_back(o);
                    mark[o]++;
                }
            }
            for (int o : nbrs) {
                int overlap = mark[o];
                int len_o = eoff[o + 1] - eoff[o];
                bool adj = overlap >= 3 || overlap >= len_e - 1 || overlap >= len_o - 1;
                // inner cells keep every neighbour, face cells only their inner neighbour
                if (adj && (e < m.num_inner || o < m.num_inner)) out.push_back(o);
                mark[o] = 0;
            }
            m.cell_off[e + 1] = (int)out.size();  // within the part; offset below
        }
    });
    m.cell_idx.clear();
    for (int p = 0; p < parts; p++) {
        int base = (int)m.cell_idx.size();
        for (int e = p * chunk; e < std::min(ne, (p + 1) * chunk); e++) m.cell_off[e + 1] += base;
        m.cell_idx.insert(m.cell_idx.end(), part[p].begin(), part[p].end());
    }
}

// renumber cells (or nodes) by `map` (old -> new) within [beg, end) (src/mesh/reorder.c:65-135)
void reorder_cells_by(tg_host_mesh &m, const std::vector<int> &map, int beg, int end)
{
    int num = end - beg;
    std::vector<int> inv(num);
    for (int i = 0; i < num; i++) inv[map[i]] = i;
    std::vector<int> noff(m.node_off), nidx(m.node_idx), coff(m.cell_off), cidx(m.cell_idx);
    for (int i = beg; i < end; i++) {
        int src = beg + inv[i - beg];
        int ln = noff[src + 1] - noff[src];
        m.node_off[i + 1] = m.node_off[i] + ln;
        std::copy(nidx.begin() + noff[src], nidx.begin() + noff[src + 1], m.node_idx.begin() + m.node_off[i]);
        int lc = coff[src + 1] - coff[src];
        m.cell_off[i + 1] = m.cell_off[i] + lc;
        std::copy(cidx.begin() + coff[src], cidx.begin() + coff[src + 1], m.cell_idx.begin() + m.cell_off[i]);
    }
    for (auto &v : m.cell_idx)
        if (beg <= v && v < end) v = beg + map[v - beg];
    for (auto &v : m.send_idx)
        if (beg <= v && v < end) v = beg + map[v - beg];
}

// breadth-first renumbering of the inner cells, neighbours queued by decreasing degree
// (generate.c:68-133)
void reorder_cells(tg_host_mesh &m)
{
    int n = m.num_inner;
    std::vector<int> map(n, -1), degree(n), queue(n);
    for (int i = 0; i < n; i++) degree[i] = m.cell_off[i + 1] - m.cell_off[i];
    int seed = 0, num = 0;
    while (num < n) {
        while (map[seed] != -1) seed = (seed + 1) % n;
        int beg = 0, end = 0;
        map[seed] = num++;
        queue[end++] = seed;
        while (beg < end) {
            int cur = queue[beg++];
            int cell[8];
            int cnt = 0;
            for (int i = m.cell_off[cur]; i < m.cell_off[cur + 1]; i++) {
                int idx = m.cell_idx[i];
                if (idx < n && map[idx] == -1) {
                    cell[cnt++] = idx;
                    map[idx] = -2;
                }
            }
            for (int i = 1; i < cnt; i++) {
                int idx = cell[i], deg = degree[idx], j = i - 1;
                while (j >= 0 && degree[cell[j]] < deg) {
                    cell[j + 1] = cell[j];
                    j -= 1;
                }
                cell[j + 1] = idx;
            }
            for (int i = 0; i < cnt; i++) {
                map[cell[i]] = num++;
                queue[end++] = cell[i];
            }
        }
    }
    reorder_cells_by(m, map, 0, n);
}

// nodes numbered by first use in cell order (generate.c:159-195, one process: all nodes inner)
void reorder_nodes(tg_host_mesh &m)
{
    int nn = (int)m.coord.size();
    std::vector<int> map(nn, -1);
    int num = 0;
    for (int v : m.node_idx)
        if (map[v] == -1) map[v] = num++;
    for (int v = 0; v < nn; v++)
        if (map[v] == -1) map[v] = num++;  // unused nodes keep their relative order at the end
    std::vector<Vec> coord(nn);
    for (int v = 0; v < nn; v++) coord[map[v]] = m.coord[v];
    m.coord.swap(coord);
    for (auto &v : m.node_idx) v = map[v];
}

struct Face {
    int inner, left, right, num_nodes;
    int node[4];
};

// a quad's nodes put in cyclic order (generate.c:227-264); false when no order is valid
bool correct_face_node_order(Face &f, const tg_host_mesh &m)
{
    if (f.num_nodes != 4) return true;
    for (int i = 0; i < 3; i++) {
        Vec c[4];
        for (int j = 0; j < 4; j++) c[j] = m.coord[f.node[j]];
        Vec a2b = vsub(c[1], c[0]), a2c = vsub(c[2], c[0]), a2d = vsub(c[3], c[0]);
        if (vdot(vcross(a2b, a2c), vcross(a2c, a2d)) > 0) return true;
        if (i + 2 < f.num_nodes) std::swap(f.node[i + 1], f.node[i + 2]);
    }
    return false;
}

int create_faces(tg_host_mesh &m)  // generate.c:267-321
{
    // the faces of chunks of inner cells, built independently and concatenated in cell order
    int parts = num_parts(m.num_inner), chunk = (m.num_inner + parts - 1) / parts;
    std::vector<std::vector<Face>> part(parts);
    std::vector<char> bad(parts, 0);
    run_parts(parts, [&](int p) {
        int beg = std::min(m.num_inner, p * chunk), end = std::min(m.num_inner, (p + 1) * chunk);
        part[p].reserve((size_t)(end - beg) * 3);
        for (int i = beg; i < end && !bad[p]; i++) {
            for (int j = m.cell_off[i]; j < m.cell_off[i + 1]; j++) {
                int l = i, r = m.cell_idx[j];
                if (l < r) {
                    Face f{};
                    f.inner = r < m.num_inner;
                    f.left = l;
                    f.right = r;
                    for (int a = m.node_off[l]; a < m.node_off[l + 1]; a++)
                        for (int b = m.node_off[r]; b < m.node_off[r + 1]; b++)
                            if (m.node_idx[a] == m.node_idx[b]) {
                                if (f.num_nodes >= 4) bad[p] = 1;
                                else f.node[f.num_nodes++] = m.node_idx[a];
                            }
                    if (bad[p] || f.num_nodes < 3 || !correct_face_node_order(f, m)) {
                        bad[p] = 1;
                        break;
                    }
                    part[p].push_back(f);
                }
            }
        }
    });
    std::vector<Face> faces;
    size_t total = 0;
    for (int p = 0; p < parts; p++) {
        if (bad[p]) return TG_ERR_INVALID;
        total += part[p].size();
    }
    faces.reserve(total);
    for (int p = 0; p < parts; p++) {
        faces.insert(faces.end(), part[p].begin(), part[p].end());
        std::vector<Face>().swap(part[p]);
    }
    // teal's order: inner faces by left cell, then the others by right cell, ties in creation order
    // (a stable sort). Faces are created by ascending left cell, so the inner ones already stand in
    // that order and only the (few) others need sorting.
    auto outer = std::stable_partition(faces.begin(), faces.end(), [](const Face &f) { return f.inner != 0; });
    std::stable_sort(outer, faces.end(), [](const Face &a, const Face &b) { return a.right < b.right; });
    int F = (int)faces.size();
    m.num_faces = F;
    m.fnode_off.assign(F + 1, 0);
    m.fnode_idx.clear();
    m.fnode_idx.reserve(4 * (size_t)F);
    m.face_cell.resize(2 * (size_t)F);
    int ni = 0, nb = 0;
    for (int i = 0; i < F; i++) {
        if (faces[i].right < m.num_inner)
            ni++;
        else if (faces[i].right < m.off_boundary)
            nb++;
        for (int j = 0; j < faces[i].num_nodes; j++) m.fnode_idx.push_back(faces[i].node[j]);
        m.fnode_off[i + 1] = (int)m.fnode_idx.size();
        m.face_cell[2 * i] = faces[i].left;
        m.face_cell[2 * i + 1] = faces[i].right;
    }
    m.num_inner_faces = ni;
    m.off_boundary_faces = ni + nb;
    // face ranges of the entities (generate.c:323-334)
    int ne = (int)m.entities.size();
    m.ent_face_off.assign(ne + 1, 0);
    m.ent_face_off[0] = ni;
    for (int e = 0; e < ne; e++) {
        m.ent_face_off[e + 1] = m.ent_face_off[e];
        if (e >= m.num_inner_entities) m.ent_face_off[e + 1] += m.ent_cell_off[e + 1] - m.ent_cell_off[e];
    }
    return TG_OK;
}

double tri_area(const Vec *c)
{
    return vnorm(vcross(vsub(c[1], c[0]), vsub(c[2], c[0]))) / 2;
}

double face_area(const Vec *c, int n)  // generate.c:336-351
{
    if (n == 3) return tri_area(c);
    Vec l[3] = {c[0], c[1], c[2]}, r[3] = {c[0], c[2], c[3]};
    return tri_area(l) + tri_area(r);
}

Vec face_center(const Vec *c, int n)  // generate.c:366-382
{
    if (n == 3) return vdiv(vadd(c[0], vadd(c[1], c[2])), 3);
    Vec l[3] = {c[0], c[1], c[2]}, r[3] = {c[0], c[2], c[3]};
    double a[2] = {tri_area(l), tri_area(r)};
    Vec ce[2] = {face_center(l, 3), face_center(r, 3)};
    Vec mm[2] = {vmul(a[0], ce[0]), vmul(a[1], ce[1])};
    return vdiv(vadd(mm[0], mm[1]), a[0] + a[1]);
}

Vec face_normal(const Vec *c, int n)  // generate.c:398-418
{
    if (n == 3) {
        Vec nrm = vcross(vsub(c[1], c[0]), vsub(c[2], c[0]));
        return vdiv(nrm, vnorm(nrm));
    }
    Vec nrm = {0, 0, 0};
    for (int i = 0; i < 4; i++) nrm = vadd(nrm, vcross(c[i], c[(i + 1) % 4]));
    return vdiv(nrm, vnorm(nrm));
}

double tet_volume(const Vec *c)
{
    Vec a2b = vsub(c[1], c[0]), a2c = vsub(c[2], c[0]), a2d = vsub(c[3], c[0]);
    return std::fabs(vdot(a2b, vcross(a2c, a2d))) / 6;
}

double cell_volume(const Vec *c, int n)  // generate.c:468-494
{
    switch (n) {
        case 4: return tet_volume(c);
        case 5: {
            Vec l[4] = {c[0], c[1], c[2], c[4]}, r[4] = {c[0], c[2], c[3], c[4]};
            return cell_volume(l, 4) + cell_volume(r, 4);
        }
        case 6: {
            Vec l[5] = {c[0], c[1], c[4], c[3], c[5]};
            Vec r[4] = {c[0], c[1], c[2], c[5]};
            return cell_volume(l, 5) + cell_volume(r, 4);
        }
        default: {
            Vec l[6] = {c[0], c[1], c[2], c[4], c[5], c[6]};
            Vec r[6] = {c[0], c[2], c[3], c[4], c[6], c[7]};
            return cell_volume(l, 6) + cell_volume(r, 6);
        }
    }
}

Vec cell_center(const Vec *c, int n)  // generate.c:517-557
{
    if (n == 4) {
        Vec s0 = vadd(c[0], c[1]), s1 = vadd(c[2], c[3]);
        return vdiv(vadd(s0, s1), 4);
    }
    Vec l[6], r[6];
    int nl, nr;
    if (n == 5) {
        Vec a[4] = {c[0], c[1], c[2], c[4]}, b[4] = {c[0], c[2], c[3], c[4]};
        std::copy(a, a + 4, l);
        std::copy(b, b + 4, r);
        nl = nr = 4;
    }
    else if (n == 6) {
        Vec a[5] = {c[0], c[1], c[4], c[3], c[5]}, b[4] = {c[0], c[1], c[2], c[5]};
        std::copy(a, a + 5, l);
        std::copy(b, b + 4, r);
        nl = 5;
        nr = 4;
    }
    else {
        Vec a[6] = {c[0], c[1], c[2], c[4], c[5], c[6]}, b[6] = {c[0], c[2], c[3], c[4], c[6], c[7]};
        std::copy(a, a + 6, l);
        std::copy(b, b + 6, r);
        nl = nr = 6;
    }
    double v[2] = {cell_volume(l, nl), cell_volume(r, nr)};
    Vec ce[2] = {cell_center(l, nl), cell_center(r, nr)};
    Vec mm[2] = {vmul(v[0], ce[0]), vmul(v[1], ce[1])};
    return vdiv(vadd(mm[0], mm[1]), v[0] + v[1]);
}

int geometry(tg_host_mesh &m)
{
    int F = m.num_faces;
    auto fcoords = [&](int f, Vec *c) {
        int n = 0;
        for (int j = m.fnode_off[f]; j < m.fnode_off[f + 1]; j++) c[n++] = m.coord[m.fnode_idx[j]];
        return n;
    };
    // face areas, centres, bases (generate.c:353-466)
    m.area.resize(F);
    m.fcenter.resize(F);
    m.basis.resize(9 * (size_t)F);
    parallel_for(F, [&](int beg, int end) {
        for (int f = beg; f < end; f++) {
            Vec c[4];
            int n = fcoords(f, c);
            m.area[f] = face_area(c, n);
            m.fcenter[f] = face_center(c, n);
        }
    });
    parallel_for(F, [&](int beg, int end) {
        for (int f = beg; f < end; f++) {
            Vec c[4];
            int n = fcoords(f, c);
            Vec nx = face_normal(c, n), ny, nz;
            double nqz = std::hypot(nx.x, nx.y);
            double nqy = std::hypot(nx.x, nx.z);
            if (nqz > nqy) {
                ny = {-nx.y / nqz, nx.x / nqz, 0};
                nz = {(-nx.x * nx.z) / nqz, (-nx.y * nx.z) / nqz, nqz};
            }
            else {
                ny = {(-nx.x * nx.y) / nqy, nqy, (-nx.y * nx.z) / nqy};
                nz = {-nx.z / nqy, 0, nx.x / nqy};
            }
            int left = m.face_cell[2 * f];
            Vec mean = {0, 0, 0};
            for (int j = m.node_off[left]; j < m.node_off[left + 1]; j++) mean = vadd(mean, m.coord[m.node_idx[j]]);
            mean = vdiv(mean, (double)(m.node_off[left + 1] - m.node_off[left]));
            if (vdot(vsub(mean, m.fcenter[f]), nx) > 0) {
                nx = vmul(-1, nx);
                ny = vmul(-1, ny);
            }
            double *b = &m.basis[9 * (size_t)f];
            b[0] = nx.x, b[1] = nx.y, b[2] = nx.z;
            b[3] = ny.x, b[4] = ny.y, b[5] = ny.z;
            b[6] = nz.x, b[7] = nz.y, b[8] = nz.z;
        }
    });
    auto normal = [&](int f) { return Vec{m.basis[9 * (size_t)f], m.basis[9 * (size_t)f + 1], m.basis[9 * (size_t)f + 2]}; };

    // cell volumes and centres (generate.c:496-630)
    m.volume.assign(m.num_cells, 0.0);
    m.sum_volume = 0;
    m.center.assign(m.num_cells, Vec{0, 0, 0});
    parallel_for(m.num_inner, [&](int beg, int end) {
        for (int i = beg; i < end; i++) {
            Vec c[8];
            int n = 0;
            for (int j = m.node_off[i]; j < m.node_off[i + 1]; j++) c[n++] = m.coord[m.node_idx[j]];
            m.volume[i] = cell_volume(c, n);
            m.center[i] = cell_center(c, n);
        }
    });
    for (int i = 0; i < m.num_inner; i++) m.sum_volume += m.volume[i];  // in cell order
    for (int f = m.num_inner_faces; f < m.off_boundary_faces; f++) {  // mirrored boundary ghosts
        int l = m.face_cell[2 * f], r = m.face_cell[2 * f + 1];
        Vec nrm = normal(f);
        Vec off = vsub(m.fcenter[f], m.center[l]);
        double factor = 2 * vdot(nrm, off);
        m.center[r] = vadd(m.center[l], vmul(factor, nrm));
    }
    // periodic ghosts: owner centre (exchange) moved by the entity's rotation and translation
    int nnb = (int)m.recv_off.size() - 1;
    std::vector<char> used(nnb, 0);
    for (int k = 0; k < nnb; k++) {
        int tag = m.tag[2 * k];
        for (int j = 0; j < nnb; j++) {
            if (!used[j] && m.tag[2 * j + 1] == tag) {
                used[j] = 1;
                for (int i = 0; i < m.recv_off[k + 1] - m.recv_off[k]; i++)
                    m.center[m.recv_off[k] + i] = m.center[m.send_idx[m.send_off[j] + i]];
                break;
            }
        }
    }
    for (int e = m.off_boundary_entities; e < (int)m.entities.size(); e++) {
        const Entity &en = m.entities[e];
        for (int j = m.ent_cell_off[e]; j < m.ent_cell_off[e + 1]; j++) {
            Vec c = m.center[j];
            Vec r0 = {en.rotation[0], en.rotation[1], en.rotation[2]};
            Vec r1 = {en.rotation[3], en.rotation[4], en.rotation[5]};
            Vec r2 = {en.rotation[6], en.rotation[7], en.rotation[8]};
            Vec rc = {vdot(r0, c), vdot(r1, c), vdot(r2, c)};
            m.center[j] = vadd(rc, en.translation);
        }
    }

    // projections (generate.c:632-646)
    m.projection.assign(m.num_cells, Vec{0, 0, 0});
    for (int f = 0; f < F; f++) {
        int l = m.face_cell[2 * f], r = m.face_cell[2 * f + 1];
        Vec inc = vmul(m.area[f] / 2, vabs(normal(f)));
        m.projection[l] = vadd(m.projection[l], inc);
        if (r < m.num_inner) m.projection[r] = vadd(m.projection[r], inc);
    }

    // cell offsets to the faces of each neighbour (generate.c:648-667). teal finds the face of the
    // pair (min, max) by binary search over the faces sorted by cell pair; a pair has exactly one
    // face (one per neighbour-list entry with left < right), so the face lists of each inner cell
    // find the same face.
    int nnz = m.cell_off[m.num_inner];
    m.offset.assign(nnz, Vec{0, 0, 0});
    int C = m.num_inner;
    std::vector<int> cf_off(C + 1, 0), cf_idx;
    for (int f = 0; f < F; f++) {
        cf_off[m.face_cell[2 * f] + 1]++;
        if (m.face_cell[2 * f + 1] < C) cf_off[m.face_cell[2 * f + 1] + 1]++;
    }
    for (int i = 0; i < C; i++) cf_off[i + 1] += cf_off[i];
    cf_idx.resize(cf_off[C]);
    {
        std::vector<int> cur(cf_off.begin(), cf_off.end() - 1);
        for (int f = 0; f < F; f++) {
            cf_idx[cur[m.face_cell[2 * f]]++] = f;
            if (m.face_cell[2 * f + 1] < C) cf_idx[cur[m.face_cell[2 * f + 1]]++] = f;
        }
    }
    std::atomic<bool> missing{false};
    parallel_for(C, [&](int beg, int end) {
        for (int i = beg; i < end; i++) {
            for (int j = m.cell_off[i]; j < m.cell_off[i + 1]; j++) {
                int o = m.cell_idx[j], l = std::min(i, o), r = std::max(i, o), face = -1;
                for (int k = cf_off[i]; k < cf_off[i + 1]; k++) {
                    int f = cf_idx[k];
                    if (m.face_cell[2 * f] == l && m.face_cell[2 * f + 1] == r) {
                        face = f;
                        break;
                    }
                }
                if (face < 0) {
                    missing.store(true, std::memory_order_relaxed);
                    continue;
                }
                m.offset[j] = vsub(m.fcenter[face], m.center[i]);
            }
        }
    });
    if (missing.load()) return TG_ERR_INVALID;

    // least-squares weights (generate.c:669-752)
    std::vector<double> r11(C, 0), r12(C, 0), r22(C, 0), r13(C, 0), r23(C, 0), r33(C, 0);
    for (int f = 0; f < F; f++) {
        int l = m.face_cell[2 * f], r = m.face_cell[2 * f + 1];
        Vec d = vsub(m.center[r], m.center[l]);
        double t2 = 1 / vdot(d, d);
        r11[l] += (t2 * d.x) * d.x;
        r12[l] += (t2 * d.x) * d.y;
        r22[l] += (t2 * d.y) * d.y;
        r13[l] += (t2 * d.x) * d.z;
        r23[l] += (t2 * d.y) * d.z;
        r33[l] += (t2 * d.z) * d.z;
        if (r < C) {
            r11[r] += (t2 * d.x) * d.x;
            r12[r] += (t2 * d.x) * d.y;
            r22[r] += (t2 * d.y) * d.y;
            r13[r] += (t2 * d.x) * d.z;
            r23[r] += (t2 * d.y) * d.z;
            r33[r] += (t2 * d.z) * d.z;
        }
    }
    for (int i = 0; i < C; i++) {
        r11[i] = std::sqrt(r11[i]);
        r12[i] = r12[i] / r11[i];
        r22[i] = std::sqrt(r22[i] - (r12[i] * r12[i]));
        r13[i] = r13[i] / r11[i];
        r23[i] = (r23[i] - (r12[i] * r13[i])) / r22[i];
        r33[i] = std::sqrt(r33[i] - ((r13[i] * r13[i]) + (r23[i] * r23[i])));
    }
    auto face_weight = [&](Vec d, int i) {
        Vec w = {0, 0, 0};
        double beta = ((r12[i] * r23[i]) - (r13[i] * r22[i])) / (r11[i] * r22[i]);
        Vec a;
        a.x = d.x / (r11[i] * r11[i]);
        a.y = (d.y - ((r12[i] / r11[i]) * d.x)) / (r22[i] * r22[i]);
        a.z = ((d.z - ((r23[i] / r22[i]) * d.y)) + (beta * d.x)) / (r33[i] * r33[i]);
        if (!is_close(d.x, 0)) w.x += a.x;
        if (!is_close(d.y, 0)) {
            w.x += ((-r12[i]) / r11[i]) * a.y;
            w.y += a.y;
        }
        if (!is_close(d.z, 0)) {
            w.x += beta * a.z;
            w.y += ((-r23[i]) / r22[i]) * a.z;
            w.z += a.z;
        }
        double t2 = 1 / vdot(d, d);
        return vmul(t2, w);
    };
    m.weight.assign(6 * (size_t)F, 0.0);
    m.foffset.resize(6 * (size_t)F);
    m.correction.resize(4 * (size_t)F);
    parallel_for(F, [&](int beg, int end) {
        for (int f = beg; f < end; f++) {
            int l = m.face_cell[2 * f], r = m.face_cell[2 * f + 1];
            Vec d = vsub(m.center[r], m.center[l]);
            Vec wl = face_weight(d, l);
            double *w = &m.weight[6 * (size_t)f];
            w[0] = wl.x, w[1] = wl.y, w[2] = wl.z;
            if (r < C) {
                Vec wr = face_weight(vmul(-1, d), r);
                w[3] = wr.x, w[4] = wr.y, w[5] = wr.z;
            }
            // offsets and corrections (generate.c:754-777)
            Vec ol = vsub(m.fcenter[f], m.center[l]), orr = vsub(m.fcenter[f], m.center[r]);
            double *o = &m.foffset[6 * (size_t)f];
            o[0] = ol.x, o[1] = ol.y, o[2] = ol.z, o[3] = orr.x, o[4] = orr.y, o[5] = orr.z;
            double nrm = vnorm(d);
            Vec unit = vdiv(d, nrm);
            double *cr = &m.correction[4 * (size_t)f];
            cr[0] = unit.x, cr[1] = unit.y, cr[2] = unit.z, cr[3] = nrm;
        }
    });
    return TG_OK;
}

int generate(tg_host_mesh &m)
{
    connect_cells(m);
    for (int i = 0; i < m.num_cells; i++) {
        if (m.cell_off[i + 1] - m.cell_off[i] > 6) return TG_ERR_INVALID;
    }
    reorder_cells(m);
    reorder_nodes(m);
    int rc = create_faces(m);
    if (rc != TG_OK) return rc;
    return geometry(m);
}

// mesh_split before generation (src/mesh/split.c:20-94): the cells of an inner or boundary entity
// whose node mean lies on the plane's non-positive side come first (in order), the others after
// them; the entity becomes "<name>-a" and "<name>-b", the second a copy of the first's transform;
// cells the periodic self-exchange sends are renumbered with them (reorder.c:123-131)
int split(tg_host_mesh &m, const char *name, const double *root_in, const double *normal_in)
{
    if (!name || !root_in || !normal_in) return TG_ERR_INVALID;
    int e = -1;
    for (int i = 0; i < m.off_boundary_entities; i++) {
        if (m.entities[i].name == name) {
            e = i;
            break;
        }
    }
    if (e < 0) return TG_ERR_INVALID;
    const Vec root = {root_in[0], root_in[1], root_in[2]}, normal = {normal_in[0], normal_in[1], normal_in[2]};
    const int beg = m.ent_cell_off[e], end = m.ent_cell_off[e + 1], n = end - beg;
    std::vector<int> map(n);
    int offset = 0;
    for (int i = 0; i < n; i++) {
        const int c = beg + i;
        Vec mean = {0, 0, 0};
        for (int j = m.node_off[c]; j < m.node_off[c + 1]; j++) mean = vadd(mean, m.coord[m.node_idx[j]]);
        mean = vdiv(mean, (double)(m.node_off[c + 1] - m.node_off[c]));
        map[i] = vdot(vsub(mean, root), normal) <= 0;
        offset += map[i];
    }
    int lhs = 0, rhs = 0;
    for (int i = 0; i < n; i++) map[i] = map[i] ? lhs++ : (offset + rhs++);
    // the entity's node lists in their new order
    std::vector<std::vector<int>> cells(n);
    for (int i = 0; i < n; i++) {
        const int c = beg + i;
        cells[map[i]].assign(m.node_idx.begin() + m.node_off[c], m.node_idx.begin() + m.node_off[c + 1]);
    }
    std::vector<int> idx(m.node_idx.begin(), m.node_idx.begin() + m.node_off[beg]);
    std::vector<int> off(m.node_off.begin(), m.node_off.begin() + beg + 1);
    for (int i = 0; i < n; i++) {
        idx.insert(idx.end(), cells[i].begin(), cells[i].end());
        off.push_back((int)idx.size());
    }
    for (int c = end; c < m.num_cells; c++) {
        idx.insert(idx.end(), m.node_idx.begin() + m.node_off[c], m.node_idx.begin() + m.node_off[c + 1]);
        off.push_back((int)idx.size());
    }
    m.node_idx.swap(idx);
    m.node_off.swap(off);
    for (int &k : m.send_idx) {
        if (beg <= k && k < end) k = beg + map[k - beg];
    }
    Entity copy = m.entities[e];
    m.entities[e].name += "-a";
    copy.name += "-b";
    m.entities.insert(m.entities.begin() + e + 1, copy);
    m.ent_cell_off.insert(m.ent_cell_off.begin() + e + 1, beg + offset);
    if (e < m.num_inner_entities) m.num_inner_entities += 1;
    m.off_boundary_entities += 1;  // the exchange tags stay as they are: they only pair entries
    return TG_OK;
}

int split_all(tg_host_mesh &m, int num_splits, const char *const *entity, const double *root, const double *normal)
{
    if (num_splits < 0 || (num_splits > 0 && (!entity || !root || !normal))) return TG_ERR_INVALID;
    for (int i = 0; i < num_splits; i++) {
        int rc = split(m, entity[i], root + 3 * i, normal + 3 * i);
        if (rc != TG_OK) return rc;
    }
    return TG_OK;
}

}  // namespace

extern "C" int tg_host_mesh_cartesian_split(const double *min_coord, const double *max_coord, const int *num_cells,
                                            const int *periodic, const double *displacement, int num_splits,
                                            const char *const *split_entity, const double *split_root,
                                            const double *split_normal, tg_host_mesh **out)
{
    if (!min_coord || !max_coord || !num_cells || !periodic || !out) return TG_ERR_INVALID;
    *out = nullptr;
    tg_host_mesh *m = new tg_host_mesh();
    int rc = cartesian(*m, min_coord, max_coord, num_cells, periodic, displacement);
    if (rc == TG_OK) rc = split_all(*m, num_splits, split_entity, split_root, split_normal);
    if (rc == TG_OK) rc = generate(*m);
    if (rc != TG_OK) {
        delete m;
        return rc;
    }
    *out = m;
    return TG_OK;
}

extern "C" int tg_host_mesh_cartesian(const double *min_coord, const double *max_coord, const int *num_cells,
                                      const int *periodic, const double *displacement, tg_host_mesh **out)
{
    return tg_host_mesh_cartesian_split(min_coord, max_coord, num_cells, periodic, displacement, 0, nullptr, nullptr,
                                        nullptr, out);
}

// One process's mesh given as teal holds it before generation (mesh_read's output, src/mesh/read.c):
// nodes, cells as node lists (inner cells with 4, 5, 6 or 8 nodes in Gmsh order, then boundary face
// cells with 3 or 4 nodes, then periodic face cells with 3 or 4 nodes), entities as cell ranges (inner,
// boundary, periodic), the periodic entities' rotation and translation (from the owner's side to the
// ghost's) and the periodic self-exchange (neighbour tags, receive and send offsets, sent cells).
extern "C" int tg_host_mesh_cells_periodic(int num_nodes, const double *coord, int num_cells, int num_inner_cells,
                                           int off_boundary_cells, const int *node_off, const int *node_idx,
                                           int num_entities, int off_boundary_entities,
                                           const char *const *entity_names, const int *entity_cell_off,
                                           const double *entity_rotation, const double *entity_translation,
                                           int num_neighbors, const int *neighbor_tag, const int *neighbor_recv_off,
                                           const int *neighbor_send_off, const int *neighbor_send_idx,
                                           int num_splits, const char *const *split_entity,
                                           const double *split_root, const double *split_normal,
                                           tg_host_mesh **out)
{
    if (!coord || !node_off || !node_idx || !entity_names || !entity_cell_off || !out) return TG_ERR_INVALID;
    *out = nullptr;
    if (num_nodes <= 0 || num_inner_cells <= 0 || off_boundary_cells < num_inner_cells ||
        num_cells < off_boundary_cells || num_entities < 1 || num_neighbors < 0) {
        return TG_ERR_INVALID;
    }
    if (node_off[0] != 0 || entity_cell_off[0] != 0 || entity_cell_off[num_entities] != num_cells) {
        return TG_ERR_INVALID;
    }
    if (off_boundary_entities < 1 || off_boundary_entities > num_entities ||
        entity_cell_off[off_boundary_entities] != off_boundary_cells) {
        return TG_ERR_INVALID;
    }
    if ((num_cells > off_boundary_cells || num_neighbors > 0) &&
        (!entity_rotation || !entity_translation || !neighbor_tag || !neighbor_recv_off || !neighbor_send_off ||
         !neighbor_send_idx)) {
        return TG_ERR_INVALID;
    }
    for (int i = 0; i < num_cells; i++) {
        int len = node_off[i + 1] - node_off[i];
        bool ok = (i < num_inner_cells) ? (len == 4 || len == 5 || len == 6 || len == 8) : (len == 3 || len == 4);
        if (!ok) return TG_ERR_INVALID;
        for (int j = node_off[i]; j < node_off[i + 1]; j++) {
            if (node_idx[j] < 0 || node_idx[j] >= num_nodes) return TG_ERR_INVALID;
        }
    }
    int num_inner_entities = 0;
    for (int e = 0; e < num_entities; e++) {
        if (entity_cell_off[e + 1] < entity_cell_off[e] || !entity_names[e]) return TG_ERR_INVALID;
        if (entity_cell_off[e + 1] <= num_inner_cells) num_inner_entities = e + 1;
    }
    if (entity_cell_off[num_inner_entities] != num_inner_cells) return TG_ERR_INVALID;
    if (num_neighbors > 0) {
        if (neighbor_recv_off[0] != off_boundary_cells || neighbor_recv_off[num_neighbors] != num_cells ||
            neighbor_send_off[0] != 0) {
            return TG_ERR_INVALID;
        }
        for (int k = 0; k < num_neighbors; k++) {
            if (neighbor_recv_off[k + 1] < neighbor_recv_off[k] || neighbor_send_off[k + 1] < neighbor_send_off[k]) {
                return TG_ERR_INVALID;
            }
        }
        for (int j = 0; j < neighbor_send_off[num_neighbors]; j++) {
            if (neighbor_send_idx[j] < 0 || neighbor_send_idx[j] >= num_inner_cells) return TG_ERR_INVALID;
        }
    }
    else if (num_cells != off_boundary_cells) {
        return TG_ERR_INVALID;
    }
    tg_host_mesh *m = new tg_host_mesh();
    m->coord.resize(num_nodes);
    for (int v = 0; v < num_nodes; v++) m->coord[v] = {coord[3 * v], coord[3 * v + 1], coord[3 * v + 2]};
    m->num_cells = num_cells;
    m->num_inner = num_inner_cells;
    m->off_boundary = off_boundary_cells;
    m->off_periodic = num_cells;
    m->node_off.assign(node_off, node_off + num_cells + 1);
    m->node_idx.assign(node_idx, node_idx + node_off[num_cells]);
    m->num_inner_entities = num_inner_entities;
    m->off_boundary_entities = off_boundary_entities;
    for (int e = 0; e < num_entities; e++) {
        Entity en{};
        en.name = entity_names[e];
        if (entity_rotation) memcpy(en.rotation, entity_rotation + 9 * (size_t)e, sizeof(en.rotation));
        if (entity_translation) {
            en.translation = {entity_translation[3 * e], entity_translation[3 * e + 1], entity_translation[3 * e + 2]};
        }
        m->entities.push_back(en);
    }
    m->ent_cell_off.assign(entity_cell_off, entity_cell_off + num_entities + 1);
    if (num_neighbors > 0) {
        m->tag.assign(neighbor_tag, neighbor_tag + 2 * (size_t)num_neighbors);
        m->recv_off.assign(neighbor_recv_off, neighbor_recv_off + num_neighbors + 1);
        m->send_off.assign(neighbor_send_off, neighbor_send_off + num_neighbors + 1);
        m->send_idx.assign(neighbor_send_idx, neighbor_send_idx + neighbor_send_off[num_neighbors]);
    }
    else {
        m->recv_off.assign(1, num_cells);
        m->send_off.assign(1, 0);
    }
    int rc = split_all(*m, num_splits, split_entity, split_root, split_normal);
    if (rc == TG_OK) rc = generate(*m);
    if (rc != TG_OK) {
        delete m;
        return rc;
    }
    *out = m;
    return TG_OK;
}

// The same without periodic entities: inner cells, then boundary face cells
extern "C" int tg_host_mesh_cells(int num_nodes, const double *coord, int num_cells, int num_inner_cells,
                                  const int *node_off, const int *node_idx, int num_entities,
                                  const char *const *entity_names, const int *entity_cell_off,
                                  tg_host_mesh **out)
{
    return tg_host_mesh_cells_periodic(num_nodes, coord, num_cells, num_inner_cells, num_cells, node_off, node_idx,
                                       num_entities, num_entities, entity_names, entity_cell_off, nullptr, nullptr, 0,
                                       nullptr, nullptr, nullptr, nullptr, 0, nullptr, nullptr, nullptr, out);
}

extern "C" int tg_host_mesh_view(const tg_host_mesh *m, tg_mesh *v)
{
    if (!m || !v) return TG_ERR_INVALID;
    memset(v, 0, sizeof(*v));
    v->num_cells = m->num_cells;
    v->num_inner_cells = m->num_inner;
    v->off_boundary_cells = m->off_boundary;
    v->off_periodic_cells = m->off_periodic;
    v->cell_cell_off = m->cell_off.data();
    v->cell_cell_idx = m->cell_idx.data();
    v->cell_volume = m->volume.data();
    v->cell_center = &m->center[0].x;
    v->cell_projection = &m->projection[0].x;
    v->cell_offset = m->offset.empty() ? nullptr : &m->offset[0].x;
    v->sum_volume = m->sum_volume;
    v->num_faces = m->num_faces;
    v->num_inner_faces = m->num_inner_faces;
    v->off_boundary_faces = m->off_boundary_faces;
    v->face_cell = m->face_cell.data();
    v->face_area = m->area.data();
    v->face_basis = m->basis.data();
    v->face_weight = m->weight.data();
    v->face_offset = m->foffset.data();
    v->face_correction = m->correction.data();
    v->num_entities = (int)m->entities.size();
    v->num_inner_entities = m->num_inner_entities;
    v->off_boundary_entities = m->off_boundary_entities;
    v->entity_face_off = m->ent_face_off.data();
    v->num_neighbors = (int)m->recv_off.size() - 1;
    v->neighbor_tag = m->tag.data();
    v->neighbor_recv_off = m->recv_off.data();
    v->neighbor_send_off = m->send_off.data();
    v->neighbor_send_idx = m->send_idx.data();
    return TG_OK;
}

extern "C" int tg_host_mesh_entity(const tg_host_mesh *m, int index, const char **name, int *cell_beg,
                                   int *cell_end)
{
    if (!m || index < 0 || index >= (int)m->entities.size()) return TG_ERR_INVALID;
    if (name) *name = m->entities[index].name.c_str();
    if (cell_beg) *cell_beg = m->ent_cell_off[index];
    if (cell_end) *cell_end = m->ent_cell_off[index + 1];
    return TG_OK;
}

extern "C" int tg_host_mesh_nodes(const tg_host_mesh *m, int *num_nodes, const double **coord,
                                  const int **cell_node_off, const int **cell_node_idx)
{
    if (!m || !num_nodes || !coord || !cell_node_off || !cell_node_idx) return TG_ERR_INVALID;
    *num_nodes = (int)m->coord.size();
    *coord = m->coord.empty() ? nullptr : &m->coord[0].x;
    *cell_node_off = m->node_off.data();
    *cell_node_idx = m->node_idx.data();
    return TG_OK;
}

extern "C" int tg_host_mesh_destroy(tg_host_mesh *m)
{
    delete m;
    return TG_OK;
}
