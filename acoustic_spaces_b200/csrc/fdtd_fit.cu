// Fitted walls on the GPU: the FP64 cut of a convex room's walls by the wave grid's cells
// (include/fdtd_b200.h: fdtd_cut_convex). The reference fits a triangle mesh by an exact lattice
// kernel on the host (cpp/include/acoustic_spaces/cut_cells.hpp, CutCells, used by set_up_fitted,
// fdtd.hpp:970-1217); this is the same measure for the rooms the reference's fitted walls are
// most often given — convex polyhedra of planar walls, one face of which may be left open — in
// double precision, one cell a thread.
//
// A room is P = {x : n_f . x <= d_f for every plane f} (n_f unit, pointing out of the room); its
// walls are the faces of P on the planes that are not open. In a cell's own coordinates
// u = (x - corner) / h in [0, 1]^3 plane f reads n_f . u <= e_f with e_f = (d_f - n_f . corner) / h.
// A wall's plane splits a cell it crosses (as the reference's fit splits a cell along the plane of
// a face that meets it), so a cell's air inside the walls is Q = cube ∩ {n_f . u <= e_f for every
// wall f}. For each cell whose walls' planes cut it (its corners on both sides):
//   * the area of each of its six faces in Q: the unit square clipped by the walls' half-planes
//     (Sutherland-Hodgman);
//   * the volume of Q by the divergence theorem, (1/3) of the sum over its faces of (u . n) times
//     the face's area: the faces at u_a = 1 give their areas, those at u_a = 0 give nothing, and
//     the section of wall plane f gives e_f times its area;
//   * each wall's area in the cell: its plane's section clipped by every other plane, the open
//     ones included (0 where the wall does not reach into the cell).
// The rest of the cell (cube minus Q) is its air outside the walls.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "fdtd_b200.h"

namespace {

constexpr int kBlockFit = 128;
constexpr int kMaxPlanes = FDTD_CUT_MAX_PLANES;
constexpr int kMaxPieces = FDTD_CUT_MAX_PIECES;
constexpr int kMaxColumns = kMaxPieces > kMaxPlanes ? kMaxPieces : kMaxPlanes;
constexpr int kMaxCut = 16;    // planes cutting one cell, at most
constexpr int kMaxPoly = 32;   // vertices of a clipped polygon, at most

// Whether plane f cuts cell (x, y, z): its corners on both sides (strictly).
__host__ __device__ inline void plane_range(const double *n, double e, double &lo, double &hi) {
    lo = 0.0, hi = 0.0;
    for (int a = 0; a < 3; ++a) {
        if (n[a] > 0) hi += n[a];
        else lo += n[a];
    }
    lo -= e, hi -= e;  // n . u - e over the cube: [lo, hi]
}

// The area of a planar polygon (3-D points) by the norm of the summed cross products.
__host__ __device__ inline double area3(const double (*p)[3], int count) {
    double s[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < count; ++i) {
        const double *a = p[i], *b = p[(i + 1) % count];
        s[0] += a[1] * b[2] - a[2] * b[1];
        s[1] += a[2] * b[0] - a[0] * b[2];
        s[2] += a[0] * b[1] - a[1] * b[0];
    }
    return 0.5 * sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
}

// Clips the polygon p (count vertices) by n . u <= e (Sutherland-Hodgman); returns the new count.
__host__ __device__ inline int clip3(double (*p)[3], int count, const double *n, double e) {
    double q[kMaxPoly][3];
    int m = 0;
    for (int i = 0; i < count && m < kMaxPoly - 1; ++i) {
        const double *a = p[i], *b = p[(i + 1) % count];
        const double sa = n[0] * a[0] + n[1] * a[1] + n[2] * a[2] - e;
        const double sb = n[0] * b[0] + n[1] * b[1] + n[2] * b[2] - e;
        if (sa <= 0.0) {
            q[m][0] = a[0], q[m][1] = a[1], q[m][2] = a[2];
            ++m;
        }
        if ((sa < 0.0 && sb > 0.0) || (sa > 0.0 && sb < 0.0)) {
            const double t = sa / (sa - sb);
            for (int k = 0; k < 3; ++k) q[m][k] = a[k] + t * (b[k] - a[k]);
            ++m;
        }
    }
    for (int i = 0; i < m; ++i) p[i][0] = q[i][0], p[i][1] = q[i][1], p[i][2] = q[i][2];
    return m;
}

// The section of the unit cube by the plane n . u = e, as a polygon ordered round its centroid.
__host__ __device__ inline int section(const double *n, double e, double (*p)[3]) {
    // The cube's twelve edges: from corner c along axis a.
    int count = 0;
    for (int a = 0; a < 3; ++a) {
        const int b = (a + 1) % 3, c = (a + 2) % 3;
        for (int j = 0; j < 4; ++j) {
            double u[3];
            u[b] = (double)(j & 1), u[c] = (double)(j >> 1);
            // n_a t + n_b u_b + n_c u_c = e
            if (n[a] == 0.0) continue;
            const double t = (e - n[b] * u[b] - n[c] * u[c]) / n[a];
            if (t < 0.0 || t > 1.0) continue;
            u[a] = t;
            p[count][0] = u[0], p[count][1] = u[1], p[count][2] = u[2];
            ++count;
        }
    }
    if (count < 3) return 0;
    // Order round the centroid in the plane's own frame.
    double cx = 0, cy = 0, cz = 0;
    for (int i = 0; i < count; ++i) cx += p[i][0], cy += p[i][1], cz += p[i][2];
    cx /= count, cy /= count, cz /= count;
    // A frame (e1, e2) of the plane.
    double e1[3];
    if (fabs(n[0]) < 0.9) e1[0] = 0, e1[1] = -n[2], e1[2] = n[1];
    else e1[0] = n[2], e1[1] = 0, e1[2] = -n[0];
    const double l = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
    e1[0] /= l, e1[1] /= l, e1[2] /= l;
    const double e2[3] = {n[1] * e1[2] - n[2] * e1[1], n[2] * e1[0] - n[0] * e1[2], n[0] * e1[1] - n[1] * e1[0]};
    double angle[12];
    for (int i = 0; i < count; ++i) {
        const double dx = p[i][0] - cx, dy = p[i][1] - cy, dz = p[i][2] - cz;
        angle[i] = atan2(dx * e2[0] + dy * e2[1] + dz * e2[2], dx * e1[0] + dy * e1[1] + dz * e1[2]);
    }
    for (int i = 1; i < count; ++i)  // insertion sort by angle
        for (int j = i; j > 0 && angle[j - 1] > angle[j]; --j) {
            const double ta = angle[j];
            angle[j] = angle[j - 1], angle[j - 1] = ta;
            for (int k = 0; k < 3; ++k) {
                const double t = p[j][k];
                p[j][k] = p[j - 1][k], p[j - 1][k] = t;
            }
        }
    return count;
}

struct CutArgs {
    const double *normals;  // planes x 3
    const double *offsets;  // planes
    const uint8_t *open;    // planes (null: every plane a wall)
    uint32_t planes;
    // The walls in pieces (pieces 0: one a plane): piece k on plane piece_plane[k], inside the
    // half-spaces piece_edges[4 e ..] for e in piece_start[k] .. piece_start[k + 1] - 1.
    uint32_t pieces;
    const uint32_t *piece_plane, *piece_start;
    const double *piece_edges;
    uint32_t columns;  // caps a cell: pieces, else planes
    double origin[3], cell;
    uint64_t nx, ny, nz;
    // Outputs (capacity cells): each cut cell's index, the volume inside the room (cells^3), the
    // areas of its six faces inside the room (-x, +x, -y, +y, -z, +z; cell faces) and each plane's
    // cap (planes values a cell).
    unsigned long long *count;
    uint64_t capacity;
    uint64_t *cell_out;
    double *volume, *face_area, *cap, *bare;
};

// One cell of the fit: whether the walls cut it (false: wholly on one side of them) and, where
// they do, the volume of its air inside the walls, the areas of its faces inside the walls and
// each wall's area in it. The walls' planes bound the regions (a cell is split along the whole of
// each wall plane that crosses it); an open plane bounds only the walls' faces (the room's open
// face is no wall, and the air meets through it).
__host__ __device__ inline bool cut_cell(const CutArgs &g, uint64_t i, double *volume_out, double *face_out,
                                         double *cap_out, double *bare_out) {
    const uint64_t x = i % g.nx, y = (i / g.nx) % g.ny, z = i / (g.nx * g.ny);
    // The cell's corner as the grid's doubles give it (origin + i cell, fdtd.hpp:1620-1634).
    const double corner[3] = {g.origin[0] + (double)x * g.cell, g.origin[1] + (double)y * g.cell,
                              g.origin[2] + (double)z * g.cell};
    int cut[kMaxCut];
    double e[kMaxCut];
    bool open[kMaxCut];
    int cuts = 0, walls = 0;
    for (uint32_t f = 0; f < g.planes; ++f) {
        const double *nf = g.normals + 3 * f;
        const double ef = (g.offsets[f] - (nf[0] * corner[0] + nf[1] * corner[1] + nf[2] * corner[2])) / g.cell;
        double lo, hi;
        plane_range(nf, ef, lo, hi);
        const bool is_open = g.open && g.open[f];
        if (lo >= 0.0 && !is_open) return false;  // the whole cell beyond a wall's plane: uncut
        if (lo < 0.0 && hi > 0.0 && cuts < kMaxCut) {
            cut[cuts] = (int)f, e[cuts] = ef, open[cuts] = is_open, ++cuts;
            walls += !is_open;
        }
        if (lo >= 0.0 && is_open && cuts < kMaxCut) {
            // wholly beyond the open face: it bounds every wall face to nothing here
            cut[cuts] = (int)f, e[cuts] = ef, open[cuts] = true, ++cuts;
        }
    }
    if (walls == 0) return false;
    // The six faces inside the walls: each a unit square in the cell's coordinates, clipped.
    for (int face = 0; face < 6; ++face) {
        const int a = face / 2;
        const double at = (double)(face & 1);
        double p[kMaxPoly][3];
        const int b = (a + 1) % 3, c = (a + 2) % 3;
        for (int k = 0; k < 4; ++k) {
            p[k][a] = at;
            p[k][b] = (double)((k == 1 || k == 2) ? 1 : 0);
            p[k][c] = (double)(k >= 2 ? 1 : 0);
        }
        int m = 4;
        for (int q = 0; q < cuts && m > 0; ++q)
            if (!open[q]) m = clip3(p, m, g.normals + 3 * cut[q], e[q]);
        face_out[face] = m >= 3 ? area3(p, m) : 0.0;
    }
    // Each wall plane's section inside the other walls (for the volume, by the divergence
    // theorem) and inside the open planes too (the wall's own area in the cell).
    double volume = face_out[1] + face_out[3] + face_out[5], bare = 0.0;
    for (uint32_t f = 0; f < g.columns; ++f) cap_out[f] = 0.0;
    for (int q = 0; q < cuts; ++q) {
        if (open[q]) continue;
        double p[kMaxPoly][3];
        int m = section(g.normals + 3 * cut[q], e[q], p);
        for (int r = 0; r < cuts && m > 0; ++r)
            if (r != q && !open[r]) m = clip3(p, m, g.normals + 3 * cut[r], e[r]);
        const double facet = m >= 3 ? area3(p, m) : 0.0;
        volume += e[q] * facet;
        for (int r = 0; r < cuts && m > 0; ++r)
            if (open[r]) m = clip3(p, m, g.normals + 3 * cut[r], e[r]);
        // (the wall's area in the cell: the pieces split it by material, a rounding apart)
        const double covered = m >= 3 ? area3(p, m) : 0.0;
        if (!g.pieces) {
            cap_out[cut[q]] = covered;
        } else {
            // each piece of the wall: the wall's part in the cell clipped by the piece's edges
            for (uint32_t k = 0; k < g.pieces && m >= 3; ++k) {
                if (g.piece_plane[k] != (uint32_t)cut[q]) continue;
                double w[kMaxPoly][3];
                for (int v = 0; v < m; ++v) w[v][0] = p[v][0], w[v][1] = p[v][1], w[v][2] = p[v][2];
                int wm = m;
                for (uint32_t h = g.piece_start[k]; h < g.piece_start[k + 1] && wm > 0; ++h) {
                    const double *edge = g.piece_edges + 4 * h;
                    const double eh =
                        (edge[3] - (edge[0] * corner[0] + edge[1] * corner[1] + edge[2] * corner[2])) / g.cell;
                    wm = clip3(w, wm, edge, eh);
                }
                cap_out[k] = wm >= 3 ? area3(w, wm) : 0.0;
            }
        }
        // the part of the facet no wall covers (beyond the open face): the air meets across it
        bare += facet - covered;
    }
    *volume_out = volume / 3.0;
    *bare_out = bare;
    return true;
}

__global__ void __launch_bounds__(kBlockFit) cut_kernel(const CutArgs g) {
    const uint64_t n = g.nx * g.ny * g.nz;
    for (uint64_t i = blockIdx.x * (uint64_t)kBlockFit + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kBlockFit) {
        double volume, face[6], cap[kMaxColumns], bare;
        if (!cut_cell(g, i, &volume, face, cap, &bare)) continue;
        const unsigned long long slot = atomicAdd(g.count, 1ull);
        if (slot >= g.capacity) continue;  // the host sees the count and grows the buffers
        g.cell_out[slot] = i;
        g.volume[slot] = volume;
        g.bare[slot] = bare;
        for (int k = 0; k < 6; ++k) g.face_area[slot * 6 + k] = face[k];
        for (uint32_t f = 0; f < g.columns; ++f) g.cap[slot * g.columns + f] = cap[f];
    }
}

thread_local std::string g_fit_error;

int fit_fail(int status, const std::string &message) {
    g_fit_error = message;
    return status;
}

}  // namespace

extern "C" {

const char *fdtd_cut_error(void) { return g_fit_error.c_str(); }

int fdtd_cut_convex(const fdtd_cut_room *room, int device, fdtd_cut_cells *out) {
    if (!room || !out) return fit_fail(FDTD_EINVAL, "no room or no output");
    std::memset(out, 0, sizeof *out);
    if (room->planes == 0 || room->planes > kMaxPlanes)
        return fit_fail(FDTD_EINVAL, "a convex room has 1 to " + std::to_string(kMaxPlanes) + " planes");
    if (!(room->cell > 0.0) || room->nx == 0 || room->ny == 0 || room->nz == 0)
        return fit_fail(FDTD_EINVAL, "the grid needs a positive cell and sizes");
    for (uint32_t f = 0; f < room->planes; ++f) {
        const double *nf = room->normals + 3 * f;
        const double l = nf[0] * nf[0] + nf[1] * nf[1] + nf[2] * nf[2];
        if (!(std::abs(l - 1.0) < 1e-9)) return fit_fail(FDTD_EINVAL, "each plane's normal is a unit vector");
    }
    const uint32_t K = room->pieces;
    std::vector<uint32_t> piece_start;
    if (K) {
        if (K > (uint32_t)kMaxPieces)
            return fit_fail(FDTD_EINVAL, "the walls have 1 to " + std::to_string(kMaxPieces) + " pieces");
        if (!room->piece_plane || !room->piece_start || !room->piece_edges)
            return fit_fail(FDTD_EINVAL, "the walls' pieces miss their planes, starts or edges");
        if (room->piece_start[0] != 0) return fit_fail(FDTD_EINVAL, "piece_start does not start at 0");
        for (uint32_t k = 0; k < K; ++k) {
            if (room->piece_plane[k] >= room->planes) return fit_fail(FDTD_EINVAL, "a piece lies on no plane of the room");
            if (room->open && room->open[room->piece_plane[k]])
                return fit_fail(FDTD_EINVAL, "a piece of wall lies on an open plane");
            if (room->piece_start[k + 1] < room->piece_start[k] || room->piece_start[k + 1] - room->piece_start[k] > 64)
                return fit_fail(FDTD_EINVAL, "a piece has 0 to 64 edges, in order");
        }
        piece_start.assign(room->piece_start, room->piece_start + K + 1);
    }
    const uint32_t edges = K ? piece_start[K] : 0;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return fit_fail(FDTD_ENODEV, "no CUDA device for the fit");
    }
    int previous = 0;
    cudaGetDevice(&previous);
    cudaSetDevice(device);
    const uint64_t n = room->nx * room->ny * room->nz;
    const uint32_t P = room->planes, columns = K ? K : P;
    // Capacity from the planes' area: a cut cell lies within a cell of a plane; start from a
    // generous guess and grow once if it fell short.
    uint64_t capacity = std::min<uint64_t>(n, 1u << 20);
    std::vector<void *> held;
    auto release = [&]() {
        for (void *p : held) cudaFree(p);
        held.clear();
        cudaSetDevice(previous);
    };
    auto check = [&](cudaError_t e, const char *what) {
        if (e == cudaSuccess) return FDTD_OK;
        const int status = e == cudaErrorMemoryAllocation ? FDTD_ENOMEM : FDTD_ECUDA;
        fit_fail(status, std::string(what) + ": " + cudaGetErrorString(e));
        return status;
    };
    int rc;
    double *d_normals = nullptr, *d_offsets = nullptr;
    unsigned long long *d_count = nullptr;
    if ((rc = check(cudaMalloc(&d_normals, 24 * P), "cudaMalloc"))) return release(), rc;
    held.push_back(d_normals);
    if ((rc = check(cudaMalloc(&d_offsets, 8 * P), "cudaMalloc"))) return release(), rc;
    held.push_back(d_offsets);
    if ((rc = check(cudaMalloc(&d_count, 8), "cudaMalloc"))) return release(), rc;
    held.push_back(d_count);
    uint8_t *d_open = nullptr;
    if ((rc = check(cudaMalloc(&d_open, P), "cudaMalloc"))) return release(), rc;
    held.push_back(d_open);
    cudaMemcpy(d_normals, room->normals, 24 * P, cudaMemcpyHostToDevice);
    cudaMemcpy(d_offsets, room->offsets, 8 * P, cudaMemcpyHostToDevice);
    std::vector<uint8_t> open(P, 0);
    if (room->open)
        for (uint32_t f = 0; f < P; ++f) open[f] = room->open[f] ? 1 : 0;
    cudaMemcpy(d_open, open.data(), P, cudaMemcpyHostToDevice);
    uint32_t *d_piece_plane = nullptr, *d_piece_start = nullptr;
    double *d_piece_edges = nullptr;
    if (K) {
        if ((rc = check(cudaMalloc(&d_piece_plane, 4 * K), "cudaMalloc"))) return release(), rc;
        held.push_back(d_piece_plane);
        if ((rc = check(cudaMalloc(&d_piece_start, 4 * (K + 1)), "cudaMalloc"))) return release(), rc;
        held.push_back(d_piece_start);
        if ((rc = check(cudaMalloc(&d_piece_edges, 32 * std::max<uint32_t>(1, edges)), "cudaMalloc"))) return release(), rc;
        held.push_back(d_piece_edges);
        cudaMemcpy(d_piece_plane, room->piece_plane, 4 * K, cudaMemcpyHostToDevice);
        cudaMemcpy(d_piece_start, piece_start.data(), 4 * (K + 1), cudaMemcpyHostToDevice);
        if (edges) cudaMemcpy(d_piece_edges, room->piece_edges, 32 * edges, cudaMemcpyHostToDevice);
    }
    for (int attempt = 0; attempt < 2; ++attempt) {
        CutArgs g{};
        g.normals = d_normals, g.offsets = d_offsets, g.open = d_open, g.planes = P;
        g.pieces = K, g.piece_plane = d_piece_plane, g.piece_start = d_piece_start, g.piece_edges = d_piece_edges;
        g.columns = columns;
        for (int a = 0; a < 3; ++a) g.origin[a] = room->origin[a];
        g.cell = room->cell, g.nx = room->nx, g.ny = room->ny, g.nz = room->nz;
        g.count = d_count, g.capacity = capacity;
        uint64_t *d_cell = nullptr;
        double *d_volume = nullptr, *d_face = nullptr, *d_cap = nullptr, *d_bare = nullptr;
        if ((rc = check(cudaMalloc(&d_cell, 8 * capacity), "cudaMalloc"))) return release(), rc;
        held.push_back(d_cell);
        if ((rc = check(cudaMalloc(&d_volume, 8 * capacity), "cudaMalloc"))) return release(), rc;
        held.push_back(d_volume);
        if ((rc = check(cudaMalloc(&d_face, 48 * capacity), "cudaMalloc"))) return release(), rc;
        held.push_back(d_face);
        if ((rc = check(cudaMalloc(&d_cap, 8 * (uint64_t)columns * capacity), "cudaMalloc"))) return release(), rc;
        held.push_back(d_cap);
        if ((rc = check(cudaMalloc(&d_bare, 8 * capacity), "cudaMalloc"))) return release(), rc;
        held.push_back(d_bare);
        g.cell_out = d_cell, g.volume = d_volume, g.face_area = d_face, g.cap = d_cap, g.bare = d_bare;
        cudaMemset(d_count, 0, 8);
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const uint64_t blocks = std::min<uint64_t>((n + kBlockFit - 1) / kBlockFit, (uint64_t)sms * 16);
        cut_kernel<<<(unsigned)blocks, kBlockFit>>>(g);
        if ((rc = check(cudaGetLastError(), "cut_kernel"))) return release(), rc;
        unsigned long long found = 0;
        if ((rc = check(cudaMemcpy(&found, d_count, 8, cudaMemcpyDeviceToHost), "cut_kernel"))) return release(), rc;
        if (found > capacity) {
            // Too few slots: free this attempt's buffers and run again with room for all.
            for (int k = 0; k < 5; ++k) cudaFree(held.back()), held.pop_back();
            capacity = found;
            continue;
        }
        out->cells = found;
        out->planes = columns;
        out->cell = static_cast<uint64_t *>(std::malloc(8 * std::max<uint64_t>(1, found)));
        out->volume = static_cast<double *>(std::malloc(8 * std::max<uint64_t>(1, found)));
        out->face_area = static_cast<double *>(std::malloc(48 * std::max<uint64_t>(1, found)));
        out->cap = static_cast<double *>(std::malloc(8 * (uint64_t)columns * std::max<uint64_t>(1, found)));
        out->bare = static_cast<double *>(std::malloc(8 * std::max<uint64_t>(1, found)));
        if (!out->cell || !out->volume || !out->face_area || !out->cap || !out->bare) {
            fdtd_cut_free(out);
            release();
            return fit_fail(FDTD_ENOMEM, "out of host memory for the fit's cells");
        }
        cudaMemcpy(out->cell, d_cell, 8 * found, cudaMemcpyDeviceToHost);
        cudaMemcpy(out->volume, d_volume, 8 * found, cudaMemcpyDeviceToHost);
        cudaMemcpy(out->face_area, d_face, 48 * found, cudaMemcpyDeviceToHost);
        cudaMemcpy(out->bare, d_bare, 8 * found, cudaMemcpyDeviceToHost);
        rc = check(cudaMemcpy(out->cap, d_cap, 8 * (uint64_t)columns * found, cudaMemcpyDeviceToHost), "cudaMemcpy");
        release();
        if (rc) fdtd_cut_free(out);
        return rc;
    }
    release();
    return fit_fail(FDTD_ECUDA, "the fit's count of cut cells changed between two runs");
}

void fdtd_cut_free(fdtd_cut_cells *out) {
    if (!out) return;
    std::free(out->cell), std::free(out->volume), std::free(out->face_area), std::free(out->cap), std::free(out->bare);
    std::memset(out, 0, sizeof *out);
}

}  // extern "C"
