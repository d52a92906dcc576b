// Direct-hop (DH) structured grid of the FemPIC move and of the 2-D NESO-advection move
// (include/oppb_dh.h): the host set-up of the grid (OP-PIC's BoundingBox and
// CellMapper::init_host) and its build on the GPU.
//
// The reference fills the map on the host by testing, for each grid box, every mesh cell in
// index order until one contains the query point (opp_lib/src/seq/opp_direct_hop_seq.cpp:
// 134-302 with the checker of apps_codegen/app_fempic_cg/seq/move_kernel_loop.hpp:170-198):
// O(boxes x cells), hours at millions of cells.  Here the answer is the same, the lowest
// index among the cells whose FP64 barycentric test accepts the point, but the candidates
// come from a binning of the cells into the grid boxes:
//   1. every cell is binned into each box that its node bounding box, widened by 1/1000 of
//      its extent, overlaps (count, exclusive scan, fill);
//   2. one thread per box runs the reference's query sequence, testing only the cells
//      binned into the box that holds each query point.
// A cell accepts a point only within the 1e-10 tolerance of its barycentric weights, far
// inside the widening, and the bin of a coordinate is monotone in it, so every accepting
// cell is among the candidates of the point's box: the lowest accepting index is found.
// The advection mesh's square cells go through the same two kernels with the app's
// all-cell checker (apps_codegen/app_neso_advection_mdir_cg/seq/move_kernel_loop.hpp:
// 194-219): a square accepts a point when the move kernel's FP64 differences p - ll lie in
// [0, cell_width] on both axes, i.e. at most one rounding beyond the square, again far inside
// the widening.  A 2-D grid has one box along z (min = max = 0), where every z bin is 0.

#include <cfloat>
#include <cmath>

#include "oppb_common.cuh"
#include "oppb_dh.h"
#include "scan.cuh"
#include "tet_f64.cuh"

namespace oppb {
namespace {

constexpr int kDhBlock = 256;
constexpr double kBoundOffset = 1e-12;  // BOUND_OFFSET, opp_lib/include/opp_direct_hop_core.h:37
constexpr double kBinWiden = 1e-3;      // cells are binned with their box widened by this share of its extent
constexpr int64_t kMaxLoop = int64_t(1) << 31;

struct GridArgs {
    double min[3], max[3];
    double h;
    int64_t dims[3];
};

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Bin of coordinate v on axis d: (v - min) / h truncated and clamped to [0, dims - 1].
// Non-decreasing in v.
__device__ __forceinline__ int64_t bin_of(const GridArgs& g, int d, double v) {
    const double t = __ddiv_rn(__dsub_rn(v, g.min[d]), g.h);
    if (!(t > 0.0)) return 0;
    if (t >= (double)(g.dims[d] - 1)) return g.dims[d] - 1;
    return (int64_t)t;
}

// Tetrahedra of the FemPIC mesh: node bounding boxes, and the move kernel's FP64 barycentric
// test (apps_codegen/app_fempic_cg/seq/move_kernel_loop.hpp:170-198).
struct TetCells {
    oppb_tet_mesh m;
    const double* npos;  // SoA [3][n_nodes]
    __device__ int32_t count() const { return m.n_cells; }
    // Node bounding box of cell c; false for a cell with a node index out of range.
    __device__ bool bounds(int32_t c, double lo[3], double hi[3]) const {
        const int4 nd = ldg_i4(m.c2n + (int64_t)c * 4);
        const int n[4] = {nd.x, nd.y, nd.z, nd.w};
#pragma unroll
        for (int d = 0; d < 3; d++) lo[d] = DBL_MAX, hi[d] = -DBL_MAX;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if ((uint32_t)n[k] >= (uint32_t)m.n_nodes) return false;
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const double v = __ldg(npos + (int64_t)d * m.n_nodes + n[k]);
                lo[d] = fmin(lo[d], v);
                hi[d] = fmax(hi[d], v);
            }
        }
        return true;
    }
    __device__ bool holds(int32_t c, const double p[3]) const {
        double l[4];
        int nb[4];
        visit_f64(m, c, p[0], p[1], p[2], l, nb);
        return inside_f64(l);
    }
};

// Squares of one NESO-advection instance (packed records {c_pos_ll x, y, c2c}, include/oppb_advec.h):
// the square [ll, ll + w]^2 at z = 0, and move_kernel's in-cell test of its first call
// (apps/app_neso_advection/kernels.h move_kernel, step 2 on both axes).
struct QuadCells {
    const double* cells;  // the instance's first record, [n][4]
    int32_t n;
    double w;             // CONST_cell_width
    __device__ int32_t count() const { return n; }
    __device__ bool bounds(int32_t c, double lo[3], double hi[3]) const {
        const double2 ll = ldg_d2(cells + (int64_t)c * 4);
        lo[0] = ll.x, lo[1] = ll.y, lo[2] = 0.0;
        hi[0] = ll.x + w, hi[1] = ll.y + w, hi[2] = 0.0;
        return true;
    }
    __device__ bool holds(int32_t c, const double p[3]) const {
        const double2 ll = ldg_d2(cells + (int64_t)c * 4);
        const double dx = __dsub_rn(p[0], ll.x), dy = __dsub_rn(p[1], ll.y);
        return (dx >= 0.0) && (dx <= w) && (dy >= 0.0) && (dy <= w);
    }
};

// Bounding box of cell c, widened; false for a cell with a node index out of range.
template <class Cells>
__device__ __forceinline__ bool cell_bins(const Cells& cs, int32_t c, const GridArgs& g, int64_t b0[3],
                                          int64_t b1[3]) {
    double lo[3], hi[3];
    if (!cs.bounds(c, lo, hi)) return false;
    const double ext = fmax(fmax(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]);
    const double w = kBinWiden * ext;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        b0[d] = bin_of(g, d, lo[d] - w);
        b1[d] = bin_of(g, d, hi[d] + w);
    }
    return true;
}

// kMode 0: add the number of (cell, box) pairs to *pairs; 1: count the cells of every box;
// 2: write each cell into its boxes' lists.
template <int kMode, class Cells>
__global__ void __launch_bounds__(kDhBlock) dh_bin_kernel(Cells cs, GridArgs g, unsigned long long* pairs,
                                                          int* counts, int* cursor, int* list) {
    const int32_t c = (int32_t)(blockIdx.x * kDhBlock + threadIdx.x);
    int64_t b0[3], b1[3];
    const bool ok = c < cs.count() && cell_bins(cs, c, g, b0, b1);
    if (kMode == 0) {
        unsigned long long s =
            ok ? (unsigned long long)((b1[0] - b0[0] + 1) * (b1[1] - b0[1] + 1) * (b1[2] - b0[2] + 1)) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFullMask, s, o);
        if ((threadIdx.x & 31) == 0 && s) atomicAdd(pairs, s);
        return;
    }
    if (!ok) return;
    for (int64_t z = b0[2]; z <= b1[2]; z++)
        for (int64_t y = b0[1]; y <= b1[1]; y++)
            for (int64_t x = b0[0]; x <= b1[0]; x++) {
                const int64_t b = x + g.dims[0] * (y + g.dims[1] * z);
                if (kMode == 1)
                    atomicAdd(counts + b, 1);
                else
                    list[atomicAdd(cursor + b, 1)] = c;
            }
}

// Lowest-index cell whose test (the move kernel's) accepts p, or kRemoved.
template <class Cells>
__device__ int32_t first_cell(const Cells& cs, const GridArgs& g, const int* offsets, const int* list,
                              const double p[3]) {
    const int64_t b = bin_of(g, 0, p[0]) + g.dims[0] * (bin_of(g, 1, p[1]) + g.dims[1] * bin_of(g, 2, p[2]));
    int32_t best = kRemoved;
    for (int k = offsets[b]; k < offsets[b + 1]; k++) {
        const int32_t c = list[k];
        if (c < best && cs.holds(c, p)) best = c;
    }
    return best;
}

// One thread per grid box: generateStructuredMesh steps 1 and 3 for the box.  On a 2-D grid
// the z nudge repeats the x/y query and the upper z corners clamp onto the lower ones, so the
// answer is the 2-D one (the reference's 4 corners).
template <class Cells>
__global__ void __launch_bounds__(kDhBlock) dh_query_kernel(Cells cs, GridArgs g, const int* offsets,
                                                            const int* list, int32_t* map, int64_t size) {
    const int64_t idx = (int64_t)blockIdx.x * kDhBlock + threadIdx.x;
    if (idx >= size) return;
    const int64_t ix = idx % g.dims[0], iy = (idx / g.dims[0]) % g.dims[1], iz = idx / (g.dims[0] * g.dims[1]);
    const int64_t ii[3] = {ix, iy, iz};
    // Box corner min + i*h (opp_direct_hop_seq.cpp:156-162) and centroid, clamped to the box's
    // upper bound (getCentroidOfBox, ASSIGN_CENTROID_TO_DIM of opp_lib/include/opp_defs.h:121-127).
    double corner[3], q[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        corner[d] = __dadd_rn(g.min[d], __dmul_rn((double)ii[d], g.h));
        q[d] = (__dadd_rn(corner[d], g.h) <= g.max[d]) ? __dadd_rn(corner[d], __dmul_rn(g.h, 0.5))
                                                       : __dmul_rn(__dadd_rn(corner[d], g.max[d]), 0.5);
    }
    int32_t cid = first_cell(cs, g, offsets, list, q);
    // Not found: nudge the centroid by h/100 along x, then y, then z (cumulative, :172-183).
    const double nudge = __ddiv_rn(g.h, 100.0);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        if (cid != kRemoved) break;
        q[d] = __dadd_rn(q[d], nudge);
        cid = first_cell(cs, g, offsets, list, q);
    }
    if (cid == kRemoved) {
        // Step 3 (:214-246): the lowest cell holding one of the box's 8 corners, each corner
        // clamped to the upper bound (GET_VERT, opp_defs.h:115).
        for (int k = 0; k < 8; k++) {
            double v[3];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const double t = ((k >> d) & 1) ? __dadd_rn(corner[d], g.h) : corner[d];
                v[d] = (t > g.max[d]) ? g.max[d] : t;
            }
            const int32_t c = first_cell(cs, g, offsets, list, v);
            if (c < cid) cid = c;
        }
    }
    map[idx] = cid;
}

// The (cell, box) pair counter of a build: fixed device scratch, so that sizing the
// workspace needs no caller memory.  Calls on one device must not overlap.
__device__ unsigned long long g_dh_pairs;

}  // namespace
}  // namespace oppb

extern "C" int oppb_dh_bounding_box(const double* n_pos, int32_t n_nodes, const double expansion[3],
                                    double min_out[3], double max_out[3]) {
    if (!n_pos || !expansion || !min_out || !max_out || n_nodes <= 0) return OPPB_ERR_ARG;
    // BoundingBox(n_pos, 3, expansion) (opp_lib/include/opp_direct_hop_core.h:70-120): the
    // running max starts at MIN_REAL = DBL_MIN, and the x/y widening reads the expansion's
    // x for both minima and its y for both maxima, as written there.
    double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, mx[3] = {DBL_MIN, DBL_MIN, DBL_MIN};
    for (int32_t i = 0; i < n_nodes; i++)
        for (int d = 0; d < 3; d++) {
            const double v = n_pos[3 * (int64_t)i + d];
            mn[d] = (mn[d] < v) ? mn[d] : v;  // std::min(v, mn)
            mx[d] = (v < mx[d]) ? mx[d] : v;  // std::max(v, mx)
        }
    mn[0] -= (expansion[0] + oppb::kBoundOffset);
    mn[1] -= (expansion[0] + oppb::kBoundOffset);
    mx[0] += (expansion[1] - oppb::kBoundOffset);
    mx[1] += (expansion[1] - oppb::kBoundOffset);
    mn[2] -= (expansion[2] + oppb::kBoundOffset);
    mx[2] += (expansion[2] - oppb::kBoundOffset);
    for (int d = 0; d < 3; d++) {
        min_out[d] = mn[d];
        max_out[d] = mx[d];
    }
    return OPPB_OK;
}

extern "C" int oppb_dh_grid_from_box(const double min[3], const double max[3], double spacing, oppb_dh_grid* g) {
    if (!min || !max || !g || !(spacing > 0.0) || !std::isfinite(spacing)) return OPPB_ERR_ARG;
    // CellMapper::init_host (:317-380): boxes per axis = 1 + the count of the loop
    // `for (v = min; v < max; v += h)`, in floating point as there.
    int64_t dims[3];
    for (int d = 0; d < 3; d++) {
        if (!std::isfinite(min[d]) || !std::isfinite(max[d])) return OPPB_ERR_ARG;
        int64_t a = 0;
        for (double v = min[d]; v < max[d]; v += spacing)
            if (++a > oppb::kMaxLoop) return OPPB_ERR_ARG;
        dims[d] = a + 1;
    }
    const double size = (double)dims[0] * (double)dims[1] * (double)dims[2];
    if (size > 2147483646.0) return OPPB_ERR_ARG;
    for (int d = 0; d < 3; d++) {
        g->min[d] = min[d];
        g->max[d] = max[d];
        g->dims[d] = dims[d];
    }
    g->spacing = spacing;
    g->inv_spacing = 1.0 / spacing;
    g->size = dims[0] * dims[1] * dims[2];
    return OPPB_OK;
}

extern "C" int oppb_dh_grid_init(const double* n_pos, int32_t n_nodes, double spacing, const double expansion[3],
                                 oppb_dh_grid* g) {
    double mn[3], mx[3];
    const int rc = oppb_dh_bounding_box(n_pos, n_nodes, expansion, mn, mx);
    return rc ? rc : oppb_dh_grid_from_box(mn, mx, spacing, g);
}

namespace oppb {
namespace {

// The build common to both meshes: bin the cells, then query every box.
template <class Cells>
int build_map(const Cells& cs, int32_t n_cells, oppb_dh_grid* grid, void* workspace, size_t ws_bytes,
              size_t* ws_needed, void* stream) {
    if (grid->size <= 0 || grid->size > 2147483646 || !(grid->spacing > 0.0) ||
        grid->size != grid->dims[0] * grid->dims[1] * grid->dims[2])
        return OPPB_ERR_ARG;
    const GridArgs g{{grid->min[0], grid->min[1], grid->min[2]},
                     {grid->max[0], grid->max[1], grid->max[2]},
                     grid->spacing,
                     {grid->dims[0], grid->dims[1], grid->dims[2]}};
    cudaStream_t s = as_stream(stream);
    unsigned long long* d_pairs = nullptr;
    if (cudaGetSymbolAddress(reinterpret_cast<void**>(&d_pairs), g_dh_pairs) != cudaSuccess) return OPPB_ERR_LAUNCH;
    const int cell_grid = ceil_div(n_cells, kDhBlock);
    if (cudaMemsetAsync(d_pairs, 0, sizeof(unsigned long long), s) != cudaSuccess) return OPPB_ERR_LAUNCH;
    dh_bin_kernel<0><<<cell_grid, kDhBlock, 0, s>>>(cs, g, d_pairs, nullptr, nullptr, nullptr);
    count_launches(1);
    unsigned long long pairs = 0;
    if (cudaMemcpyAsync(&pairs, d_pairs, sizeof pairs, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return OPPB_ERR_LAUNCH;
    if (pairs > 2147483647ull) return OPPB_ERR_ARG;  // grid far finer than the cells
    const int64_t n = grid->size;
    const size_t need = align256(sizeof(int) * (size_t)(n + 1)) + align256(sizeof(int) * (size_t)n) +
                        align256(sizeof(int) * (size_t)(pairs ? pairs : 1)) +
                        align256(sizeof(int) * scan_scratch_ints(n + 1));
    if (ws_needed) *ws_needed = need;
    if (!workspace || ws_bytes < need || !aligned(workspace, 256)) return OPPB_ERR_WORKSPACE;
    char* w = static_cast<char*>(workspace);
    int* offsets = reinterpret_cast<int*>(w);
    w += align256(sizeof(int) * (size_t)(n + 1));
    int* cursor = reinterpret_cast<int*>(w);
    w += align256(sizeof(int) * (size_t)n);
    int* list = reinterpret_cast<int*>(w);
    w += align256(sizeof(int) * (size_t)(pairs ? pairs : 1));
    int* scratch = reinterpret_cast<int*>(w);
    if (cudaMemsetAsync(offsets, 0, sizeof(int) * (size_t)(n + 1), s) != cudaSuccess) return OPPB_ERR_LAUNCH;
    dh_bin_kernel<1><<<cell_grid, kDhBlock, 0, s>>>(cs, g, nullptr, offsets, nullptr, nullptr);
    count_launches(1);
    device_exclusive_scan(offsets, offsets, n + 1, scratch, s);  // offsets[n] = pairs
    if (cudaMemcpyAsync(cursor, offsets, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return OPPB_ERR_LAUNCH;
    dh_bin_kernel<2><<<cell_grid, kDhBlock, 0, s>>>(cs, g, nullptr, nullptr, cursor, list);
    dh_query_kernel<<<ceil_div(n, kDhBlock), kDhBlock, 0, s>>>(cs, g, offsets, list, grid->map, n);
    count_launches(2);
    return launch_status();
}

}  // namespace
}  // namespace oppb

extern "C" int oppb_dh_build(const oppb_tet_mesh* mesh, const double* n_pos, oppb_dh_grid* grid, void* workspace,
                             size_t ws_bytes, size_t* ws_needed, void* stream) {
    using namespace oppb;
    if (!mesh || !n_pos || !grid || !grid->map || mesh->n_cells <= 0 || mesh->n_nodes <= 0) return OPPB_ERR_ARG;
    if (!mesh->det || !mesh->nav || !mesh->c2n || !aligned(mesh->det, 32) || !aligned(mesh->nav, 32) ||
        !aligned(mesh->c2n, 16))
        return OPPB_ERR_ARG;
    return build_map(TetCells{*mesh, n_pos}, mesh->n_cells, grid, workspace, ws_bytes, ws_needed, stream);
}

extern "C" int oppb_dh_bounding_box_2d(const double* pos, int32_t n, const double expansion[3], double min_out[3],
                                       double max_out[3]) {
    if (!pos || !expansion || !min_out || !max_out || n <= 0) return OPPB_ERR_ARG;
    // BoundingBox(pos, 2, expansion) (opp_lib/include/opp_direct_hop_core.h:70-120): z stays
    // 0; the x/y widening reads the expansion's x for both minima and its y for both maxima.
    double mn[2] = {DBL_MAX, DBL_MAX}, mx[2] = {DBL_MIN, DBL_MIN};
    for (int32_t i = 0; i < n; i++)
        for (int d = 0; d < 2; d++) {
            const double v = pos[2 * (int64_t)i + d];
            mn[d] = (mn[d] < v) ? mn[d] : v;  // std::min(v, mn)
            mx[d] = (v < mx[d]) ? mx[d] : v;  // std::max(v, mx)
        }
    mn[0] -= (expansion[0] + oppb::kBoundOffset);
    mn[1] -= (expansion[0] + oppb::kBoundOffset);
    mx[0] += (expansion[1] - oppb::kBoundOffset);
    mx[1] += (expansion[1] - oppb::kBoundOffset);
    min_out[0] = mn[0], min_out[1] = mn[1], min_out[2] = 0.0;
    max_out[0] = mx[0], max_out[1] = mx[1], max_out[2] = 0.0;
    return OPPB_OK;
}

extern "C" int oppb_dh_grid_init_2d(const double* pos, int32_t n, double spacing, const double expansion[3],
                                    oppb_dh_grid* g) {
    double mn[3], mx[3];
    const int rc = oppb_dh_bounding_box_2d(pos, n, expansion, mn, mx);
    return rc ? rc : oppb_dh_grid_from_box(mn, mx, spacing, g);
}

extern "C" int oppb_dh_build_quad(const double* cells, int32_t n_cells, double cell_width, oppb_dh_grid* grid,
                                  void* workspace, size_t ws_bytes, size_t* ws_needed, void* stream) {
    using namespace oppb;
    if (!cells || !aligned(cells, 32) || n_cells <= 0 || !grid || !grid->map || !(cell_width > 0.0) ||
        grid->dims[2] != 1)
        return OPPB_ERR_ARG;
    return build_map(QuadCells{cells, n_cells, cell_width}, n_cells, grid, workspace, ws_bytes, ws_needed, stream);
}
