// links_device.cu -- surface link list built on the device.
//
// Device counterpart of build_surface_links / build_surface_links_3d
// (aero/lbm/boundary.py:232-280, aero/lbm/boundary3d.py:279-329): a link
// (i, [z,] y, x) joins a fluid cell to the solid cell in direction e_i, the
// neighbour index CLIPPED to the grid; the list is direction-major and in C
// order of the cells within a direction; q = clip(float32(phi[cell]), 1e-4, 1)
// when phi is given, else 0.5.  Links only lie in the solid's bounding box
// grown by one cell (a clipped neighbour is at most one cell away on every
// axis), and within one direction the C order of that box's cells is the
// grid's, so a first pass finds the box and the rest run on it alone.  The
// box's list splits into units (one direction, 1024 consecutive box cells)
// in list order; each CTA takes a run of units.  Three passes follow: count
// every CTA's links, scan the counts, write every CTA's links from its offset
// with ranks taken in cell order (warp ballots).  The result is the
// reference's list entry for entry.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>

#include "../../include/aero_b200.h"
#include "lbm_dispatch.h"
#include "lbm_lattice.cuh"

using namespace aero;

namespace {

constexpr int kLinkThreads = 256;
constexpr int kUnitCells = 1024;      // cells of one unit: one direction, consecutive cells
constexpr int kScanThreads = 1024;
constexpr int kTargetGroups = 148 * 16;  // CTAs of the count and write passes on large grids

constexpr int kBoxInts = 8;  // scratch head: the solid's bounding box, 32 bytes

// The list is the units in order (direction 1..Q-1, then box cells in C
// order); CTA b of the count and write passes takes `group` consecutive units.
struct LinkGrid {
  int dims, nx, ny, nz, Q;
  int ox, oy, oz, bnx, bny, bnz;  // the box: origin and extent
  uint32_t bcells, units_per_dir;
  int64_t units, group, ngroups;
};

// Direction vectors of a lattice as a table the kernels index at run time.
struct DirTable {
  int8_t e[19][3];
};

template <class L>
constexpr DirTable dir_table() {
  DirTable t{};
  for (int i = 0; i < L::Q; i++) {
    t.e[i][0] = (int8_t)L::ex[i];
    t.e[i][1] = (int8_t)L::ey[i];
    t.e[i][2] = (int8_t)L::ez[i];
  }
  return t;
}

__constant__ DirTable c_dirs[2] = {dir_table<D2Q9>(), dir_table<D3Q19>()};

struct Cell {
  uint32_t x, y, z;
};

// Grid coordinates of box cell b.
__device__ __forceinline__ Cell box_cell(const LinkGrid &g, uint32_t b) {
  const uint32_t r = b / (uint32_t)g.bnx;
  return {b - r * (uint32_t)g.bnx + g.ox, r % (uint32_t)g.bny + g.oy, r / (uint32_t)g.bny + g.oz};
}

__device__ __forceinline__ uint32_t cell_index(const LinkGrid &g, Cell p) {
  return (p.z * (uint32_t)g.ny + p.y) * (uint32_t)g.nx + p.x;
}

// Whether direction i of box cell b (grid cell p, index c) is a link: fluid
// cell, solid clipped neighbour.
__device__ __forceinline__ bool is_link(const LinkGrid &g, const uint8_t *__restrict__ solid, int i, uint32_t b,
                                        Cell p, uint32_t c) {
  if (b >= g.bcells || solid[c]) return false;
  const int8_t *e = c_dirs[g.dims - 2].e[i];
  const int xn = min(max((int)p.x + e[0], 0), g.nx - 1);
  const int yn = min(max((int)p.y + e[1], 0), g.ny - 1);
  const int zn = min(max((int)p.z + e[2], 0), g.nz - 1);
  return solid[((uint32_t)zn * (uint32_t)g.ny + (uint32_t)yn) * (uint32_t)g.nx + (uint32_t)xn] != 0;
}

__device__ __forceinline__ int block_sum(int v, int *red) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  __syncthreads();  // red is free again
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  int t = 0;
#pragma unroll
  for (int w = 0; w < kLinkThreads / 32; w++) t += red[w];
  return t;
}

// Pass 0: the solid cells' bounding box, as atomic maxima of (x, -x, y, -y,
// z, -z) into box[0..6), which start at 0x80808080 (below any -coordinate):
// a row per CTA iteration, so only the row index is divided.
__global__ void __launch_bounds__(kLinkThreads) k_solid_bbox(const uint8_t *__restrict__ solid, int nx, int ny,
                                                              int64_t nrows, int *__restrict__ box) {
  int m[6];
#pragma unroll
  for (int k = 0; k < 6; k++) m[k] = INT_MIN;
  for (int64_t r = blockIdx.x; r < nrows; r += gridDim.x) {
    const uint8_t *row = solid + r * nx;
    const int y = (int)(r % ny), z = (int)(r / ny);
    for (int x = threadIdx.x; x < nx; x += kLinkThreads) {
      if (row[x]) {
        m[0] = max(m[0], x);
        m[1] = max(m[1], -x);
        m[2] = max(m[2], y);
        m[3] = max(m[3], -y);
        m[4] = max(m[4], z);
        m[5] = max(m[5], -z);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 6; k++) {
    int v = m[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = max(v, __shfl_down_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0 && v != INT_MIN) atomicMax(box + k, v);
  }
}

// Pass 1: the number of links in CTA b's units.
__global__ void __launch_bounds__(kLinkThreads) k_link_count(LinkGrid g, const uint8_t *__restrict__ solid,
                                                              int64_t *__restrict__ counts) {
  __shared__ int red[kLinkThreads / 32];
  const int64_t u0 = (int64_t)blockIdx.x * g.group;
  const int64_t u1 = min(u0 + g.group, g.units);
  int64_t total = 0;
  for (int64_t u = u0; u < u1; u++) {
    const int i = 1 + (int)(u / g.units_per_dir);
    const uint32_t c0 = (uint32_t)(u % g.units_per_dir) * kUnitCells;
    int n = 0;
    for (int k = threadIdx.x; k < kUnitCells; k += kLinkThreads) {
      const uint32_t b = c0 + k;
      const Cell p = box_cell(g, b);
      n += is_link(g, solid, i, b, p, cell_index(g, p));
    }
    total += block_sum(n, red);
  }
  if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

// Pass 2: exclusive prefix of the CTA counts, in place, in tiles of
// kScanThreads; counts[n] receives the number of links.  One CTA.
__global__ void __launch_bounds__(kScanThreads) k_link_scan(int64_t *__restrict__ counts, int64_t n) {
  __shared__ int64_t wsum[kScanThreads / 32];
  __shared__ int64_t carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t t0 = 0; t0 < n; t0 += kScanThreads) {
    const int64_t k = t0 + threadIdx.x;
    const int64_t v = k < n ? counts[k] : 0;
    int64_t incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int64_t o = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += o;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      int64_t w = wsum[lane];
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int64_t o = __shfl_up_sync(0xffffffffu, w, off);
        if (lane >= off) w += o;
      }
      wsum[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const int64_t before = carry + (warp ? wsum[warp - 1] : 0);
    if (k < n) counts[k] = before + incl - v;
    __syncthreads();
    if (threadIdx.x == 0) carry += wsum[kScanThreads / 32 - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) counts[n] = carry;
}

// Pass 3: CTA b writes the links of its units from its offset, in list
// order: warp ballots rank the links of each 256 cells, a running base
// carries the rank across them.
__global__ void __launch_bounds__(kLinkThreads) k_link_write(LinkGrid g, const uint8_t *__restrict__ solid,
                                                              const double *__restrict__ phi,
                                                              const int64_t *__restrict__ offsets,
                                                              int32_t *__restrict__ links, float *__restrict__ q) {
  __shared__ int wcount[kLinkThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lw = g.dims + 1;
  int64_t base = offsets[blockIdx.x];
  const int64_t u0 = (int64_t)blockIdx.x * g.group;
  const int64_t u1 = min(u0 + g.group, g.units);
  for (int64_t u = u0; u < u1; u++) {
    const int i = 1 + (int)(u / g.units_per_dir);
    const uint32_t c0 = (uint32_t)(u % g.units_per_dir) * kUnitCells;
    for (int k = 0; k < kUnitCells; k += kLinkThreads) {
      const uint32_t b = c0 + k + threadIdx.x;
      const Cell p = box_cell(g, b);
      const uint32_t c = cell_index(g, p);
      const bool hit = is_link(g, solid, i, b, p, c);
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      if (lane == 0) wcount[warp] = __popc(m);
      __syncthreads();
      int64_t before = base, add = 0;
#pragma unroll
      for (int w = 0; w < kLinkThreads / 32; w++) {
        const int n = wcount[w];
        before += w < warp ? n : 0;
        add += n;
      }
      if (hit) {
        const int64_t at = before + __popc(m & ((1u << lane) - 1u));
        int32_t *row = links + at * lw;
        row[0] = i;
        if (g.dims == 3) {
          row[1] = (int32_t)p.z;
          row[2] = (int32_t)p.y;
          row[3] = (int32_t)p.x;
        } else {
          row[1] = (int32_t)p.y;
          row[2] = (int32_t)p.x;
        }
        float qv = 0.5f;
        if (phi) {
          qv = (float)phi[c];  // round to nearest, as numpy's astype(float32)
          qv = qv < 1e-4f ? 1e-4f : (qv > 1.0f ? 1.0f : qv);  // NaN stays NaN, as np.clip
        }
        q[at] = qv;
      }
      base += add;
      __syncthreads();  // wcount is rewritten by the next 256 cells
    }
  }
}

int check_grid(int32_t dims, int32_t nx, int32_t ny, int32_t nz, LinkGrid *g) {
  if ((dims != 2 && dims != 3) || nx < 1 || ny < 1 || nz < 1 || (dims == 2 && nz != 1))
    return set_error(AERO_ERR_INVALID, "bad grid for the link build");
  const int64_t cells = (int64_t)nx * ny * nz;
  if (cells > 0x7fffffffLL - kUnitCells) return set_error(AERO_ERR_UNSUPPORTED, "grid too large for the link build");
  g->dims = dims;
  g->nx = nx;
  g->ny = ny;
  g->nz = nz;
  g->Q = dims == 2 ? 9 : 19;
  return AERO_OK;
}

// Units and CTA groups of the box [lo, hi] (inclusive, grid coordinates).
void set_box(LinkGrid *g, const int lo[3], const int hi[3]) {
  g->ox = lo[0];
  g->oy = lo[1];
  g->oz = lo[2];
  g->bnx = hi[0] - lo[0] + 1;
  g->bny = hi[1] - lo[1] + 1;
  g->bnz = hi[2] - lo[2] + 1;
  const int64_t cells = (int64_t)g->bnx * g->bny * g->bnz;
  g->bcells = (uint32_t)cells;
  g->units_per_dir = (uint32_t)((cells + kUnitCells - 1) / kUnitCells);
  g->units = (int64_t)(g->Q - 1) * g->units_per_dir;
  g->group = std::max<int64_t>(1, (g->units + kTargetGroups - 1) / kTargetGroups);
  g->ngroups = (g->units + g->group - 1) / g->group;
}

// Scratch for the largest box, the whole grid: never fewer CTA groups than a
// smaller box has (at most min(units, kTargetGroups)).
uint64_t scratch_bytes(const LinkGrid &g) {
  const int64_t units = (int64_t)(g.Q - 1) * (((int64_t)g.nx * g.ny * g.nz + kUnitCells - 1) / kUnitCells);
  return 4 * kBoxInts + 8 * ((uint64_t)std::min<int64_t>(units, kTargetGroups) + 1);
}

}  // namespace

extern "C" {

int aero_surface_links_scratch_size(int32_t dims, int32_t nx, int32_t ny, int32_t nz, uint64_t *bytes) {
  if (!bytes) return set_error(AERO_ERR_INVALID, "NULL argument");
  LinkGrid g;
  const int rc = check_grid(dims, nx, ny, nz, &g);
  if (rc != AERO_OK) return rc;
  *bytes = scratch_bytes(g);
  return AERO_OK;
}

int aero_surface_links_device(int32_t dims, int32_t nx, int32_t ny, int32_t nz, const uint8_t *solid,
                              const double *phi, void *scratch, uint64_t scratch_size, int32_t *links, float *q,
                              int64_t capacity, int64_t *n_links, void *stream) {
  if (!solid || !scratch || !n_links) return set_error(AERO_ERR_INVALID, "NULL argument");
  LinkGrid g;
  int rc = check_grid(dims, nx, ny, nz, &g);
  if (rc != AERO_OK) return rc;
  if (scratch_size < scratch_bytes(g)) return set_error(AERO_ERR_INVALID, "scratch smaller than aero_surface_links_scratch_size");
  if (reinterpret_cast<uintptr_t>(scratch) % 8) return set_error(AERO_ERR_INVALID, "scratch must be 8-byte aligned");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int *box = static_cast<int *>(scratch);
  int64_t *counts = reinterpret_cast<int64_t *>(box + kBoxInts);
  const int64_t nrows = (int64_t)ny * nz;
  cudaError_t e = cudaMemsetAsync(box, 0x80, 4 * kBoxInts, st);
  if (e != cudaSuccess) return set_error(AERO_ERR_CUDA, cudaGetErrorString(e));
  k_solid_bbox<<<(unsigned)std::min<int64_t>(nrows, 148 * 8), kLinkThreads, 0, st>>>(solid, nx, ny, nrows, box);
  int hb[kBoxInts];
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(hb, box, sizeof(hb), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_error(AERO_ERR_CUDA, cudaGetErrorString(e));
  *n_links = 0;
  if (hb[0] < 0) return AERO_OK;  // no solid cell: no links
  const int n_[3] = {nx, ny, nz};
  int lo[3], hi[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = std::max(-hb[2 * a + 1] - 1, 0);
    hi[a] = std::min(hb[2 * a] + 1, n_[a] - 1);
  }
  set_box(&g, lo, hi);
  const unsigned grid = (unsigned)g.ngroups;
  k_link_count<<<grid, kLinkThreads, 0, st>>>(g, solid, counts);
  k_link_scan<<<1, kScanThreads, 0, st>>>(counts, g.ngroups);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(AERO_ERR_CUDA, cudaGetErrorString(e));
  int64_t n = 0;
  e = cudaMemcpyAsync(&n, counts + g.ngroups, sizeof(n), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_error(AERO_ERR_CUDA, cudaGetErrorString(e));
  *n_links = n;
  if (n > capacity) return set_error(AERO_ERR_CAPACITY, "link output holds fewer entries than *n_links");
  if (n > 0) {
    if (!links || !q) return set_error(AERO_ERR_INVALID, "NULL output arrays");
    k_link_write<<<grid, kLinkThreads, 0, st>>>(g, solid, phi, counts, links, q);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(AERO_ERR_CUDA, cudaGetErrorString(e));
  }
  return AERO_OK;
}

}  // extern "C"
