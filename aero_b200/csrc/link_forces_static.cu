// link_forces_static.cu -- momentum-exchange forces without any allocation.
//
// Some callers cannot call cudaMalloc at all: real-time loops whose device
// memory is fixed up front, and host frameworks that hand out only the
// buffers they own and do not let a library allocate.  For them this
// file provides aero_link_forces_static(): the same force evaluation the
// engine performs every step (per-link contributions followed by a fixed-
// order FP64 reduction), on populations the caller already has on the GPU,
// with the per-link scratch taken from a file-scope __device__ array instead
// of a workspace.
//
// The scratch array is shared by every call on a device and keeps the last
// call's contents; each call overwrites the entries it uses before reading
// them, so nothing needs clearing, but two calls that overlap on the GPU
// (different streams, no ordering between them) race on it.
//
// Every call made outside stream capture looks the array's address up with
// cudaGetSymbolAddress, with the call's device current, and refreshes a
// per-device cache (so a device reset, which reloads the module, cannot
// leave a stale address behind).  A call made while its stream is being
// captured uses the cached address, since the lookup may load the module;
// the first call on a device must therefore come before any stream capture.
//
// Link rows with a direction outside 1..Q-1 or a cell outside the grid
// (which the reference's fancy indexing rejects with IndexError,
// forces.py:27-33) make the call write NaN to every output value, so a
// malformed list cannot pass for a plausible force.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/aero_b200.h"
#include "lbm_dispatch.h"

namespace {

constexpr int kStaticMaxLinks = 32768;  // 32768 links x 16 doubles = 4 MiB per GPU
constexpr int kSlot = 16;               // 12 force values, bin index, padding
constexpr int kMaxDevices = 64;

// Device-resident scratch: per-link contributions of the last call.  In host
// code the name is only a stand-in; kernels get its address from
// cudaGetSymbolAddress (see scratch_ptr).
static __device__ __align__(256) double g_link_scratch[kStaticMaxLinks * kSlot];

__constant__ int c_ex[2][19] = {
    {0, 1, 0, -1, 0, 1, -1, -1, 1},
    {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0}};
__constant__ int c_ey[2][19] = {
    {0, 0, 1, 0, -1, 1, 1, -1, -1},
    {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1}};
__constant__ int c_ez[2][19] = {
    {0, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1}};
__constant__ int c_opp[2][19] = {
    {0, 3, 4, 1, 2, 7, 8, 5, 6},
    {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15}};
__constant__ double c_w[2][19] = {
    {4.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36},
    {1.0 / 3, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 36, 1.0 / 36, 1.0 / 36,
     1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36}};

struct Geometry {
  int dims, Q, nx, ny, nz;
  long long ncells;
  double cx, cy, cz;
};

// One thread per link: f_pre[i] + f_post[opp i], its split into the part of
// feq(f_pre moments) and the rest, and its moment about the centre
// (forces.py:15-127, forces3d.py:8-131).
__global__ void k_link_contrib(const double *__restrict__ f_pre, const double *__restrict__ f_post,
                               const int *__restrict__ links, long long n_links, Geometry g, double *scratch) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_links) return;
  const int t = g.dims == 3 ? 1 : 0, lw = g.dims == 3 ? 4 : 3;
  const int *lk = links + k * lw;
  const int i = lk[0], z = g.dims == 3 ? lk[1] : 0, y = lk[lw - 2], x = lk[lw - 1];
  double *out = scratch + k * kSlot;
  if (i < 1 || i >= g.Q || x < 0 || x >= g.nx || y < 0 || y >= g.ny || z < 0 || z >= g.nz) {
    for (int j = 0; j < 12; j++) out[j] = 0.0;
    out[12] = -1.0;  // marks the row invalid: the reduction then writes NaN
    return;
  }
  const long long c = ((long long)z * g.ny + y) * g.nx + x;
  const int o = c_opp[t][i];
  double rho = 0, jx = 0, jy = 0, jz = 0;
  for (int a = 0; a < g.Q; a++) {
    const double v = f_pre[a * g.ncells + c];
    rho += v;
    jx += c_ex[t][a] * v;
    jy += c_ey[t][a] * v;
    jz += c_ez[t][a] * v;
  }
  const double inv = rho > 0.0 ? 1.0 / rho : 0.0;
  const double ux = jx * inv, uy = jy * inv, uz = jz * inv, usq = ux * ux + uy * uy + uz * uz;
  const double ex = c_ex[t][i], ey = c_ey[t][i], ez = c_ez[t][i];
  const double eu = ex * ux + ey * uy + ez * uz;
  const double feq_out = c_w[t][i] * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * usq);
  const double feq_in = c_w[t][o] * rho * (1.0 - 3.0 * eu + 4.5 * eu * eu - 1.5 * usq);
  const double fo = f_pre[i * g.ncells + c], fin = f_post[o * g.ncells + c];
  const double mom = fo + fin, mp = feq_out + feq_in, mv = (fo - feq_out) + (fin - feq_in);
  const double rx = x - g.cx, ry = y - g.cy, rz = z - g.cz;
  const double dfx = ex * mom, dfy = ey * mom, dfz = ez * mom;
  out[0] = dfx;
  out[1] = dfy;
  out[2] = dfz;
  out[3] = ex * mp;
  out[4] = ey * mp;
  out[5] = ez * mp;
  out[6] = ex * mv;
  out[7] = ey * mv;
  out[8] = ez * mv;
  out[9] = ry * dfz - rz * dfy;
  out[10] = rz * dfx - rx * dfz;
  out[11] = rx * dfy - ry * dfx;
  out[12] = g.dims == 3 ? z : y;
}

// One block: fixed-order sums of the contributions (deterministic); a row
// with bin -1 (invalid direction or coordinate) makes every output NaN.
constexpr int kReduceBlock = 256;
__global__ void __launch_bounds__(kReduceBlock) k_link_reduce(const double *scratch, long long n_links,
                                                              double *out12) {
  __shared__ double sm[12][kReduceBlock / 32];
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  double a[12];
  for (int j = 0; j < 12; j++) a[j] = 0.0;
  int bad = 0;
  for (long long k = t; k < n_links; k += kReduceBlock) {
    for (int j = 0; j < 12; j++) a[j] += scratch[k * kSlot + j];
    bad |= scratch[k * kSlot + 12] < 0.0 ? 1 : 0;
  }
  for (int j = 0; j < 12; j++) {
    double v = a[j];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) sm[j][wid] = v;
  }
  bad = __syncthreads_or(bad);
  if (t < 12) {
    double v = 0.0;
    for (int w = 0; w < kReduceBlock / 32; w++) v += sm[t][w];
    out12[t] = bad ? __longlong_as_double(0x7ff8000000000000LL) : v;
  }
}

// Block b: the force profile of row (2D) / plane (3D) b, i.e. the sum of
// (dfx, dfy, dfz) over the links whose bin is b.  Each thread takes a fixed
// stride of the link list and the block reduces in a fixed order, so the
// result is deterministic; the blocks run in parallel, one pass over the
// link list each, instead of one thread scanning every link per bin.  Any
// invalid row makes the whole profile NaN, as it makes the totals.
__global__ void __launch_bounds__(kReduceBlock) k_link_profile(const double *scratch, long long n_links,
                                                               double *profile) {
  __shared__ double sm[3][kReduceBlock / 32];
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const double b = (double)blockIdx.x;
  double p0 = 0.0, p1 = 0.0, p2 = 0.0;
  int bad = 0;
  for (long long k = t; k < n_links; k += kReduceBlock) {
    const double bin = scratch[k * kSlot + 12];
    bad |= bin < 0.0 ? 1 : 0;
    if (bin != b) continue;
    p0 += scratch[k * kSlot + 0];
    p1 += scratch[k * kSlot + 1];
    p2 += scratch[k * kSlot + 2];
  }
  for (int off = 16; off > 0; off >>= 1) {
    p0 += __shfl_down_sync(0xffffffffu, p0, off);
    p1 += __shfl_down_sync(0xffffffffu, p1, off);
    p2 += __shfl_down_sync(0xffffffffu, p2, off);
  }
  if (lane == 0) {
    sm[0][wid] = p0;
    sm[1][wid] = p1;
    sm[2][wid] = p2;
  }
  bad = __syncthreads_or(bad);
  if (t < 3) {
    double v = 0.0;
    for (int w = 0; w < kReduceBlock / 32; w++) v += sm[t][w];
    profile[3 * blockIdx.x + t] = bad ? __longlong_as_double(0x7ff8000000000000LL) : v;
  }
}

std::mutex g_mu;
double *g_addr[kMaxDevices] = {nullptr};

// Device address of g_link_scratch on the current device.  Outside stream
// capture it is looked up on every call (with that device current) and the
// per-device cache refreshed; during capture the cached address is used,
// and a device never looked up before capture is an error.
cudaError_t scratch_ptr(cudaStream_t st, double **ptr, int *device) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  *device = dev;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(st, &cap);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_mu);
  if (cap == cudaStreamCaptureStatusNone) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_link_scratch);
    if (e != cudaSuccess) return e;
    g_addr[dev] = static_cast<double *>(p);
  } else if (!g_addr[dev]) {
    return cudaErrorStreamCaptureUnsupported;
  }
  *ptr = g_addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" {

int aero_link_forces_static(int32_t dims, int32_t nx, int32_t ny, int32_t nz, const double *f_pre,
                            const double *f_post, const int32_t *links, int64_t n_links, const double *center,
                            double *out, double *profile, void *stream) {
  if ((dims != 2 && dims != 3) || nx < 1 || ny < 1 || nz < 1 || (dims == 2 && nz != 1) || !f_pre || !f_post ||
      !out || !center || n_links < 0 || (n_links > 0 && !links)) {
    return aero::set_error(AERO_ERR_INVALID, "aero_link_forces_static: invalid argument");
  }
  if (n_links > kStaticMaxLinks) {
    char msg[160];
    snprintf(msg, sizeof(msg), "aero_link_forces_static: %lld links exceed the fixed capacity of %d links",
             (long long)n_links, kStaticMaxLinks);
    return aero::set_error(AERO_ERR_CAPACITY, msg);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double *scratch = nullptr;
  int dev = -1;
  cudaError_t e = scratch_ptr(st, &scratch, &dev);
  if (e == cudaErrorStreamCaptureUnsupported) {
    return aero::set_error(AERO_ERR_STATE,
                           "aero_link_forces_static: the first call on a device must come before stream capture");
  }
  if (e != cudaSuccess) {
    return aero::set_error(AERO_ERR_CUDA, cudaGetErrorString(e));
  }
  Geometry g{dims, dims == 2 ? 9 : 19, nx, ny, nz, (long long)nx * ny * nz, center[0], center[1], center[2]};
  if (n_links > 0) {
    const int b = 128;
    k_link_contrib<<<(unsigned)((n_links + b - 1) / b), b, 0, st>>>(f_pre, f_post, links, n_links, g, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return aero::set_error(AERO_ERR_CUDA, cudaGetErrorString(e));
  }
  k_link_reduce<<<1, kReduceBlock, 0, st>>>(scratch, n_links, out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return aero::set_error(AERO_ERR_CUDA, cudaGetErrorString(e));
  if (profile) {
    k_link_profile<<<(unsigned)(dims == 3 ? nz : ny), kReduceBlock, 0, st>>>(scratch, n_links, profile);
    e = cudaGetLastError();
    if (e != cudaSuccess) return aero::set_error(AERO_ERR_CUDA, cudaGetErrorString(e));
  }
  return AERO_OK;
}

}  // extern "C"
