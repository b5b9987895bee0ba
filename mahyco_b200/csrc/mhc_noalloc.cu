// mhc_noalloc.cu -- allocation-free variant of the CFL time-step reduction.
//
// Who needs it: a host code that owns all of its device memory -- a mesh
// framework with its own pooled allocator, a solver running inside a
// region where device allocation is forbidden (device-memory budget already
// handed out, real-time or certified loops), or any caller that cannot
// call cudaMalloc at that point.  Such a caller passes its own device
// buffers (inputs and the output) and the reduction keeps its intermediate
// per-block minima in a fixed array that lives in the library itself.
//
// The array is a file-scope __device__ object: every GPU that loads the
// library holds its MHC_NOALLOC_SCRATCH_BYTES until the process exits, and
// every call on a device uses the same array.  Calls that overlap on the
// GPU (two streams at once) therefore race on it and must be serialised by
// the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/mahyco_b200.h"
#include "mhc_device.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = MHC_NOALLOC_MAX_CELLS / kThreads;
static_assert(kMaxBlocks * 8 == MHC_NOALLOC_SCRATCH_BYTES, "scratch size");

// per-block partial minima of l / (c + vmax); fully rewritten by every call
__device__ __align__(256) double g_noalloc_scratch[kMaxBlocks];

// host-side device addresses of g_noalloc_scratch, one per device, looked
// up once; they do not survive a cudaDeviceReset (the module is loaded
// again at another address), so a process that resets a device must not
// call this entry point on it afterwards
constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;
thread_local std::string g_noalloc_err;

using mhc::Mesh;

// block minimum of l / (c + vmax) over the cells of one block
// (MahycoModule::computeDeltaT, MahycoModule.cc:1766-1790); the node speed
// vmax enters only when the remap's is-euler-scheme is Full
// (MahycoModule.cc:1771), otherwise it is 0
__global__ void __launch_bounds__(kThreads)
k_cfl_partial(Mesh M, const double* l, const double* c, const double* vx, const double* vy,
              const double* vz, int euler_full, double* partial) {
  long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double dx = 1.7976931348623157e308;
  if (cell < M.ncell) {
    int i, j, k;
    mhc::cell_ijk(M, cell, i, j, k);
    double vmax = 0.;
    for (int n = 0; euler_full && n < (M.dim == 3 ? 8 : 4); ++n) {
      int a, b, d;
      mhc::local_node_offset(n, a, b, d);
      long long nn = mhc::node_id(M, i + a, j + b, k + d);
      double x = vx[nn], y = vy[nn], z = vz[nn];
      vmax = mhc::amax(sqrt(x * x + y * y + z * z), vmax);
    }
    dx = l[cell] / (c[cell] + vmax);
    if (!(dx >= 0.)) dx = -1.;  // NaN or negative: reported by the final pass
  }
  for (int o = 16; o > 0; o >>= 1) dx = fmin(dx, __shfl_xor_sync(0xffffffffu, dx, o));
  __shared__ double red[kThreads / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dx;
  __syncthreads();
  if (threadIdx.x < 32) {
    dx = threadIdx.x < kThreads / 32 ? red[threadIdx.x] : 1.7976931348623157e308;
    for (int o = 16; o > 0; o >>= 1) dx = fmin(dx, __shfl_xor_sync(0xffffffffu, dx, o));
    if (threadIdx.x == 0) partial[blockIdx.x] = dx;
  }
}

// minimum of the partials, then the growth, maximum and minimum bounds
__global__ void __launch_bounds__(kThreads)
k_cfl_final(const double* partial, int nblocks, double cfl, double old_dt, double dt_max, double dt_min,
            double* out) {
  double m = 1.7976931348623157e308;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) m = fmin(m, partial[b]);
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double red[kThreads / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    m = red[0];
    for (int w = 1; w < kThreads / 32; ++w) m = fmin(m, red[w]);
    double new_dt;
    if (m < 0.) {
      new_dt = -1.;  // a cell produced NaN or a negative l / (c + vmax)
    } else {
      new_dt = cfl * m;
      new_dt = mhc::amin(new_dt, 1.05 * old_dt);
      new_dt = mhc::amin(new_dt, dt_max);
      if (new_dt < dt_min) new_dt = -2.;
    }
    out[0] = new_dt;
  }
}

// device address of the scratch array on the current device; the first
// call on each device looks it up (not allowed during stream capture)
int scratch_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { g_noalloc_err = cudaGetErrorString(e); return MHC_ERR_CUDA; }
  if (dev < 0 || dev >= kMaxDevices) { g_noalloc_err = "device index out of range"; return MHC_ERR_ARG; }
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      g_noalloc_err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return MHC_ERR_CUDA;
    }
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<double*>(g_scratch_addr[dev]);
  return MHC_OK;
}

}  // namespace

const char* mhc_noalloc_last_error(void) { return g_noalloc_err.c_str(); }

int mhc_cfl_delta_t_noalloc(int dim, int nx, int ny, int nz, const double* char_length,
                            const double* sound_speed, const double* vx, const double* vy,
                            const double* vz, int euler_full, double cfl, double old_deltat,
                            double deltat_max, double deltat_min, double* deltat_out, void* stream) {
  if ((dim != 2 && dim != 3) || nx < 1 || ny < 1 || (dim == 3 && nz < 1)) {
    g_noalloc_err = "bad mesh dimensions";
    return MHC_ERR_ARG;
  }
  if (!char_length || !sound_speed || !deltat_out || (euler_full && (!vx || !vy || !vz))) {
    g_noalloc_err = "null buffer";
    return MHC_ERR_ARG;
  }
  Mesh M;
  M.dim = dim;
  M.ncx = nx; M.ncy = ny; M.ncz = dim == 3 ? nz : 1;
  M.nnx = nx + 1; M.nny = ny + 1; M.nnz = dim == 3 ? nz + 1 : 1;
  M.ncell = (long long)M.ncx * M.ncy * M.ncz;
  M.nnode = (long long)M.nnx * M.nny * M.nnz;
  M.o[0] = M.o[1] = M.o[2] = 0.;
  M.h[0] = M.h[1] = M.h[2] = 0.;
  if (M.ncell > MHC_NOALLOC_MAX_CELLS) {
    g_noalloc_err = "mesh has " + std::to_string(M.ncell) + " cells; the allocation-free variant handles at most " +
                    std::to_string(MHC_NOALLOC_MAX_CELLS) + " (use mhc_compute_delta_t on a case instead)";
    return MHC_ERR_ARG;
  }
  double* scratch = nullptr;
  int r = scratch_address(&scratch);
  if (r != MHC_OK) return r;
  const int nblocks = (int)((M.ncell + kThreads - 1) / kThreads);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_cfl_partial<<<nblocks, kThreads, 0, s>>>(M, char_length, sound_speed, vx, vy, vz, euler_full ? 1 : 0,
                                             scratch);
  k_cfl_final<<<1, kThreads, 0, s>>>(scratch, nblocks, cfl, old_deltat, deltat_max, deltat_min, deltat_out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_noalloc_err = cudaGetErrorString(e);
    return MHC_ERR_CUDA;
  }
  return MHC_OK;
}
