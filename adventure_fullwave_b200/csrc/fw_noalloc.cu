// Batched skyline LDL^T substitution that allocates no device memory.
//
// Some callers cannot allocate device memory when they need a solve: code
// running inside a host framework that owns the device memory through its
// own pool and forbids raw cudaMalloc/cudaFree in its loop (a cudaFree waits
// for the whole device), or a real-time loop that must not enter the
// driver's allocator at all.  They pass every input and output buffer
// themselves; the work vectors the substitution needs live in one
// file-scope device array of fixed size instead of memory allocated per call.
//
// The scratch array is shared by every call in the process on a given GPU,
// and it keeps whatever the last call left in it.  Each call writes every
// row it uses before reading it, so nothing has to start at zero.  Two calls
// whose kernels overlap on the same GPU (different streams, or different
// host threads) use the same rows of the array and race: the caller must
// order them on one stream or synchronise between them.
//
// The device address of the array is looked up on every call, in the
// context current on the calling thread: after a cudaDeviceReset, or from a
// context of the caller's own, the library's module is loaded again and the
// array has a new address.  The first call in a context loads the module,
// so it should come before any stream capture the caller starts.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/fwgpu.h"

namespace {

// 262,144 complex FP64 rows: 4 MiB per GPU that loads the library, held
// until the process exits.
constexpr int64_t kNoAllocMaxRows = FWGPU_NOALLOC_MAX_ROWS;
static __device__ __align__(256) double2 g_noalloc_work[kNoAllocMaxRows];

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// One warp per system, in the reference's skyline layout: row i holds
// columns idx1[i]..i at mat[idx2[i] + j], unit L off the diagonal and 1/d
// on it (advlas_skyline.c:12-25,79-128).  Forward row dot products, scaling
// by 1/d, backward column updates (advlas_skyline_ldl_solve, :134-167).
// b and x may be the same buffer: a system reads all its rows of b before
// it writes any row of x, and systems do not share rows.
__global__ void skyline_solve_noalloc_kernel(int32_t n_systems, int32_t total_rows, const int32_t *__restrict__ row_off,
                                             const int64_t *__restrict__ mat_off, const int32_t *__restrict__ idx1,
                                             const int32_t *__restrict__ idx2, const double2 *__restrict__ mat,
                                             const double2 *b, double2 *x, double2 *__restrict__ work) {
  const int s = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (s >= n_systems) return;
  const int lane = threadIdx.x & 31;
  const int r0 = row_off[s];
  const int n = row_off[s + 1] - r0;
  // a system outside the caller's rows would reach past the work array
  if (r0 < 0 || n < 0 || r0 + n > total_rows) return;
  const int32_t *i1 = idx1 + r0;
  const int32_t *i2 = idx2 + r0;
  const double2 *m = mat + mat_off[s];
  double2 *w = work + r0;
  for (int i = lane; i < n; i += 32) w[i] = b[r0 + i];
  __syncwarp();
  // a first column outside [0, i] would reach rows of the shared work array
  // that belong to other systems: it is clamped (the result of such a
  // malformed system is meaningless, but no other system's rows are touched)
  for (int i = 1; i < n; i++) {
    double re = 0.0, im = 0.0;
    const int lo = min(max(i1[i], 0), i);
    for (int j = lo + lane; j < i; j += 32) {
      const double2 t = cmul(m[i2[i] + j], w[j]);
      re += t.x;
      im += t.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
      re += __shfl_xor_sync(0xffffffffu, re, o);
      im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if (lane == 0) w[i] = make_double2(w[i].x - re, w[i].y - im);
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) w[i] = cmul(w[i], m[i2[i] + i]);
  __syncwarp();
  for (int i = n - 1; i >= 1; i--) {
    const double2 xi = w[i];
    const int lo = min(max(i1[i], 0), i);
    for (int j = lo + lane; j < i; j += 32) {
      const double2 t = cmul(m[i2[i] + j], xi);
      w[j] = make_double2(w[j].x - t.x, w[j].y - t.y);
    }
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) x[r0 + i] = w[i];
}

}  // namespace

namespace fw {
// defined with the rest of the error reporting in fw_capi.cu
void record_error(const std::string &msg);
}  // namespace fw

namespace {
int noalloc_error(int code, const std::string &msg) {
  fw::record_error(msg);
  return code;
}
}  // namespace

extern "C" int fwgpu_skyline_solve_noalloc(int32_t n_systems, int32_t total_rows, const int32_t *d_row_off,
                                           const int64_t *d_mat_off, const int32_t *d_idx1, const int32_t *d_idx2,
                                           const double *d_mat, const double *d_b, double *d_x, void *stream) {
  if (n_systems < 0 || total_rows < 0) return noalloc_error(FWGPU_ERR_ARG, "negative size");
  if (total_rows > kNoAllocMaxRows)
    return noalloc_error(FWGPU_ERR_ARG, "total_rows " + std::to_string(total_rows) + " exceeds the fixed work array of " +
                                            std::to_string(kNoAllocMaxRows) + " rows");
  if (n_systems == 0 || total_rows == 0) return FWGPU_OK;
  if (!d_row_off || !d_mat_off || !d_idx1 || !d_idx2 || !d_mat || !d_b || !d_x)
    return noalloc_error(FWGPU_ERR_ARG, "null buffer");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_error(FWGPU_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  // the array's address in the current context (a host-side name of a
  // __device__ array is not a device address)
  void *ptr = nullptr;
  e = cudaGetSymbolAddress(&ptr, g_noalloc_work);
  if (e != cudaSuccess)
    return noalloc_error(FWGPU_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  double2 *work = (double2 *)ptr;
  const int threads = 128;
  const unsigned blocks = (unsigned)(((int64_t)n_systems * 32 + threads - 1) / threads);
  skyline_solve_noalloc_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(
      n_systems, total_rows, d_row_off, d_mat_off, d_idx1, d_idx2, (const double2 *)d_mat, (const double2 *)d_b, (double2 *)d_x,
      work);
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_error(FWGPU_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return FWGPU_OK;
}
