// Allocation-free form of the finest-level operator apply (A p and p . A p).
//
// Some host applications cannot let a plug-in allocate device memory: a game
// engine or renderer that has reserved the GPU's memory for its own pool, or a
// framework whose caching allocator holds the free memory, so that a cudaMalloc
// from this library would fail or break the host's memory budget.  For them this
// entry point does all of its work in caller-provided buffers plus one fixed
// scratch array that lives in this library's device image.
//
// The scratch array below is file-scope device memory: every GPU that loads
// the library holds it (about 128 KB) until the process exits.  Its name is a
// host-side stand-in, not a device address, so every call looks the address up
// with cudaGetSymbolAddress (with the caller's device current; the lookup
// allocates nothing) and passes it to the kernel.  Looking it up on every call
// keeps the address right after a device reset recreates the context.  Every
// call on a device shares the one array and it keeps the last call's contents,
// so calls whose GPU work overlaps (different streams, or the same stream from
// several threads without ordering) race on it.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/fluid_pp.h"
#include "device_util.cuh"

namespace {

// Partials of at most kNoAllocMaxTiles work tiles (32x8x4 cells each), then
// the arrival counter of the last-tile reduction.
constexpr int kNoAllocMaxTiles = 16384;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxTiles + 32];

// [a, a + na) and [b, b + nb) share a byte.
bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
  const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return x < y + nb && y < x + na;
}

}  // namespace

namespace fpp {
void set_global_error(const std::string& message);   // read back by fluid_pp_last_error(NULL)

constexpr int kNoAllocDepth = 4;   // cells per thread along z in the 32x8x4 work tiles

// out = A p on the finest level and *p_dot_ap = p . A p (float64, tile order).
// A is the ghost-fluid operator of k_spmv: diag on liquid cells, -1 to liquid
// neighbours; air entries of p are treated as zero.
__global__ void k_spmv_noalloc(int nx, int ny, int nz, const uint8_t* __restrict__ label,
                               const float* __restrict__ diag, const float* __restrict__ p, float* __restrict__ out,
                               double* __restrict__ p_dot_ap, double* scratch, int ntiles) {
  __shared__ double sh[32];
  __shared__ int flag;
  unsigned* counter = reinterpret_cast<unsigned*>(scratch + kNoAllocMaxTiles);
  const int sy = nx, sz = nx * ny;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    double dq = 0;
    int x, y, z, i;
    for (TileIt it(t, nx, ny, nz, kNoAllocDepth); it.next(x, y, z, i);) {
      float q = 0.0f;
      if (label[i]) {
        auto nb = [&](bool in, int j) { return (in && label[j]) ? p[j] : 0.0f; };
        const float s = d4sum6(nb(x > 0, i - 1), nb(x + 1 < nx, i + 1), nb(y > 0, i - sy), nb(y + 1 < ny, i + sy),
                               nb(z > 0, i - sz), nb(z + 1 < nz, i + sz));
        q = diag[i] * p[i] - s;
        dq += double(p[i]) * q;
      }
      out[i] = q;
    }
    const double a = block_sum(dq, sh);
    if (threadIdx.x == 0) scratch[t] = a;
    if (arrive_last(counter, ntiles, &flag)) {
      const double total = gather_slot(scratch, 0, ntiles, 0, sh);
      if (threadIdx.x == 0) *p_dot_ap = total;
    }
  }
}

}  // namespace fpp

extern "C" int fluid_pp_apply_operator_noalloc(int nx, int ny, int nz, const unsigned char* label,
                                               const float* diag, const float* p, float* out, double* p_dot_ap,
                                               void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || !label || !diag || !p || !out || !p_dot_ap) {
    fpp::set_global_error("fluid_pp_apply_operator_noalloc: null pointer or empty lattice");
    return FLUID_PP_INVALID_ARG;
  }
  const long long tiles = (long long)((nx + fpp::kTX - 1) / fpp::kTX) * ((ny + fpp::kTY - 1) / fpp::kTY) *
                          ((nz + fpp::kNoAllocDepth - 1) / fpp::kNoAllocDepth);
  if (tiles > kNoAllocMaxTiles || (long long)nx * ny * nz > (1LL << 30)) {
    fpp::set_global_error("fluid_pp_apply_operator_noalloc: lattice needs " + std::to_string(tiles) +
                    " work tiles of 32x8x4 cells; the fixed scratch holds " + std::to_string(kNoAllocMaxTiles));
    return FLUID_PP_INVALID_ARG;
  }
  // The kernel reads label, diag and p through restrict pointers while it
  // writes out and *p_dot_ap: an output that shares memory with an input would
  // give wrong neighbour values, so aliasing is rejected.
  const size_t cells = size_t(nx) * size_t(ny) * size_t(nz);
  const size_t vbytes = cells * sizeof(float);
  if (overlaps(out, vbytes, p, vbytes) || overlaps(out, vbytes, diag, vbytes) || overlaps(out, vbytes, label, cells) ||
      overlaps(p_dot_ap, sizeof(double), p, vbytes) || overlaps(p_dot_ap, sizeof(double), diag, vbytes) ||
      overlaps(p_dot_ap, sizeof(double), label, cells) || overlaps(p_dot_ap, sizeof(double), out, vbytes)) {
    fpp::set_global_error("fluid_pp_apply_operator_noalloc: out and p_dot_ap must not overlap label, diag, p or "
                          "each other");
    return FLUID_PP_INVALID_ARG;
  }
  // The scratch address of the current device, looked up on every call (the
  // array's host-side name is not a device address).
  void* ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (e != cudaSuccess) {
    fpp::set_global_error(std::string("fluid_pp_apply_operator_noalloc: cudaGetSymbolAddress: ") +
                          cudaGetErrorString(e));
    return FLUID_PP_CUDA;
  }
  double* scratch = static_cast<double*>(ptr);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The arrival counter must start at zero; the partials are all overwritten.
  e = cudaMemsetAsync(scratch + kNoAllocMaxTiles, 0, sizeof(double), s);
  if (e == cudaSuccess) {
    const int grid = int(tiles < 148 * 8 ? tiles : 148 * 8);
    fpp::k_spmv_noalloc<<<grid, fpp::kThreads, 0, s>>>(nx, ny, nz, label, diag, p, out, p_dot_ap, scratch, int(tiles));
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    fpp::set_global_error(std::string("fluid_pp_apply_operator_noalloc: ") + cudaGetErrorString(e));
    return FLUID_PP_CUDA;
  }
  return FLUID_PP_OK;
}

