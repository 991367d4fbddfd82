// pmx_heev_batched_noalloc: the batched Hermitian eigensolver on caller-owned
// device buffers, with its scratch in one fixed file-scope device array, so
// that a call allocates nothing.
//
// pmx_heev_batched stages the matrices, the item table and the
// inverse-iteration vectors in device buffers that the context grows with
// cudaMalloc. Two kinds of caller cannot let the library allocate:
//   * a host program that reserved the device memory up front for its own
//     pool (a caching allocator that holds most of HBM): a cudaMalloc here
//     can fail, or take memory the pool counted on;
//   * code on a latency path that drives several streams: cudaMalloc and
//     cudaFree synchronise the device, which stalls every stream of the
//     process for the length of whatever is in flight.
// This entry point runs the same eigensolver kernel; the item table and the
// inverse-iteration vectors live in g_noalloc_scratch (16 MiB, fixed at build
// time), inputs and outputs in the caller's device memory.
#include <cuda_runtime.h>

#include <mutex>

#include "../../../include/picomax.h"
#include "pmx_device.hpp"

namespace {

using pmx::dev::EigItem;

constexpr size_t kScratchBytes = size_t(16) << 20;  // the whole array
constexpr int kMaxItems = 1024;                     // matrices per call
constexpr size_t kItemBytes = (kMaxItems * sizeof(EigItem) + 255) / 256 * 256;
constexpr size_t kVecDoubles = (kScratchBytes - kItemBytes) / sizeof(double);
// Above n = 832 the eigensolver keeps per-warp partial sums in global scratch,
// which this entry point's item layout does not provide.
constexpr int kMaxN = 832;
constexpr int kMaxDevices = 64;

// Shared by every call on a device: [item table | inverse-iteration vectors].
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

unsigned char* g_scratch_ptr[kMaxDevices];
cudaError_t g_setup_status[kMaxDevices];
std::once_flag g_setup_once[kMaxDevices];

// Item i: matrix at A + i n^2, eigenvalues at w + i nev, eigenvectors at
// z + i nev n, inverse-iteration vectors at 4 n nev i of the scratch.
__global__ void noalloc_items_kernel(EigItem* items, int batch, int n, int nev, int want_vec) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= batch) return;
  EigItem it{};
  it.n = n;
  it.nev = want_vec ? nev : 0;
  it.nval = nev;
  it.want_vec = want_vec;
  it.h_off = (long long)i * n * n;
  it.w_off = (long long)i * nev;
  it.z_off = (long long)i * nev * n;
  it.s_off = (long long)i * 4 * n * nev;
  items[i] = it;
}

}  // namespace

extern "C" int pmx_heev_batched_noalloc(void* stream, int n, int batch, double* A, int nev, double* w, double* z,
                                        int* info) {
  if (n <= 0 || batch < 0 || nev <= 0 || nev > n || nev > 512 || (batch > 0 && (!A || !w || !info)))
    return PMX_ERR_INVALID;
  if (n > kMaxN || batch > kMaxItems) return PMX_ERR_LIMIT;
  if (z && (size_t)4 * n * nev * (size_t)batch > kVecDoubles) return PMX_ERR_LIMIT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PMX_ERR_NO_DEVICE;
  if (dev < 0 || dev >= kMaxDevices) return PMX_ERR_LIMIT;
  // set-up, once per device, with that device current
  std::call_once(g_setup_once[dev], [dev]() {
    void* p = nullptr;
    g_setup_status[dev] = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    g_scratch_ptr[dev] = g_setup_status[dev] == cudaSuccess ? static_cast<unsigned char*>(p) : nullptr;
  });
  if (g_setup_status[dev] != cudaSuccess || !g_scratch_ptr[dev]) return PMX_ERR_CUDA;
  if (batch == 0) return PMX_OK;

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  EigItem* items = reinterpret_cast<EigItem*>(g_scratch_ptr[dev]);
  double* vecs = reinterpret_cast<double*>(g_scratch_ptr[dev] + kItemBytes);
  // every call rewrites the item table and each vector slot before reading
  // it, so nothing left by the previous call needs clearing
  noalloc_items_kernel<<<(batch + 127) / 128, 128, 0, st>>>(items, batch, n, nev, z ? 1 : 0);
  if (cudaGetLastError() != cudaSuccess) return PMX_ERR_CUDA;
  double2* a2 = reinterpret_cast<double2*>(A);
  const cudaError_t err = pmx::dev::launch_heev(items, batch, n, nev, a2, w, z ? reinterpret_cast<double2*>(z) : a2,
                                                vecs, info, st);
  return err == cudaSuccess ? PMX_OK : PMX_ERR_CUDA;
}
