// smem_attr.cu -- per-device bookkeeping of the dynamic shared-memory limit
// of each kernel.
//
// cudaFuncAttributeMaxDynamicSharedMemorySize belongs to a kernel in one
// device's context: raising it while device 0 is current leaves the default
// 48 KB on device 1 (and a kernel with static shared memory gets less than
// 48 KB of dynamic memory by default).  The launchers call
// pxp::raise_dynamic_smem before every launch; the attribute is set on the
// current device the first time a (kernel, device) pair asks for at least
// that many bytes, and the lookup is a short locked map search afterwards.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

#include "pxp_kernels.h"

namespace {
std::mutex g_mutex;
std::map<std::pair<const void *, int>, int> g_set;  // (kernel, device) -> bytes set
}  // namespace

cudaError_t pxp::raise_dynamic_smem(const void *kernel, int bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_mutex);
  auto key = std::make_pair(kernel, dev);
  auto it = g_set.find(key);
  if (it != g_set.end() && it->second >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  g_set[key] = bytes;
  return cudaSuccess;
}

namespace {
std::map<std::pair<const void *, int>, int> g_carve;  // (kernel, device) -> percent set
}  // namespace

cudaError_t pxp::prefer_smem_carveout(const void *kernel, int bytes, int ctas) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_mutex);
  auto key = std::make_pair(kernel, dev);
  if (g_carve.count(key)) return cudaSuccess;
  int per_sm = 0;
  e = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  if (e != cudaSuccess) return e;
  // the driver adds 1 KB a CTA and rounds the percentage up to the next
  // carve-out it supports: ask for the largest percentage that still rounds
  // to the smallest supported carve-out holding the CTAs
  static const int kCarveKB[] = {0, 8, 16, 32, 64, 100, 132, 164, 196, 228};
  const long long need = ((long long)bytes + 1024) * (ctas > 0 ? ctas : 1);
  int pct = 100;
  for (int kb : kCarveKB)
    if (1024LL * kb >= need && per_sm > 0) {
      pct = (int)((100LL * 1024 * kb) / per_sm);
      break;
    }
  if (pct > 100) pct = 100;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
  if (e != cudaSuccess) return e;
  g_carve[key] = pct;
  return cudaSuccess;
}
