// persistent.cuh -- persistent CTAs over a work queue of jobs (the batched
// FFTSolver2D kernels).
//
// A batch group launches at most one wave of CTAs (the SMs times the CTAs a
// SM holds).  CTA b takes job b first; when it finishes a job it takes the
// next one from a device counter (atomicAdd, reset to zero before the
// launch), so job indices gridDim.x, gridDim.x + 1, ... go to the CTAs in the
// order they become free.  The host orders a group's jobs by steps, longest
// first, so the shorter jobs fill in behind the longer ones.  Without a
// counter every job has its own CTA (grid = number of jobs).
#pragma once
#include <cuda_runtime.h>

namespace pxp {

// The next job of this CTA; every thread of the CTA calls it after its last
// use of the previous job's shared memory.
__device__ __forceinline__ int next_job(unsigned *queue, int *s_slot) {
  __syncthreads();
  if (threadIdx.x == 0)
    *s_slot = queue != nullptr ? (int)gridDim.x + (int)atomicAdd(queue, 1u) : 0x7fffffff;
  __syncthreads();
  return *s_slot;
}

// Grid of a job launch: one CTA per job, or with a queue at most one wave.
inline int persistent_grid(const void *kernel, int threads, size_t smem, int njobs,
                           const unsigned *queue) {
  if (queue == nullptr) return njobs;
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) != cudaSuccess ||
      per < 1)
    per = 1;
  const int wave = sms * per;
  return njobs < wave ? njobs : wave;
}

}  // namespace pxp
