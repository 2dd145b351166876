// adi_noalloc.cu -- ADI steps on a caller-owned device field with no device
// memory allocation.
//
// An ADI step (ADI::solveStep, src/alternatingDirectionSolver.cpp:136-155)
// needs one field-sized buffer between its x and y half steps.  The solver
// handle of capi.cu allocates that buffer with cudaMalloc; this entry point
// instead keeps it in a fixed array compiled into the library
// (kNoAllocScratchBytes, 4 MiB per GPU that loads the library, held until
// the process exits) and calls no cudaMalloc, cudaFree or any allocating
// routine.  It runs the general half-step kernel (adi.cu), whose sphere list
// travels in the kernel parameters.
//
// Who needs it: callers that must not allocate device memory while they
// run -- code whose device memory is already carved up by another allocator
// (a framework's caching allocator or a fixed per-process pool) and
// latency-critical loops, where cudaMalloc/cudaFree can synchronise the
// device and stall every other stream.  Errors are reported through
// pxp_last_error(NULL, ...).
//
// The array is shared by every call on a device and keeps the last call's
// contents.  Nothing in it has to start at zero: each x half step writes all
// n*n points before the y half step reads them.  Calls that overlap on the
// GPU (concurrent streams, or several host threads) race on the array and
// must be serialised by the caller.
//
// The array's device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, on the first call that
// uses the device; that first call should therefore come before any stream
// capture.  The call makes problem->device current for its launches and
// gives the caller's current device back before it returns.  Every plane the
// steps sample is checked before the first launch: a refused call (more
// than 16 spheres meeting one plane) leaves the field untouched.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/paxpro_b200.h"
#include "pxp_kernels.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;  // 4 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_adi_scratch[kNoAllocScratchBytes];

std::mutex g_mutex;
void *g_scratch_ptr[kMaxDevices] = {};

// Errors are reported through pxp_last_error(NULL, ...).
int fail(int code, const char *msg) {
  pxp::set_last_error(msg);
  return code;
}

// Device address of the scratch array on the current device (set-up once per
// device).  The host-side name g_adi_scratch is not a device address.
int scratch_for_current_device(void **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(PXP_ERR_CUDA, "cudaGetDevice failed");
  if (dev < 0 || dev >= kMaxDevices) return fail(PXP_ERR_UNSUPPORTED, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mutex);
  if (g_scratch_ptr[dev] == nullptr) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_adi_scratch);
    if (e != cudaSuccess || p == nullptr) {
      char m[160];
      std::snprintf(m, sizeof(m), "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      pxp::set_last_error(m);
      return PXP_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return PXP_OK;
}

// Spheres that can contain a point of plane z, the handle path's test
// (fl(dz^2) < fl(R^2)), copied in list order into out (when not null) up to
// kInlineSpheres; returns how many there are.
int spheres_meeting(const pxp_sphere *spheres, int nspheres, double z, pxp::Sphere *out) {
  int c = 0;
  for (int i = 0; i < nspheres; ++i) {
    volatile double dz = z - spheres[i].cz;
    volatile double dz2 = dz * dz;
    volatile double r2 = spheres[i].radius * spheres[i].radius;
    if (!(dz2 < r2)) continue;
    if (out && c < pxp::kInlineSpheres)
      out[c] = {spheres[i].cx, spheres[i].cy, spheres[i].cz, spheres[i].radius, spheres[i].delta,
                spheres[i].beta};
    ++c;
  }
  return c;
}

// The launches of pxp_adi_steps_noalloc, on the current device; the planes
// were checked by the caller.
int run_steps(const pxp_problem *p, pxp::Precision prec, unsigned n, const pxp_sphere *spheres,
              int nspheres, void *dfield, unsigned first_step, int nsteps, cudaStream_t st) {
  void *scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  const double dzh = p->z.step / 2.0;  // ADI::xImplicit (src/alternatingDirectionSolver.cpp:18)
  const double k = p->wavenumber;
  const double kdx2 = k * p->x.step * p->x.step, kdy2 = k * p->y.step * p->y.step;
  pxp::AdiHalf a{};
  a.n = (int)n;
  // sizes other than powers of two: systems padded with decoupled rows, as
  // the solver handle runs them
  a.n_pad = pxp::adi_padded_n((int)n) != (int)n ? pxp::adi_padded_n((int)n) : 0;
  a.use_tbc = p->transparent_bc ? 1 : 0;
  a.inv_dzh = 1.0 / dzh;
  a.k = k;
  a.xmin = p->x.min;
  a.dx = p->x.step;
  a.ymin = p->y.min;
  a.dy = p->y.step;
  a.spheres_all = nullptr;
  a.save = nullptr;
  for (int i = 0; i < nsteps; ++i) {
    const unsigned step = first_step + (unsigned)i;
    const double z = p->z.min + step * p->z.step;  // getZ
    // x half step: field -> scratch (ADI::xImplicit, :8-76)
    a.in = dfield;
    a.out = scratch;
    a.stride_pos = n;
    a.stride_sys = 1;
    a.y_implicit = 0;
    a.kd2_impl = kdx2;
    a.kd2_expl = kdy2;
    a.z = z;
    a.nspheres = spheres_meeting(spheres, nspheres, a.z, a.spheres);
    cudaError_t e = pxp::launch_adi_half(prec, a, st);
    if (e != cudaSuccess) return fail(PXP_ERR_CUDA, cudaGetErrorString(e));
    // y half step: scratch -> field (ADI::yImplicit, :78-134)
    a.in = scratch;
    a.out = dfield;
    a.stride_pos = 1;
    a.stride_sys = n;
    a.y_implicit = 1;
    a.kd2_impl = kdy2;
    a.kd2_expl = kdx2;
    a.z = z + dzh;
    a.nspheres = spheres_meeting(spheres, nspheres, a.z, a.spheres);
    e = pxp::launch_adi_half(prec, a, st);
    if (e != cudaSuccess) return fail(PXP_ERR_CUDA, cudaGetErrorString(e));
  }
  return PXP_OK;
}

}  // namespace

extern "C" {

int pxp_adi_steps_noalloc(const pxp_problem *p, const pxp_sphere *spheres, int nspheres,
                          void *dfield, unsigned first_step, int nsteps, void *stream) {
  if (p == nullptr || dfield == nullptr || nsteps < 0 || first_step < 1 || nspheres < 0 ||
      (nspheres > 0 && spheres == nullptr))
    return fail(PXP_ERR_INVALID, "pxp_adi_steps_noalloc: invalid argument");
  if (p->kind != PXP_ADI) return fail(PXP_ERR_INVALID, "pxp_adi_steps_noalloc: kind must be PXP_ADI");
  if (p->precision != PXP_FP64 && p->precision != PXP_FP32)
    return fail(PXP_ERR_INVALID, "pxp_adi_steps_noalloc: unknown precision");
  if (!(p->x.step > 0.0) || !(p->y.step > 0.0) || !(p->z.step > 0.0) || !(p->wavenumber > 0.0))
    return fail(PXP_ERR_INVALID, "pxp_adi_steps_noalloc: steps and wavenumber must be positive");
  const unsigned n = pxp_node_count(p->x.min, p->x.max, p->x.step);
  const pxp::Precision prec = p->precision == PXP_FP64 ? pxp::kFP64 : pxp::kFP32;
  const size_t csize = prec == pxp::kFP64 ? 16 : 8;
  const size_t bytes = (size_t)n * n * csize;
  if (bytes > kNoAllocScratchBytes) {
    char m[200];
    std::snprintf(m, sizeof(m),
                  "pxp_adi_steps_noalloc: field of %u x %u needs %zu bytes of scratch; the "
                  "maximum is %zu (4 MiB)",
                  n, n, bytes, kNoAllocScratchBytes);
    return fail(PXP_ERR_UNSUPPORTED, m);
  }
  if (!pxp::adi_padded_supported(prec, (int)n))
    return fail(PXP_ERR_UNSUPPORTED, "pxp_adi_steps_noalloc: grid size not supported");

  const double dzh = p->z.step / 2.0;  // ADI::xImplicit (src/alternatingDirectionSolver.cpp:18)
  // Every plane the call samples (getZ(step) for the x half step, getZ(step) +
  // dz/2 for the y half step) is checked before the first launch, so a call
  // that is refused leaves the caller's field untouched.
  for (int i = 0; i < nsteps; ++i) {
    const double z = p->z.min + (first_step + (unsigned)i) * p->z.step;  // getZ
    if (spheres_meeting(spheres, nspheres, z, nullptr) > pxp::kInlineSpheres ||
        spheres_meeting(spheres, nspheres, z + dzh, nullptr) > pxp::kInlineSpheres)
      return fail(PXP_ERR_UNSUPPORTED,
                  "pxp_adi_steps_noalloc: more than 16 spheres meet one plane; nothing was run");
  }

  // Run on the problem's device and give the caller's current device back.
  int caller_dev = 0;
  if (cudaGetDevice(&caller_dev) != cudaSuccess) return fail(PXP_ERR_CUDA, "cudaGetDevice failed");
  if (caller_dev != p->device && cudaSetDevice(p->device) != cudaSuccess)
    return fail(PXP_ERR_CUDA, "cudaSetDevice failed");
  const int rc = run_steps(p, prec, n, spheres, nspheres, dfield, first_step, nsteps,
                           (cudaStream_t)stream);
  if (caller_dev != p->device) cudaSetDevice(caller_dev);
  return rc;
}

}  // extern "C"
