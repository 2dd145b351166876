// capi.cu -- the C ABI (include/paxpro_b200.h): solver handles, device state,
// host-side FP64 tables and kernel launches.
//
// A handle owns one CUDA stream, the resident field, the per-solver tables
// and the save slots.  Nothing here throws across the ABI: every entry point
// catches, records a message on the handle and returns a status.
//
// Host tables that the reference evaluates with std::complex (the FFTSolver2D
// propagator, src/fftSolver2D.cpp:15-19, and the transmission factor,
// src/fftSolver2D.cpp:46-48) are built here with the same std::complex
// expressions (this file's host code is compiled with -ffp-contract=off), so
// the FP64 device path multiplies by exactly the reference's values.  FP32
// served mode rounds the FP64 values (phase reduced in FP64) to complex64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <tuple>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/paxpro_b200.h"
#include "pxp_kernels.h"

using cd = std::complex<double>;

namespace {

const double PI = std::acos(-1.0);
std::mutex g_err_mutex;
std::string g_last_error;

void set_global_error(const std::string &m) {
  std::lock_guard<std::mutex> lk(g_err_mutex);
  g_last_error = m;
}

bool is_pow2(long long n) { return n > 0 && (n & (n - 1)) == 0; }

}  // namespace

void pxp::set_last_error(const char *msg) { set_global_error(msg ? msg : ""); }

struct pxp_solver_s {
  pxp_problem prob{};
  unsigned nx = 0, ny = 1, nz = 0;
  long long npts = 0;
  pxp::Precision prec = pxp::kFP64;
  size_t csize = 16;
  cudaStream_t stream = nullptr;
  // resident state
  void *d_field = nullptr;
  void *d_saves = nullptr;
  int max_slots = 0;
  int save_every = 0;
  // FFT 1-D tables
  void *d_kern = nullptr, *d_trans = nullptr, *d_tw = nullptr;
  void *d_wn = nullptr;  // exp(-2 pi i m / n) (shared table, not owned)
  void *d_chirp = nullptr, *d_bconv = nullptr;  // Bluestein tables (shared, not owned)
  long long trans_stride = 0;
  int trans_step0 = 1;
  // CN material planes (FP64)
  double *d_mat = nullptr;  // [delta | beta | delta_prev | beta_prev] planes
  long long mat_block = 0;  // doubles per block of d_mat
  long long mat_stride = 0;
  int mat_step0 = 1;
  // job descriptors in device memory
  void *d_job = nullptr;
  // 2-transverse-dim solvers
  void *d_field2 = nullptr;                  // ping-pong buffer
  void *d_lu = nullptr;                      // factor tables of step-invariant matrices
  int adi_tab_run[2][2] = {};                // x / y staged ADI tables: identical chunks
  bool cn_const = false;                     // CN matrix step-invariant
  size_t dev_bytes = 0;                      // device memory held by the handle
  pxp::Fft1dJob job_fft{};                   // host copies of the job descriptors
  pxp::CnJob job_cn{};
  int batch_remaining = 0;                   // steps left while admitted to a batch
  std::vector<pxp_sphere> spheres;           // first-hit sphere material
  // CSG material: device copy [modules | parts | shapes] and, per module, the
  // z range that can contain its material (lo > hi: none; -inf/+inf: any)
  void *d_csg = nullptr;
  int csg_nmodules = 0, csg_nparts = 0;
  std::vector<double> csg_zlo, csg_zhi;
  pxp::Sphere *d_spheres = nullptr;
  // field the far field subtracts (complex128, npts; null when not set)
  void *d_ref = nullptr;
  // per-step flux windows and sums of the 2-D step kernels
  int2 *d_flux_win = nullptr;
  double *d_flux = nullptr;
  int flux_step0 = 0, flux_count = 0;
  // host copies
  std::vector<double> h_delta, h_beta;
  int plane_first = 1, plane_count = 0;  // per-step material planes (0 = z-invariant)
  // 3-D kinds: sampled material planes for steps plane_first .. +plane_count-1,
  // planes3_per a step (FFTSolver3D 1, ADI 2): [delta planes | beta planes]
  double *d_planes3 = nullptr;
  size_t planes3_cap = 0;  // doubles allocated
  int planes3_per = 0;
  bool planes3_invariant = false;  // one plane (a z-invariant table) for every step
  bool material_set = false;
  bool ic_set = false;
  unsigned current_step = 1;
  unsigned timeouts_seen = 0;  // device count of ran-out kernel waits at creation
  // saved fields: save_pts points each (3-D kinds: save_n x save_n block
  // averages of the field when the transverse downsampling ratio is above 1,
  // staged through d_save_stage)
  unsigned save_n = 0;
  long long save_pts = 0;
  void *d_save_stage = nullptr;
  // captured block of step-invariant steps (replay_steps) and the buffers
  // and launch choices it was captured with
  cudaGraphExec_t graph = nullptr;
  std::vector<const void *> graph_sig;
  std::string err;

  int fail(int code, const std::string &m) {
    err = m;
    set_global_error(m);
    return code;
  }
  int cuda_fail(cudaError_t e, const char *what) {
    return fail(PXP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
};

namespace {

#define PXP_TRY_CUDA(h, expr)                        \
  do {                                               \
    cudaError_t e_ = (expr);                         \
    if (e_ != cudaSuccess) return (h)->cuda_fail(e_, #expr); \
  } while (0)

// Device memory of a handle comes from the stream-ordered allocator on the
// handle's stream (cudaMallocAsync), so creating and destroying solvers does
// not synchronise the device (serving creates and retires many).
template <typename T> void free_dev(T *&p, cudaStream_t s = nullptr) {
  if (p) cudaFreeAsync((void *)p, s);
  p = nullptr;
}

// Keep freed pool memory for reuse instead of returning it at every
// synchronisation (once per device; a process-local pool attribute).
void retain_pool(int device) {
  static std::mutex m;
  static bool done[64] = {};
  std::lock_guard<std::mutex> lk(m);
  if (device < 0 || device >= 64 || done[device]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    unsigned long long thr = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  done[device] = true;
}

// Twiddles of the shared-memory Stockham transform in pass order (layout of
// fft_smem.cuh): for each pass (sub-transform length ns, radix r = 8 while it
// divides the rest, then 4 or 2), entries (q-1)*ns + k = exp(-2 pi i q k /
// (ns r)), in extended precision.  At least n entries are allocated.
std::vector<cd> twiddles(int n, int maxr = 8) {
  std::vector<cd> w(std::max(n, 1));
  const long double pi_l = 3.141592653589793238462643383279502884L;
  int off = 0;
  for (int ns = 1; ns < n;) {
    const int r = n / ns >= maxr ? maxr : (n / ns >= 8 ? 8 : n / ns);
    if (r < 2) break;  // n not a power of two: no further pass divides it
    for (int q = 1; q < r; ++q)
      for (int k = 0; k < ns; ++k) {
        long double a = -2.0L * pi_l * (long double)(q * k) / (long double)(ns * r);
        w[off + (q - 1) * ns + k] = cd((double)cosl(a), (double)sinl(a));
      }
    off += (r - 1) * ns;
    ns *= r;
  }
  return w;
}

// FFTSolver2D::spatialFreq (src/fftSolver2D.cpp:52-59).
double spatial_freq(unsigned indx, unsigned size, double step) {
  if (indx > size / 2) indx = size - indx;
  return 2.0 * PI * indx / (step * size);
}

// FFTSolver2D::kernel (src/fftSolver2D.cpp:15-19).
cd kernel_2d(double kx, double dz, double k) {
  cd A(0.0, 0.5 * dz / k);
  return std::exp(-A * kx * kx);
}

// Transmission factor of FFTSolver2D::refraction (src/fftSolver2D.cpp:46-48).
cd transmission(double k, double beta, double delta, double dz) {
  cd im(0.0, 1.0);
  return std::exp(-k * (beta + im * delta) * dz);
}

// Host-to-device copy on the handle's stream, finished before returning (the
// host buffers are temporaries).
int h2d(pxp_solver_s *h, void *dst, const void *src, size_t bytes) {
  PXP_TRY_CUDA(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream));
  PXP_TRY_CUDA(h, cudaStreamSynchronize(h->stream));
  return PXP_OK;
}

// Upload complex128 host values in the solver's precision.
int upload_complex(pxp_solver_s *h, void *dst, const cd *src, long long n) {
  if (h->prec == pxp::kFP64) {
    if (int rc_ = h2d(h, dst, src, sizeof(cd) * n)) return rc_;
  } else {
    std::vector<float> tmp(2 * n);
    for (long long i = 0; i < n; ++i) {
      tmp[2 * i] = (float)src[i].real();
      tmp[2 * i + 1] = (float)src[i].imag();
    }
    if (int rc_ = h2d(h, dst, tmp.data(), sizeof(float) * 2 * n)) return rc_;
  }
  return PXP_OK;
}

// Constant-factor tables of the FFT kernels (twiddles, propagators,
// transmissions, Bluestein chirps): complex128 entries in FP64 mode; in FP32
// served mode each complex128 value w split into two complex64 parts, hi =
// fl32(w) and lo = fl32(w - hi), stored (hi.re, hi.im, lo.re, lo.im), which
// the kernels multiply with one chain of FP32 FMAs (fft_smem.cuh).  Both
// forms take 16 bytes an entry.
size_t table_entry_bytes(const pxp_solver_s *) { return 16; }

std::vector<float> split_table(const std::vector<cd> &t) {
  std::vector<float> o(4 * t.size());
  for (size_t i = 0; i < t.size(); ++i) {
    const double re = t[i].real(), im = t[i].imag();
    const float hr = (float)re, hi = (float)im;
    o[4 * i] = hr;
    o[4 * i + 1] = hi;
    o[4 * i + 2] = (float)(re - (double)hr);
    o[4 * i + 3] = (float)(im - (double)hi);
  }
  return o;
}

int upload_table(pxp_solver_s *h, void *dst, const cd *src, long long n) {
  if (h->prec == pxp::kFP64) {
    PXP_TRY_CUDA(h, cudaMemcpyAsync(dst, src, sizeof(cd) * n, cudaMemcpyHostToDevice, h->stream));
  } else {
    const std::vector<float> sp = split_table(std::vector<cd>(src, src + n));
    PXP_TRY_CUDA(h, cudaMemcpyAsync(dst, sp.data(), sizeof(float) * sp.size(),
                                    cudaMemcpyHostToDevice, h->stream));
  }
  PXP_TRY_CUDA(h, cudaStreamSynchronize(h->stream));
  return PXP_OK;
}

int alloc(pxp_solver_s *h, void **p, size_t bytes, const char *what) {
  cudaError_t e = cudaMallocAsync(p, bytes, h->stream);
  if (e == cudaSuccess) h->dev_bytes += bytes;
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return h->fail(e == cudaErrorMemoryAllocation ? PXP_ERR_NOMEM : PXP_ERR_CUDA,
                   std::string("allocating ") + what + ": " + cudaGetErrorString(e));
  }
  return PXP_OK;
}

// ---- shared read-only tables ---------------------------------------------
// Twiddle and propagator tables depend only on the device, the length and the
// grid steps, so solvers with the same ones share a single device copy,
// built once and kept until the process exits (serving creates many solvers
// with the same grids).  The handles do not own these copies.
struct TableKey {
  int device, kind;  // kind 0: twiddles (radix 8), 1: 1-D propagator, 2: kx^2 per
                     // column, 3: twiddles (radix 16), 4: exp(-2 pi i m / n), m < n,
                     // 11: the FFTSolver3D register-line kernel's twiddle table
  unsigned n;
  double dx, dz, k;
  int split;  // 1: the FP32 split form (split_table), 0: complex128 / doubles
  bool operator<(const TableKey &o) const {
    return std::tie(device, kind, n, dx, dz, k, split) <
           std::tie(o.device, o.kind, o.n, o.dx, o.dz, o.k, o.split);
  }
};

std::mutex g_table_mutex;
std::map<TableKey, void *> g_tables;

// Upload a shared table (complex128 values, or their split form) and
// register it under key; the caller holds g_table_mutex.
int store_shared(pxp_solver_s *h, const TableKey &key, const std::vector<cd> &t, void **out,
                 const char *what) {
  std::vector<float> sp;
  if (key.split) sp = split_table(t);
  void *p = nullptr;
  if (cudaMalloc(&p, sizeof(cd) * t.size()) != cudaSuccess) {
    cudaGetLastError();
    return h->fail(PXP_ERR_NOMEM, std::string(what) + " allocation");
  }
  const cudaError_t e = cudaMemcpy(p, key.split ? (const void *)sp.data() : (const void *)t.data(),
                                   sizeof(cd) * t.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(p);
    return h->cuda_fail(e, (std::string(what) + " upload").c_str());
  }
  g_tables[key] = p;
  *out = p;
  return PXP_OK;
}

int shared_table_n(pxp_solver_s *h, int kind, unsigned n, void **out);

int shared_table(pxp_solver_s *h, int kind, void **out) { return shared_table_n(h, kind, h->nx, out); }

// The table of the given kind for length n (the grid's own length for the
// propagator and kx^2 tables).
int shared_table_n(pxp_solver_s *h, int kind, unsigned n, void **out) {
  TableKey key{h->prob.device, kind, n, (kind == 1 || kind == 2) ? h->prob.x.step : 0.0,
               kind == 1 ? h->prob.z.step : 0.0, kind == 1 ? h->prob.wavenumber : 0.0,
               (h->prec == pxp::kFP32 && kind != 2) ? 1 : 0};
  std::lock_guard<std::mutex> lk(g_table_mutex);
  auto it = g_tables.find(key);
  if (it != g_tables.end()) {
    *out = it->second;
    return PXP_OK;
  }
  std::vector<cd> t;
  std::vector<double> t2;
  if (kind == 0 || kind == 3) {
    t = twiddles((int)n, kind == 3 ? 16 : 8);
  } else if (kind == 4) {
    // exp(-2 pi i m / n), m < n, in extended precision
    t.resize(n);
    const long double pi_l = 3.141592653589793238462643383279502884L;
    for (unsigned m = 0; m < n; ++m) {
      const long double a = -2.0L * pi_l * (long double)m / (long double)n;
      t[m] = cd((double)cosl(a), (double)sinl(a));
    }
  } else if (kind == 11) {
    // the register-line kernel's twiddles of its earlier radix-8 passes:
    // exp(-2 pi i m / n) at the exponents that kernel lists
    std::vector<int> ex(n);
    const int cnt = pxp::fft3d_lines_tw_exponents((int)n, ex.data(), (int)n);
    if (cnt <= 0) {
      *out = nullptr;
      return PXP_OK;
    }
    t.resize(cnt);
    const long double pi_l = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < cnt; ++i) {
      const long double a = -2.0L * pi_l * (long double)ex[i] / (long double)n;
      t[i] = cd((double)cosl(a), (double)sinl(a));
    }
  } else if (kind == 1) {
    t.resize(n);
    for (unsigned i = 0; i < n; ++i)
      t[i] = kernel_2d(spatial_freq(i, n, h->prob.x.step), h->prob.z.step, h->prob.wavenumber);
  } else {
    // fl(kx*kx) with kx = spatialFreqX (src/fftSolver3D.cpp:32-40)
    t2.resize(n);
    for (unsigned i = 0; i < n; ++i) {
      const double kx = spatial_freq(i, n, h->prob.x.step);
      t2[i] = kx * kx;
    }
  }
  if (kind != 2) return store_shared(h, key, t, out, "shared table");
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, sizeof(double) * n);
  if (e != cudaSuccess) return h->fail(PXP_ERR_NOMEM, "shared table allocation");
  e = cudaMemcpy(p, t2.data(), sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return h->cuda_fail(e, "shared table upload");
  g_tables[key] = p;
  *out = p;
  return PXP_OK;
}

// FFTSolver3D: one factor of the separable propagator, exp(-i a k_i^2) with
// k_i = spatialFreq(i) for the x (axis 0) or y (axis 1) step and
// a = dz / (2k), the phase reduced in extended precision; complex128 in
// FP64, the split form in FP32.
int prop3_table(pxp_solver_s *h, int axis, void **out) {
  const unsigned n = h->nx;
  const double step = axis == 0 ? h->prob.x.step : h->prob.y.step;
  TableKey key{h->prob.device, 10, n, step, h->prob.z.step, h->prob.wavenumber,
               h->prec == pxp::kFP32 ? 1 : 0};
  std::lock_guard<std::mutex> lk(g_table_mutex);
  auto it = g_tables.find(key);
  if (it != g_tables.end()) {
    *out = it->second;
    return PXP_OK;
  }
  const long double a = 0.5L * (long double)h->prob.z.step / (long double)h->prob.wavenumber;
  std::vector<cd> t(n);
  for (unsigned i = 0; i < n; ++i) {
    const long double kx = spatial_freq(i, n, step);
    const long double phi = a * kx * kx;
    t[i] = cd((double)cosl(phi), -(double)sinl(phi));
  }
  return store_shared(h, key, t, out, "propagator table");
}

// ---- FFT 1-D -------------------------------------------------------------
// In-place radix-2 FFT in extended precision (host tables only).
void fft_ld(std::vector<std::complex<long double>> &a, int sign) {
  const size_t n = a.size();
  for (size_t i = 1, j = 0; i < n; ++i) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  const long double pi_l = 3.141592653589793238462643383279502884L;
  for (size_t len = 2; len <= n; len <<= 1) {
    for (size_t i = 0; i < n; i += len)
      for (size_t k = 0; k < len / 2; ++k) {
        const long double ang = (long double)sign * 2.0L * pi_l * (long double)k / (long double)len;
        const std::complex<long double> w(cosl(ang), sinl(ang));
        const std::complex<long double> x = a[i + k], y = a[i + k + len / 2] * w;
        a[i + k] = x + y;
        a[i + k + len / 2] = x - y;
      }
  }
}

// Tables of the Bluestein path for n (not a power of two), shared per
// device and n: kind 7 the chirp exp(-i pi j^2 / n), j < n (angle from the
// exact index j^2 mod 2n); kind 8 the transform of the filter
// b_j = exp(+i pi j^2 / n) for |j| < n wrapped to length m, divided by m;
// kind 9 the Stockham twiddles of length m.
int bluestein_table(pxp_solver_s *h, int kind, void **out) {
  const unsigned n = h->nx;
  const int m = pxp::fft1d_bluestein_m((int)n);
  TableKey key{h->prob.device, kind, n, 0.0, 0.0, 0.0, h->prec == pxp::kFP32 ? 1 : 0};
  std::lock_guard<std::mutex> lk(g_table_mutex);
  auto it = g_tables.find(key);
  if (it != g_tables.end()) {
    *out = it->second;
    return PXP_OK;
  }
  const long double pi_l = 3.141592653589793238462643383279502884L;
  auto chirp = [&](unsigned long long j, int sign) {
    const unsigned long long r = (j * j) % (2ULL * n);
    const long double a = (long double)sign * pi_l * (long double)r / (long double)n;
    return std::complex<long double>(cosl(a), sinl(a));
  };
  std::vector<cd> t;
  if (kind == 7) {
    t.resize(n);
    for (unsigned j = 0; j < n; ++j) {
      const std::complex<long double> c = chirp(j, -1);
      t[j] = cd((double)c.real(), (double)c.imag());
    }
  } else if (kind == 8) {
    std::vector<std::complex<long double>> b((size_t)m, std::complex<long double>(0.0L, 0.0L));
    for (unsigned j = 0; j < n; ++j) {
      b[j] = chirp(j, +1);
      if (j > 0) b[(size_t)m - j] = b[j];
    }
    fft_ld(b, -1);
    t.resize((size_t)m);
    for (int k = 0; k < m; ++k)
      t[(size_t)k] = cd((double)(b[(size_t)k].real() / m), (double)(b[(size_t)k].imag() / m));
  } else {
    t = twiddles(m);
  }
  return store_shared(h, key, t, out, "Bluestein table");
}

int fft1d_setup(pxp_solver_s *h) {
  int rc;
  if ((rc = shared_table(h, 1, &h->d_kern))) return rc;
  if (h->nx & (h->nx - 1)) {
    // not a power of two: the Bluestein path's tables (the Stockham twiddles
    // are those of its power-of-two length)
    if ((rc = bluestein_table(h, 7, &h->d_chirp))) return rc;
    if ((rc = bluestein_table(h, 8, &h->d_bconv))) return rc;
    if ((rc = bluestein_table(h, 9, &h->d_tw))) return rc;
  } else if (pxp::fft1d_pair_size(h->prec, (int)h->nx)) {
    // two CTAs of n/2 points: the n/2-point Stockham twiddles and
    // exp(-2 pi i k / n) for the split between the halves
    if ((rc = shared_table_n(h, 0, h->nx / 2, &h->d_tw))) return rc;
    if ((rc = shared_table_n(h, 4, h->nx, &h->d_chirp))) return rc;
  } else if ((rc = shared_table(h, 0, &h->d_tw))) {
    return rc;
  }
  if (pxp::fft1d_r16_enabled((int)h->nx) && (rc = shared_table(h, 4, &h->d_wn))) return rc;
  return alloc(h, &h->d_job, sizeof(pxp::Fft1dJob), "job descriptor");
}

// Transmission tables t (FP64) or t/N (FP32) from delta/beta planes.
int fft1d_set_trans(pxp_solver_s *h, const double *delta, const double *beta, int nplanes,
                    int first_step) {
  const unsigned n = h->nx;
  std::vector<cd> t((size_t)n * nplanes);
  const double k = h->prob.wavenumber, dz = h->prob.z.step;
  for (int p = 0; p < nplanes; ++p)
    for (unsigned i = 0; i < n; ++i) {
      size_t j = (size_t)p * n + i;
      cd v = transmission(k, beta[j], delta[j], dz);
      if (h->prec == pxp::kFP32) v = v / (double)n;
      t[j] = v;
    }
  free_dev(h->d_trans, h->stream);
  int rc;
  if ((rc = alloc(h, &h->d_trans, table_entry_bytes(h) * t.size(), "transmission table")))
    return rc;
  if ((rc = upload_table(h, h->d_trans, t.data(), (long long)t.size()))) return rc;
  h->trans_stride = nplanes > 1 ? n : 0;
  h->trans_step0 = first_step;
  h->material_set = true;
  return PXP_OK;
}

int fft1d_write_job(pxp_solver_s *h) {
  pxp::Fft1dJob j{};
  j.field = h->d_field;
  j.kern = h->d_kern;
  j.trans = h->d_trans;
  j.trans_stride = h->trans_stride;
  j.twiddle = h->d_tw;
  j.saves = h->d_saves;
  j.n = (int)h->nx;
  j.save_every = h->save_every;
  j.max_slots = h->max_slots;
  j.trans_step0 = h->trans_step0;
  j.flux = pxp::FluxSpec{h->d_flux_win, h->d_flux, h->flux_step0, h->flux_count};
  j.chirp = h->d_chirp;
  j.bconv = h->d_bconv;
  j.m = pxp::fft1d_bluestein_m((int)h->nx);
  j.wn = h->d_wn;
  h->job_fft = j;
  if (int rc_ = h2d(h, h->d_job, &j, sizeof(j))) return rc_;
  return PXP_OK;
}

// ---- CN --------------------------------------------------------------------
int cn_build_lu(pxp_solver_s *h, const double *delta, const double *beta);

int cn_set_planes(pxp_solver_s *h, const double *delta, const double *beta, int nsteps,
                  int first_step, bool two_planes_per_step) {
  // Device layout: 4 blocks [delta | beta | delta_prev | beta_prev], each
  // nsteps * n doubles; per-step stride n.
  const unsigned n = h->nx;
  const size_t per = (size_t)n * nsteps;
  std::vector<double> buf(4 * per);
  for (int s = 0; s < nsteps; ++s) {
    const size_t src0 = (size_t)(two_planes_per_step ? 2 * s : s) * n;
    const size_t src1 = (size_t)(two_planes_per_step ? 2 * s + 1 : s) * n;
    std::memcpy(&buf[0 * per + (size_t)s * n], delta + src0, sizeof(double) * n);
    std::memcpy(&buf[1 * per + (size_t)s * n], beta + src0, sizeof(double) * n);
    std::memcpy(&buf[2 * per + (size_t)s * n], delta + src1, sizeof(double) * n);
    std::memcpy(&buf[3 * per + (size_t)s * n], beta + src1, sizeof(double) * n);
  }
  free_dev(h->d_mat, h->stream);
  int rc;
  if ((rc = alloc(h, (void **)&h->d_mat, sizeof(double) * buf.size(), "material planes")))
    return rc;
  if (int rc_ = h2d(h, h->d_mat, buf.data(), sizeof(double) * buf.size())) return rc_;
  h->mat_block = (long long)per;
  h->mat_stride = nsteps > 1 ? n : 0;
  h->mat_step0 = first_step;
  h->material_set = true;
  // step-invariant matrix when the same plane serves every step
  h->cn_const = false;
  if (nsteps == 1 && pxp::cn_const_supported(h->prec, pxp::cn_padded_n((int)n))) {
    int rc2 = cn_build_lu(h, delta, beta);
    if (rc2) return rc2;
    h->cn_const = true;
  }
  return PXP_OK;
}

// ---- step-invariant matrices --------------------------------------------------
// Thomas factor tables of a tridiagonal matrix with diagonal `diag` and
// constant symmetric off-diagonal `sub` (include/thomasAlgorithm.tpp:2-32
// forward sweep): g_i = 1/den_i, h_i = -sub * g_i, see scan_solve.cuh.
void thomas_factor(const std::vector<cd> &diag, cd sub, std::vector<cd> &out_gh) {
  const size_t n = diag.size();
  out_gh.assign(2 * n, cd(0.0));
  cd den = diag[0];
  for (size_t i = 0; i < n; ++i) {
    if (i > 0) den = diag[i] - sub * (sub * out_gh[i - 1]);
    const cd g = cd(1.0) / den;
    out_gh[i] = g;
    out_gh[n + i] = -sub * g;
  }
}

// CrankNicholson matrix for a z-invariant medium (src/crancNicholson.cpp:
// 46-52 with F = G = H = 1, J = 0), evaluated with the reference's
// std::complex expressions.
int cn_build_lu(pxp_solver_s *h, const double *delta, const double *beta) {
  const unsigned n = h->nx;
  // the kernels solve np rows: rows n..np-1 pad the system (diagonal kCnPad)
  const unsigned np = (unsigned)pxp::cn_padded_n((int)n);
  const cd IMAG_UNIT(0.0, 1.0);
  const double dx = h->prob.x.step, dz = h->prob.z.step, k = h->prob.wavenumber;
  const double rho = dz / (k * dx * dx), r = k * dz;
  const double Hp = 1.0, Hm = 1.0, gval = 1.0, fval = 1.0;
  std::vector<cd> diag(np, cd(pxp::kCnPad, 0.0));
  for (unsigned i = 0; i < n; ++i)
    diag[i] = fval * 1.0 + 0.25 * (Hp + Hm) * gval * IMAG_UNIT * rho +
              0.5 * (beta[i] * r + IMAG_UNIT * delta[i] * r);
  const cd sub = -0.25 * IMAG_UNIT * rho * Hm * gval;
  std::vector<cd> gh;
  thomas_factor(diag, sub, gh);
  free_dev(h->d_lu, h->stream);
  int rc;
  if ((rc = alloc(h, &h->d_lu, sizeof(cd) * 2 * np, "factor tables"))) return rc;
  if (int rc_ = h2d(h, h->d_lu, gh.data(), sizeof(cd) * 2 * np)) return rc_;
  return PXP_OK;
}

// Length of each staged table of the ADI vacuum half steps: the FP64
// one-wave kernel's padded system length, or n where that kernel does not
// run n (the tables are then not read).
int adi_tab_len(unsigned n) {
  const int w = pxp::adi_wave_n((int)n);
  return w > 0 ? w : (int)n;
}

// ADI vacuum matrices of the x and y half steps (src/alternatingDirection
// Solver.cpp:38, :103 with beta = delta = 0): tables [gx | hx | gy | hy].
int adi_build_lu(pxp_solver_s *h) {
  const unsigned n = h->nx;
  const cd im(0.0, 1.0);
  const double dz = h->prob.z.step / 2.0, k = h->prob.wavenumber;
  const double dx = h->prob.x.step, dy = h->prob.y.step;
  const double beta = 0.0, delta = 0.0;
  std::vector<cd> dgx(n, 1.0 / dz + im / (k * dx * dx) + beta * k + im * delta * k);
  std::vector<cd> dgy(n, 1.0 / dz + im / (k * dy * dy + beta * k + im * delta * k));
  std::vector<cd> gx, gy;
  thomas_factor(dgx, -0.5 * im / (k * dx * dx), gx);
  thomas_factor(dgy, -0.5 * im / (k * dy * dy), gy);
  // [gx | hx | gy | hy] in natural order, then the x and y tables staged for
  // the FP64 one-wave kernel ([g | h | pf | pb] each, for its system length
  // nw; rows n .. nw-1 decoupled: g = 1, h = 0)
  const unsigned nw = (unsigned)adi_tab_len(n);
  std::vector<cd> tabs(4 * (size_t)n + 8 * (size_t)nw);
  std::copy(gx.begin(), gx.end(), tabs.begin());
  std::copy(gy.begin(), gy.end(), tabs.begin() + 2 * n);
  std::vector<cd> pad(2 * (size_t)nw);
  for (int half = 0; half < 2; ++half) {
    const std::vector<cd> &gv = half == 0 ? gx : gy;
    for (unsigned i = 0; i < nw; ++i) {
      pad[i] = i < n ? gv[i] : cd(1.0, 0.0);
      pad[nw + i] = i < n ? gv[n + i] : cd(0.0, 0.0);
    }
    const double *t = reinterpret_cast<const double *>(pad.data());
    if (!pxp::adi_const_staged_tables((int)nw, t, t + 2 * nw,
                                      reinterpret_cast<double *>(tabs.data() + 4 * n + 4 * half * nw),
                                      h->adi_tab_run[half]))
      h->adi_tab_run[half][0] = h->adi_tab_run[half][1] = 0;
  }
  free_dev(h->d_lu, h->stream);
  int rc;
  if ((rc = alloc(h, &h->d_lu, sizeof(cd) * tabs.size(), "factor tables"))) return rc;
  if (int rc_ = h2d(h, h->d_lu, tabs.data(), sizeof(cd) * tabs.size())) return rc_;
  return PXP_OK;
}

// ---- ADI -------------------------------------------------------------------
// getZ (src/paraxialSimulation.cpp:250-253)
double get_z(const pxp_solver_s *h, unsigned iz) { return h->prob.z.min + iz * h->prob.z.step; }

// ---- step graphs -------------------------------------------------------------
// Steps whose launches do not depend on the step index (vacuum planes, no
// save) are enqueued in blocks of kGraphSteps from a CUDA graph: the block's
// launches are captured once per handle and replayed, so the host pays one
// graph launch per block instead of two kernel launches per step, and the
// device runs the block's kernels back to back.  The signature lists every
// buffer and launch choice baked into the block; a change re-captures it.
// PXP_STEP_GRAPHS=0 turns the graphs off (every step launched directly).
constexpr int kGraphSteps = 32;

bool step_graphs_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("PXP_STEP_GRAPHS");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <typename F>
int replay_steps(pxp_solver_s *h, const std::vector<const void *> &sig, int blocks, F enqueue_block) {
  if (!h->graph || h->graph_sig != sig) {
    if (h->graph) cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return h->cuda_fail(e, "step graph capture");
    const int rc = enqueue_block();
    e = cudaStreamEndCapture(h->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return h->cuda_fail(e, "step graph capture");
    e = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      h->graph = nullptr;
      return h->cuda_fail(e, "step graph instantiation");
    }
    h->graph_sig = sig;
  }
  for (int b = 0; b < blocks; ++b) {
    const cudaError_t e = cudaGraphLaunch(h->graph, h->stream);
    if (e != cudaSuccess) return h->cuda_fail(e, "step graph launch");
  }
  return PXP_OK;
}

bool save_at(const pxp_solver_s *h, unsigned step) {
  return h->save_every > 0 && step % (unsigned)h->save_every == 0 &&
         (int)(step / (unsigned)h->save_every) - 1 < h->max_slots;
}

char *save_slot(const pxp_solver_s *h, unsigned step) {
  return (char *)h->d_saves + (size_t)(step / h->save_every - 1) * h->csize * h->save_pts;
}

// The step's full field is in the staging buffer: reduce it into its slot.
int save_downsample(pxp_solver_s *h, char *slot) {
  const cudaError_t e = pxp::launch_block_average(h->prec, h->d_save_stage, slot, (int)h->nx,
                                                  (int)h->save_n, h->stream);
  return e == cudaSuccess ? PXP_OK : h->cuda_fail(e, "saved-field downsampling");
}

// Spheres that can contain a point of the plane z: the oracle's and the
// kernel's test is ((dx^2 + dy^2) + dz^2) < R^2 with rounded operations, and
// the rounded sum of non-negative terms is never below dz^2, so a sphere
// with fl(dz^2) >= fl(R^2) is never hit and may be dropped (list order kept).
void active_spheres(const pxp_solver_s *h, double z, std::vector<pxp::Sphere> &out) {
  out.clear();
  for (const pxp_sphere &sp : h->spheres) {
    volatile double dz = z - sp.cz;
    volatile double dz2 = dz * dz;
    volatile double r2 = sp.radius * sp.radius;
    if (dz2 < r2) out.push_back({sp.cx, sp.cy, sp.cz, sp.radius, sp.delta, sp.beta});
  }
}

// Modules whose z range meets [zlo, zhi]; the others contain no point of
// those planes, so dropping them changes no material lookup.
unsigned long long csg_active(const pxp_solver_s *h, double zlo, double zhi) {
  unsigned long long m = 0;
  for (int i = 0; i < h->csg_nmodules; ++i)
    if (h->csg_zlo[i] <= zhi && h->csg_zhi[i] >= zlo) m |= 1ull << i;
  return m;
}

pxp::Csg csg_params(const pxp_solver_s *h, double zlo, double zhi) {
  pxp::Csg c{};
  if (!h->d_csg) return c;
  c.modules = (const pxp::CsgModule *)h->d_csg;
  c.parts = (const pxp::CsgPart *)(c.modules + h->csg_nmodules);
  c.shapes = (const pxp::CsgShape *)(c.parts + h->csg_nparts);
  c.nmodules = h->csg_nmodules;
  c.active = csg_active(h, std::min(zlo, zhi), std::max(zlo, zhi));
  return c;
}

// Device planes of a 3-D kind for step `step`, plane `which` (ADI: 0 = x half
// step, 1 = y half step): delta and beta, or null when no planes are set.
void planes3_at(const pxp_solver_s *h, unsigned step, int which, const double **delta,
                const double **beta) {
  *delta = *beta = nullptr;
  if (h->d_planes3 == nullptr) return;
  if (h->planes3_invariant) {
    *delta = h->d_planes3;
    *beta = h->d_planes3 + h->npts;
    return;
  }
  if (h->plane_count <= 0) return;
  const long long nplanes = (long long)h->plane_count * h->planes3_per;
  const long long p = ((long long)step - h->plane_first) * h->planes3_per + which;
  *delta = h->d_planes3 + p * h->npts;
  *beta = h->d_planes3 + (nplanes + p) * h->npts;
}

int adi_fill_spheres(pxp_solver_s *h, pxp::AdiHalf &a, double z) {
  a.csg = csg_params(h, z, z);
  std::vector<pxp::Sphere> act;
  active_spheres(h, z, act);
  a.nspheres = (int)act.size();
  if (a.nspheres <= pxp::kInlineSpheres) {
    for (int i = 0; i < a.nspheres; ++i) a.spheres[i] = act[i];
    a.spheres_all = nullptr;
  } else {
    // too many active spheres for the parameter block: the full list
    a.nspheres = (int)h->spheres.size();
    a.spheres_all = h->d_spheres;
  }
  return PXP_OK;
}

// One ADI step (x half, then y half) launched directly.
int adi_step(pxp_solver_s *h, unsigned step) {
  const pxp_problem &p = h->prob;
  const double dzh = p.z.step / 2.0;  // ADI::xImplicit (src/alternatingDirectionSolver.cpp:18)
  const double k = p.wavenumber;
  const double kdx2 = k * p.x.step * p.x.step, kdy2 = k * p.y.step * p.y.step;
  const long long n = h->nx;
  pxp::AdiHalf a{};
  a.n = (int)n;
  a.n_pad = pxp::adi_padded_n((int)n) != (int)n ? pxp::adi_padded_n((int)n) : 0;
  a.use_tbc = p.transparent_bc ? 1 : 0;
  a.inv_dzh = 1.0 / dzh;
  a.k = k;
  a.xmin = p.x.min;
  a.dx = p.x.step;
  a.ymin = p.y.min;
  a.dy = p.y.step;
  // x implicit: systems are rows (y), positions run along x (stride Ny)
  a.in = h->d_field;
  a.out = h->d_field2;
  a.save = nullptr;
  a.stride_pos = n;
  a.stride_sys = 1;
  a.y_implicit = 0;
  a.kd2_impl = kdx2;
  a.kd2_expl = kdy2;
  a.z = get_z(h, step);
  a.tab_c0 = h->adi_tab_run[0][0];
  a.tab_c1 = h->adi_tab_run[0][1];
  adi_fill_spheres(h, a, a.z);
  planes3_at(h, step, 0, &a.plane_delta, &a.plane_beta);
  const cd *lu = (const cd *)h->d_lu;
  cudaError_t e = (a.nspheres == 0 && !a.csg.active && !a.plane_delta && !a.use_tbc && lu)
                      ? pxp::launch_adi_half_const(h->prec, a, lu, lu + n, lu + 4 * n, h->stream)
                      : pxp::launch_adi_half(h->prec, a, h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "ADI x half step");
  // y implicit: systems are columns (x), positions run along y (stride 1)
  a.in = h->d_field2;
  a.out = h->d_field;
  char *slot = save_at(h, step) ? save_slot(h, step) : nullptr;
  a.save = slot && h->d_save_stage ? h->d_save_stage : slot;
  a.stride_pos = 1;
  a.stride_sys = n;
  a.y_implicit = 1;
  a.kd2_impl = kdy2;
  a.kd2_expl = kdx2;
  a.z = get_z(h, step) + dzh;
  a.tab_c0 = h->adi_tab_run[1][0];
  a.tab_c1 = h->adi_tab_run[1][1];
  adi_fill_spheres(h, a, a.z);
  planes3_at(h, step, 1, &a.plane_delta, &a.plane_beta);
  e = (a.nspheres == 0 && !a.csg.active && !a.plane_delta && !a.use_tbc && lu)
          ? pxp::launch_adi_half_const(h->prec, a, lu + 2 * n, lu + 3 * n,
                                       lu + 4 * n + 4 * adi_tab_len((unsigned)n), h->stream)
          : pxp::launch_adi_half(h->prec, a, h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "ADI y half step");
  if (slot && h->d_save_stage) return save_downsample(h, slot);
  return PXP_OK;
}

// Both halves of the step on the vacuum kernel and no save: the step's
// launches are then the same as any other such step's.
bool adi_plain_step(const pxp_solver_s *h, unsigned step, std::vector<pxp::Sphere> &tmp) {
  if (h->prob.transparent_bc || !h->d_lu || save_at(h, step) || h->plane_count > 0 ||
      h->planes3_invariant)
    return false;
  const double z = get_z(h, step);
  if (csg_active(h, z, z + h->prob.z.step / 2.0)) return false;
  active_spheres(h, z, tmp);
  if (!tmp.empty()) return false;
  active_spheres(h, z + h->prob.z.step / 2.0, tmp);
  return tmp.empty();
}

int adi_steps(pxp_solver_s *h, unsigned first, int nsteps) {
  std::vector<pxp::Sphere> tmp;
  const std::vector<const void *> sig = {h->d_field, h->d_field2, h->d_lu, (const void *)(size_t)1};
  for (int i = 0; i < nsteps;) {
    // a block is replayed only after a direct step of this call has set up
    // every launch's one-time state
    if (i > 0 && step_graphs_enabled() && nsteps - i >= kGraphSteps) {
      int run = 0;
      while (i + run < nsteps && adi_plain_step(h, first + (unsigned)(i + run), tmp)) ++run;
      const int blocks = run / kGraphSteps;
      if (blocks > 0) {
        const unsigned s0 = first + (unsigned)i;
        const int rc = replay_steps(h, sig, blocks, [&] {
          for (int j = 0; j < kGraphSteps; ++j)
            if (int r = adi_step(h, s0 + (unsigned)j)) return r;
          return (int)PXP_OK;
        });
        if (rc) return rc;
        i += blocks * kGraphSteps;
        continue;
      }
    }
    if (int rc = adi_step(h, first + (unsigned)i)) return rc;
    ++i;
  }
  return PXP_OK;
}

// ---- FFT 3-D ---------------------------------------------------------------
// Spheres that can contain any material sample of the step between planes z0
// and z1 (the end points and the refraction-integral points between them):
// the sphere's z extent, widened by a relative margin, must meet [z0, z1].
// Dropping the others is exact: a sphere that contains no sample point
// changes no first-hit lookup.
void slab_spheres(const pxp_solver_s *h, double z0, double z1, std::vector<pxp::Sphere> &out) {
  out.clear();
  const double lo = std::min(z0, z1), hi = std::max(z0, z1);
  const double margin = 1e-9 * (std::fabs(lo) + std::fabs(hi) + 1.0);
  for (const pxp_sphere &sp : h->spheres)
    if (sp.cz + sp.radius > lo - margin && sp.cz - sp.radius < hi + margin)
      out.push_back({sp.cx, sp.cy, sp.cz, sp.radius, sp.delta, sp.beta});
}

// Launch-variant autotuner of the FFTSolver3D passes.  The first solver with
// a given (device, precision, n) times every variant of each pass (x and y
// separately) on a zeroed scratch field -- launches replayed from a CUDA
// graph, so host-side launch set-up never counts -- then times whole steps
// (x and y passes interleaved) of every variant and of the two per-pass
// winners combined, and keeps the fastest step; every
// solver with that key runs the winners from its first step on, so a field
// never depends on when tuning happened (the variants' transforms round
// differently).  PXP_FFT3D_VARIANT=0..5 pins both passes' variant instead.
std::mutex g_tune_mutex;
std::map<std::tuple<int, int, unsigned>, int> g_fft3d_variant;

// PXP_TUNE_LOG=1: the tuners print each candidate's time to stderr.
bool tune_log() {
  static const bool on = [] {
    const char *e = std::getenv("PXP_TUNE_LOG");
    return e && e[0] == '1';
  }();
  return on;
}

// A tuned choice: the x pass's variant and the y pass's (modes 0, 2, 3).
int fft3d_variant_code(int vx, int vy) { return vx + 8 * vy; }
int fft3d_variant_of(int code, int mode) { return mode == 1 ? code % 8 : code / 8; }

int fft3d_variant(pxp_solver_s *h, const pxp::Fft3dPass &q0, const void *kx2, const void *tw16,
                  const void *wn, int *out) {
  if (const char *env = std::getenv("PXP_FFT3D_VARIANT")) {
    const int v = std::atoi(env);
    if (v >= 0 && v < pxp::kFft3dVariants) {
      *out = fft3d_variant_code(v, v);
      return PXP_OK;
    }
  }
  if (h->nx & (h->nx - 1)) {  // one kernel (Bluestein) for other sizes: nothing to tune
    *out = 0;
    return PXP_OK;
  }
  const auto key = std::make_tuple(h->prob.device, (int)h->prec, h->nx);
  std::lock_guard<std::mutex> lk(g_tune_mutex);
  auto it = g_fft3d_variant.find(key);
  if (it != g_fft3d_variant.end()) {
    *out = it->second;
    return PXP_OK;
  }
  const size_t bytes = h->csize * h->npts;
  void *scratch = nullptr;
  cudaError_t e = cudaMallocAsync(&scratch, bytes, h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "FFT3D tuning scratch");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  pxp::Fft3dPass q = q0;
  q.field = scratch;
  q.save = nullptr;
  q.nspheres = 0;
  q.spheres_all = nullptr;
  // the x pass (mode 1) and the y pass (mode 2) are separate launches with
  // the same field layout before and after, so each takes its own fastest
  // variant
  // Device time of `enqueue` (one launch or one step): four copies captured
  // in a CUDA graph, the graph launched once untimed and then three times
  // between events, the fastest kept -- no host-side launch set-up between
  // the kernels (steps are replayed from graphs as well), however short
  // they are.  A direct launch first sets up each kernel's one-time state.
  auto graph_time = [&](auto enqueue) -> float {
    float tmin = 1e30f;
    if (e != cudaSuccess) return tmin;
    if ((e = enqueue()) != cudaSuccess || (e = cudaStreamSynchronize(h->stream)) != cudaSuccess)
      return tmin;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaError_t ge = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
    if (ge == cudaSuccess) {
      cudaError_t ce = cudaSuccess;
      for (int k = 0; k < 4 && ce == cudaSuccess; ++k) ce = enqueue();
      ge = cudaStreamEndCapture(h->stream, &graph);
      if (ge == cudaSuccess) ge = ce;
    }
    if (ge == cudaSuccess) ge = cudaGraphInstantiate(&exec, graph, 0);
    if (ge == cudaSuccess) ge = cudaGraphLaunch(exec, h->stream);
    for (int rep = 0; rep < 3 && ge == cudaSuccess; ++rep) {
      cudaEventRecord(e0, h->stream);
      ge = cudaGraphLaunch(exec, h->stream);
      cudaEventRecord(e1, h->stream);
      if (ge == cudaSuccess) ge = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (ge == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
        tmin = std::min(tmin, ms / 4.f);
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (ge == cudaSuccess) return tmin;
    // no graph (capture refused): direct launches behind an untimed one
    cudaGetLastError();
    tmin = 1e30f;
    for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
      e = enqueue();
      cudaEventRecord(e0, h->stream);
      for (int k = 0; k < 3 && e == cudaSuccess; ++k) e = enqueue();
      cudaEventRecord(e1, h->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
        tmin = std::min(tmin, ms / 3.f);
    }
    return tmin;
  };
  int best_v[2] = {0, 0};
  float best[2] = {1e30f, 1e30f};
  if ((e = cudaMemsetAsync(scratch, 0, bytes, h->stream)) == cudaSuccess) {
    for (int v = 0; v < pxp::kFft3dVariants && e == cudaSuccess; ++v) {
      for (int pass = 0; pass < 2 && e == cudaSuccess; ++pass) {
        const int mode = pass == 0 ? 1 : 2;
        const float t = graph_time([&] {
          q.mode = mode;
          return pxp::launch_fft3d_pass(h->prec, q, v, (const double *)kx2, tw16, wn, h->stream);
        });
        if (tune_log())
          std::fprintf(stderr, "pxp fft3d tune n=%u prec=%d variant %d %s pass: %.2f us\n", h->nx,
                       (int)h->prec, v, mode == 1 ? "x" : "y", t * 1e3f);
        if (t < best[pass]) {
          best[pass] = t;
          best_v[pass] = v;
        }
      }
    }
  }
  // the per-pass winners against each variant for both passes, timed as
  // whole steps (x pass, y pass, interleaved as the solver runs them): a
  // pass timed in isolation meets the caches its own previous launch left
  std::vector<int> cands;
  for (int v = 0; v < pxp::kFft3dVariants; ++v) cands.push_back(fft3d_variant_code(v, v));
  if (best_v[0] != best_v[1]) cands.push_back(fft3d_variant_code(best_v[0], best_v[1]));
  int best_code = cands.back();
  float best_step = 1e30f;
  for (int code : cands) {
    if (e != cudaSuccess) break;
    const float t = graph_time([&] {
      q.mode = 1;
      cudaError_t r = pxp::launch_fft3d_pass(h->prec, q, fft3d_variant_of(code, 1),
                                             (const double *)kx2, tw16, wn, h->stream);
      q.mode = 2;
      if (r == cudaSuccess)
        r = pxp::launch_fft3d_pass(h->prec, q, fft3d_variant_of(code, 2), (const double *)kx2,
                                   tw16, wn, h->stream);
      return r;
    });
    if (tune_log())
      std::fprintf(stderr, "pxp fft3d tune n=%u prec=%d step x v%d + y v%d: %.2f us\n", h->nx,
                   (int)h->prec, fft3d_variant_of(code, 1), fft3d_variant_of(code, 2), t * 1e3f);
    if (t < best_step) {
      best_step = t;
      best_code = code;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(scratch, h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "FFT3D tuning");
  g_fft3d_variant[key] = best_code;
  *out = best_code;
  return PXP_OK;
}

// Launch-variant tuner of the 2-D step kernels: FFTSolver2D at 512..4096
// points (shared-memory Stockham kernel or register-resident radix-16
// kernel) and CrankNicholson's step-invariant path at 4096 rows (one CTA or
// a cluster of two).  As for FFTSolver3D, the first solver with a given
// (device, precision, kind, size) times every variant on a scratch copy of
// its own job (zeroed field; no saves, flux sums or per-step tables; 64
// steps a launch, three rounds of an untimed launch and a timed one, the
// fastest kept) and every
// solver with that key -- alone or in a batch -- runs the winner from its
// first step, so a field never depends on when tuning ran (the variants
// agree within the FP64 tolerance, not bit for bit).  PXP_FFT1D_R16=0|1 and
// PXP_CN_CLUSTER=0|1 pin the variant instead.
std::map<std::tuple<int, int, int, unsigned>, int> g_2d_variant;

bool cn_uses_const(const pxp_solver_s *h);

int variant_2d(pxp_solver_s *h, int *out) {
  *out = -1;
  const bool fft = h->prob.kind == PXP_FFT_SOLVER_2D;
  if (!fft && !(h->prob.kind == PXP_CRANK_NICHOLSON && cn_uses_const(h))) return PXP_OK;
  const int n = fft ? (int)h->nx : pxp::cn_padded_n((int)h->nx);
  const int nv = fft ? pxp::fft1d_variants(h->prec, n) : pxp::cn_const_variants(h->prec, n);
  if (nv < 2) return PXP_OK;
  if (const char *env = std::getenv(fft ? "PXP_FFT1D_R16" : "PXP_CN_CLUSTER")) {
    if (env[0] == '0' || env[0] == '1') {
      *out = env[0] - '0';
      return PXP_OK;
    }
  }
  const auto key = std::make_tuple(h->prob.device, (int)h->prec, (int)h->prob.kind, (unsigned)n);
  std::lock_guard<std::mutex> lk(g_tune_mutex);
  auto it = g_2d_variant.find(key);
  if (it != g_2d_variant.end()) {
    *out = it->second;
    return PXP_OK;
  }
  const size_t job_bytes = fft ? sizeof(pxp::Fft1dJob) : sizeof(pxp::CnJob);
  const size_t field_bytes = h->csize * (size_t)n;
  void *scratch = nullptr, *djob = nullptr;
  cudaError_t e = cudaMallocAsync(&scratch, field_bytes, h->stream);
  if (e == cudaSuccess) e = cudaMallocAsync(&djob, job_bytes, h->stream);
  if (e != cudaSuccess) {
    if (scratch) cudaFreeAsync(scratch, h->stream);
    return h->cuda_fail(e, "2-D kernel tuning scratch");
  }
  pxp::Fft1dJob jf = h->job_fft;
  pxp::CnJob jc = h->job_cn;
  if (fft) {
    jf.field = scratch;
    jf.saves = nullptr;
    jf.save_every = 0;
    jf.trans_stride = 0;
    jf.flux = pxp::FluxSpec{};
  } else {
    jc.field = scratch;
    jc.saves = nullptr;
    jc.save_every = 0;
    jc.flux = pxp::FluxSpec{};
  }
  e = cudaMemsetAsync(scratch, 0, field_bytes, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(djob, fft ? (const void *)&jf : (const void *)&jc, job_bytes,
                        cudaMemcpyHostToDevice, h->stream);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  int best_v = 0;
  float best = 1e30f;
  constexpr int kTuneSteps = 64;
  auto launch_v = [&](int v) {
    return fft ? pxp::launch_fft1d(h->prec, (const pxp::Fft1dJob *)djob, 1, n, 1, kTuneSteps,
                                   h->stream, false, v)
               : pxp::launch_cn_const(h->prec, (const pxp::CnJob *)djob, 1, n, 1, kTuneSteps,
                                      h->stream, false, v);
  };
  for (int v = 0; v < nv && e == cudaSuccess; ++v) {
    float tmin = 1e30f;
    for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
      e = launch_v(v);  // untimed: the device is busy while the timed launch is prepared
      cudaEventRecord(e0, h->stream);
      if (e == cudaSuccess) e = launch_v(v);
      cudaEventRecord(e1, h->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
        tmin = std::min(tmin, ms);
    }
    if (tmin < best) {
      best = tmin;
      best_v = v;
    }
  }
  // the job descriptor must stay valid until the launches that read it ran
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFreeAsync(djob, h->stream);
  cudaFreeAsync(scratch, h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "2-D kernel tuning");
  g_2d_variant[key] = best_v;
  *out = best_v;
  return PXP_OK;
}

int fft3d_steps(pxp_solver_s *h, unsigned first, int nsteps) {
  const pxp_problem &p = h->prob;
  const int n = (int)h->nx;
  pxp::Fft3dPass q{};
  q.field = h->d_field;
  q.twiddle = h->d_tw;
  q.chirp = h->d_chirp;
  q.bconv = h->d_bconv;
  q.m = pxp::fft1d_bluestein_m(n);
  q.n = n;
  q.a = 0.5 * p.z.step / p.wavenumber;  // FFTSolver3D::kernel (src/fftSolver3D.cpp:24-30)
  q.two_pi = 2.0 * PI;
  q.stepn_x = p.x.step * n;
  q.stepn_y = p.y.step * n;
  q.k = p.wavenumber;
  q.dz = p.z.step;
  q.xmin = p.x.min;
  q.dx = p.x.step;
  q.ymin = p.y.min;
  q.dy = p.y.step;
  q.norm = (double)((unsigned)n * (unsigned)n);
  if (p.absorber_damping > 0.0) {  // FFTSolver3D::absorbingBC (src/fftSolver3D.cpp:327-349)
    q.thick_x = (int)(unsigned)(p.absorber_width / p.x.step + 1);
    q.thick_y = (int)(unsigned)(p.absorber_width / p.y.step + 1);
    q.inv_damp_x = p.x.step / p.absorber_damping;
    q.inv_damp_y = p.y.step / p.absorber_damping;
  }
  void *kx2 = nullptr, *tw16 = nullptr, *wn = nullptr;
  if (int rc = shared_table(h, 2, &kx2)) return rc;
  if (!(n & (n - 1))) {  // the power-of-two variants' twiddle tables
    if (int rc = shared_table(h, 3, &tw16)) return rc;
    if (int rc = shared_table(h, 4, &wn)) return rc;
    void *twl = nullptr;
    if (int rc = shared_table(h, 11, &twl)) return rc;
    q.tw_lines = twl;
  }
  // the propagator's x and y factor tables (FP32 always; FP64 unless
  // PXP_FFT3D_JOINT_PROP=1 asks for the reference's joint argument)
  const char *joint = std::getenv("PXP_FFT3D_JOINT_PROP");
  if (h->prec == pxp::kFP32 || !(joint && joint[0] == '1')) {
    void *px = nullptr, *py = nullptr;
    if (int rc = prop3_table(h, 0, &px)) return rc;
    if (int rc = prop3_table(h, 1, &py)) return rc;
    q.prop_x = px;
    q.prop_y = py;
  }
  int variant = 0;
  if (int rc = fft3d_variant(h, q, kx2, tw16, wn, &variant)) return rc;
  cudaError_t e;
  q.mode = 0;  // forward transform along y of the real-space field
  if ((e = pxp::launch_fft3d_pass(h->prec, q, fft3d_variant_of(variant, q.mode), (const double *)kx2, tw16, wn, h->stream)) != cudaSuccess)
    return h->cuda_fail(e, "FFT3D forward y pass");
  std::vector<pxp::Sphere> act;
  // step i of this call: x pass, then the y pass (mode 3 on the last step
  // leaves the field in real space)
  auto one_step = [&](int i) -> int {
    const unsigned step = first + (unsigned)i;
    q.mode = 1;
    q.save = nullptr;
    if ((e = pxp::launch_fft3d_pass(h->prec, q, fft3d_variant_of(variant, q.mode), (const double *)kx2, tw16, wn, h->stream)) !=
        cudaSuccess)
      return h->cuda_fail(e, "FFT3D x pass");
    q.mode = (i == nsteps - 1) ? 3 : 2;
    q.z1 = get_z(h, step);
    q.z0 = get_z(h, step - 1);
    slab_spheres(h, q.z0, q.z1, act);
    q.csg = csg_params(h, q.z0, q.z1);
    planes3_at(h, step, 0, &q.plane_delta, &q.plane_beta);
    q.nspheres = (int)act.size();
    if (q.nspheres <= pxp::kInlineSpheres) {
      for (int j = 0; j < q.nspheres; ++j) q.spheres[j] = act[j];
      q.spheres_all = nullptr;
    } else {
      q.nspheres = (int)h->spheres.size();
      q.spheres_all = h->d_spheres;
    }
    char *slot = save_at(h, step) ? save_slot(h, step) : nullptr;
    q.save = slot && h->d_save_stage ? h->d_save_stage : slot;
    if ((e = pxp::launch_fft3d_pass(h->prec, q, fft3d_variant_of(variant, q.mode), (const double *)kx2, tw16, wn, h->stream)) !=
        cudaSuccess)
      return h->cuda_fail(e, "FFT3D y pass");
    if (slot && h->d_save_stage) return save_downsample(h, slot);
    return PXP_OK;
  };
  // no sphere in the step's slab, no save, not the last step of the call:
  // the step's launches are the same as any other such step's (the slab's z
  // planes are read only for spheres)
  auto plain = [&](int i) {
    const unsigned step = first + (unsigned)i;
    if (i == nsteps - 1 || save_at(h, step) || h->plane_count > 0 || h->planes3_invariant)
      return false;
    slab_spheres(h, get_z(h, step - 1), get_z(h, step), act);
    return act.empty() && !csg_active(h, std::min(get_z(h, step - 1), get_z(h, step)),
                                      std::max(get_z(h, step - 1), get_z(h, step)));
  };
  const std::vector<const void *> sig = {h->d_field, h->d_tw, kx2, tw16, wn,
                                         (const void *)(size_t)(16 + variant)};
  for (int i = 0; i < nsteps;) {
    if (i > 0 && step_graphs_enabled() && nsteps - i > kGraphSteps) {
      int run = 0;
      while (i + run < nsteps && plain(i + run)) ++run;
      const int blocks = run / kGraphSteps;
      if (blocks > 0) {
        const int i0 = i;
        const int rc = replay_steps(h, sig, blocks, [&] {
          for (int j = 0; j < kGraphSteps; ++j)
            if (int r = one_step(i0 + j)) return r;
          return (int)PXP_OK;
        });
        if (rc) return rc;
        i += blocks * kGraphSteps;
        continue;
      }
    }
    if (int rc = one_step(i)) return rc;
    ++i;
  }
  return PXP_OK;
}

int cn_write_job(pxp_solver_s *h) {
  pxp::CnJob j{};
  const unsigned n = h->nx;
  const double dx = h->prob.x.step, dz = h->prob.z.step, k = h->prob.wavenumber;
  j.field = h->d_field;
  j.delta = h->d_mat;
  j.beta = h->d_mat + h->mat_block;
  j.delta_prev = h->d_mat + 2 * h->mat_block;
  j.beta_prev = h->d_mat + 3 * h->mat_block;
  j.mat_stride = h->mat_stride;
  j.saves = h->d_saves;
  j.rho = dz / (k * dx * dx);  // CrankNicholson::solveStep (src/crancNicholson.cpp:25-26)
  j.r = k * dz;
  j.n = pxp::cn_padded_n((int)n);
  j.n_real = (int)n;
  j.save_every = h->save_every;
  j.max_slots = h->max_slots;
  j.mat_step0 = h->mat_step0;
  j.transparent = h->prob.transparent_bc ? 1 : 0;
  j.lu_g = h->d_lu;
  j.lu_h = h->d_lu ? (const void *)((const cd *)h->d_lu + pxp::cn_padded_n((int)n)) : nullptr;
  j.flux = pxp::FluxSpec{h->d_flux_win, h->d_flux, h->flux_step0, h->flux_count};
  h->job_cn = j;
  if (int rc_ = h2d(h, h->d_job, &j, sizeof(j))) return rc_;
  return PXP_OK;
}

}  // namespace

extern "C" {

unsigned pxp_node_count(double mn, double mx, double step) {
  return (unsigned)((mx - mn) / step + 1.0);
}

const char *pxp_status_string(int status) {
  switch (status) {
    case PXP_OK: return "ok";
    case PXP_ERR_INVALID: return "invalid argument";
    case PXP_ERR_NOMEM: return "out of memory";
    case PXP_ERR_CUDA: return "CUDA error";
    case PXP_ERR_ABORTED: return "aborted";
    case PXP_ERR_BUDGET: return "step or wait budget exceeded";
    case PXP_ERR_NOT_READY: return "not ready";
    case PXP_ERR_UNSUPPORTED: return "unsupported size or precision";
    default: return "unknown status";
  }
}

const char *pxp_build_info(void) { return "paxpro_b200 sm_100a"; }

int pxp_last_error(pxp_solver s, char *buf, size_t len) {
  if (buf == nullptr || len == 0) return PXP_ERR_INVALID;
  std::string m;
  if (s) {
    m = s->err;
  } else {
    std::lock_guard<std::mutex> lk(g_err_mutex);
    m = g_last_error;
  }
  std::snprintf(buf, len, "%s", m.c_str());
  return PXP_OK;
}

int pxp_solver_create(const pxp_problem *problem, pxp_solver *out) {
  if (problem == nullptr || out == nullptr) {
    set_global_error("pxp_solver_create: null argument");
    return PXP_ERR_INVALID;
  }
  *out = nullptr;
  pxp_solver_s *h = new (std::nothrow) pxp_solver_s();
  if (h == nullptr) return PXP_ERR_NOMEM;
  h->prob = *problem;
  const pxp_problem &p = h->prob;
  auto bad = [&](const std::string &m) {
    set_global_error(m);
    delete h;
    return PXP_ERR_INVALID;
  };
  if (p.kind < PXP_FFT_SOLVER_2D || p.kind > PXP_ADI) return bad("unknown solver kind");
  if (p.precision != PXP_FP64 && p.precision != PXP_FP32) return bad("unknown precision");
  if (!(p.x.step > 0.0) || !(p.z.step > 0.0) || !(p.wavenumber > 0.0))
    return bad("discretisation steps and wavenumber must be positive");
  const bool three_d = p.kind == PXP_FFT_SOLVER_3D || p.kind == PXP_ADI;
  if (three_d && !(p.y.step > 0.0)) return bad("vertical step must be positive");
  h->nx = pxp_node_count(p.x.min, p.x.max, p.x.step);
  h->nz = pxp_node_count(p.z.min, p.z.max, p.z.step);
  h->ny = three_d ? h->nx : 1;  // Solver3D::setSimulator forces Ny = Nx (src/solver3D.cpp:24)
  h->npts = (long long)h->nx * h->ny;
  {
    // transverse downsampling of saved fields: Solver3D keeps Nx/ratio x
    // Nx/ratio block averages (src/solver3D.cpp:26, 36, 94-112); Solver2D
    // filters with the VISA low-pass filter (src/solver2D.cpp:34-39), which
    // this build does not provide
    const unsigned r = p.x.downsampling_ratio > 1 ? p.x.downsampling_ratio : 1;
    if (r > 1 && !three_d) {
      set_global_error("transverse downsampling_ratio > 1 of the 2-D solvers (a VISA low-pass "
                       "filter in the reference) is not provided: use 1");
      delete h;
      return PXP_ERR_UNSUPPORTED;
    }
    h->save_n = h->nx / r;
    if (h->save_n == 0) return bad("downsampling_ratio larger than the transverse node count");
    h->save_pts = three_d ? (long long)h->save_n * h->save_n : h->npts;
  }
  h->prec = p.precision == PXP_FP64 ? pxp::kFP64 : pxp::kFP32;
  h->csize = h->prec == pxp::kFP64 ? 16 : 8;
  if (h->nx < 4 || h->nz < 2) return bad("grid too small (need Nx >= 4, Nz >= 2)");
  bool supported = false;
  switch (p.kind) {
    case PXP_FFT_SOLVER_2D: supported = pxp::fft1d_supported(h->prec, (int)h->nx); break;
    case PXP_CRANK_NICHOLSON:
      // a grid that is padded to the kernel's row count takes Dirichlet ends
      // only; 8192 and 16384 rows beyond the general kernel's size run the
      // step-invariant path on a cluster (z-invariant medium, Dirichlet ends:
      // checked when stepping)
      supported = (pxp::cn_supported(h->prec, (int)h->nx) ||
                   (!p.transparent_bc &&
                    pxp::cn_const_supported(h->prec, pxp::cn_padded_n((int)h->nx)))) &&
                  (!p.transparent_bc || pxp::cn_padded_n((int)h->nx) == (int)h->nx);
      break;
    case PXP_ADI:
      // other sizes run padded on the general kernel
      supported = pxp::adi_supported(h->prec, (int)h->nx) ||
                  pxp::adi_padded_supported(h->prec, (int)h->nx);
      break;
    case PXP_FFT_SOLVER_3D: supported = pxp::fft3d_supported(h->prec, (int)h->nx); break;
    default: supported = false;
  }
  if (!supported) {
    set_global_error("solver kind / size / precision not supported by this build (Nx=" +
                     std::to_string(h->nx) + ")");
    delete h;
    return PXP_ERR_UNSUPPORTED;
  }
  cudaError_t e = cudaSetDevice(p.device);
  if (e == cudaSuccess) retain_pool(p.device);
  if (e == cudaSuccess) e = cudaStreamCreate(&h->stream);
  if (e != cudaSuccess) {
    set_global_error(std::string("CUDA initialisation: ") + cudaGetErrorString(e));
    delete h;
    return PXP_ERR_CUDA;
  }
  h->timeouts_seen = pxp::wait_timeouts(h->stream);
  int rc = PXP_OK;
  auto cleanup_fail = [&](int code) {
    std::string m = h->err;
    pxp_solver_destroy(h);
    set_global_error(m);
    return code;
  };
  if ((rc = alloc(h, &h->d_field, h->csize * h->npts, "field"))) return cleanup_fail(rc);
  PXP_TRY_CUDA(h, cudaMemset(h->d_field, 0, h->csize * h->npts));
  h->save_every = p.save_every > 0 ? p.save_every : 0;
  if (h->save_every) {
    h->max_slots = (int)((h->nz - 1) / (unsigned)h->save_every);
    if (h->max_slots > 0 &&
        (rc = alloc(h, &h->d_saves, h->csize * h->save_pts * (size_t)h->max_slots, "save slots")))
      return cleanup_fail(rc);
    if (h->max_slots > 0 && h->save_pts != h->npts &&
        (rc = alloc(h, &h->d_save_stage, h->csize * h->npts, "save staging")))
      return cleanup_fail(rc);
  }
  std::vector<double> zeros(h->npts, 0.0);
  switch (p.kind) {
    case PXP_FFT_SOLVER_2D:
      if ((rc = fft1d_setup(h))) return cleanup_fail(rc);
      if ((rc = fft1d_set_trans(h, zeros.data(), zeros.data(), 1, 1))) return cleanup_fail(rc);
      if ((rc = fft1d_write_job(h))) return cleanup_fail(rc);
      break;
    case PXP_CRANK_NICHOLSON:
      if ((rc = alloc(h, &h->d_job, sizeof(pxp::CnJob), "job descriptor"))) return cleanup_fail(rc);
      if ((rc = cn_set_planes(h, zeros.data(), zeros.data(), 1, 1, false))) return cleanup_fail(rc);
      if ((rc = cn_write_job(h))) return cleanup_fail(rc);
      break;
    case PXP_ADI:
      if ((rc = alloc(h, &h->d_field2, h->csize * h->npts, "second field buffer")))
        return cleanup_fail(rc);
      // vacuum factor tables for the step-invariant kernels (grids those run)
      // the vacuum fast path: powers of two in both precisions, any size the
      // FP64 one-wave kernel takes
      if (pxp::adi_supported(h->prec, (int)h->nx) ||
          (h->prec == pxp::kFP64 && pxp::adi_wave_n((int)h->nx) > 0))
        if ((rc = adi_build_lu(h))) return cleanup_fail(rc);
      break;
    case PXP_FFT_SOLVER_3D:
      if (h->nx & (h->nx - 1)) {
        // not a power of two: the Bluestein tables of the line transforms
        if ((rc = bluestein_table(h, 7, &h->d_chirp))) return cleanup_fail(rc);
        if ((rc = bluestein_table(h, 8, &h->d_bconv))) return cleanup_fail(rc);
        if ((rc = bluestein_table(h, 9, &h->d_tw))) return cleanup_fail(rc);
      } else if ((rc = shared_table(h, 0, &h->d_tw))) {
        return cleanup_fail(rc);
      }
      break;
  }
  *out = h;
  return PXP_OK;
}

int pxp_solver_destroy(pxp_solver h) {
  if (h == nullptr) return PXP_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  h->graph = nullptr;
  free_dev(h->d_field, h->stream);
  free_dev(h->d_saves, h->stream);
  free_dev(h->d_save_stage, h->stream);
  h->d_kern = nullptr;  // shared table, not owned
  free_dev(h->d_trans, h->stream);
  h->d_tw = nullptr;  // shared table, not owned
  h->d_wn = nullptr;  // shared table, not owned
  free_dev(h->d_mat, h->stream);
  free_dev(h->d_planes3, h->stream);
  free_dev(h->d_job, h->stream);
  free_dev(h->d_field2, h->stream);
  free_dev(h->d_spheres, h->stream);
  free_dev(h->d_csg, h->stream);
  free_dev(h->d_lu, h->stream);
  free_dev(h->d_ref, h->stream);
  free_dev(h->d_flux_win, h->stream);
  free_dev(h->d_flux, h->stream);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return PXP_OK;
}

static int rewrite_job(pxp_solver_s *h) {
  switch (h->prob.kind) {
    case PXP_FFT_SOLVER_2D: return fft1d_write_job(h);
    case PXP_CRANK_NICHOLSON: return cn_write_job(h);
    default: return PXP_OK;
  }
}

// Copy nplanes sampled planes of a 3-D kind to the device ([delta planes |
// beta planes]); the planes replace a sphere or CSG material.
static int store_planes3(pxp_solver_s *h, const double *delta, const double *beta, size_t nplanes) {
  const size_t need = 2 * nplanes * (size_t)h->npts;
  if (need > h->planes3_cap) {
    free_dev(h->d_planes3, h->stream);
    h->dev_bytes -= sizeof(double) * h->planes3_cap;
    h->planes3_cap = 0;
    if (int rc = alloc(h, (void **)&h->d_planes3, sizeof(double) * need, "3-D material planes"))
      return rc;
    h->planes3_cap = need;
  }
  const size_t half = nplanes * (size_t)h->npts;
  PXP_TRY_CUDA(h, cudaMemcpyAsync(h->d_planes3, delta, sizeof(double) * half,
                                  cudaMemcpyHostToDevice, h->stream));
  PXP_TRY_CUDA(h, cudaMemcpyAsync(h->d_planes3 + half, beta, sizeof(double) * half,
                                  cudaMemcpyHostToDevice, h->stream));
  PXP_TRY_CUDA(h, cudaStreamSynchronize(h->stream));
  h->spheres.clear();
  free_dev(h->d_spheres, h->stream);
  free_dev(h->d_csg, h->stream);
  h->csg_nmodules = h->csg_nparts = 0;
  h->csg_zlo.clear();
  h->csg_zhi.clear();
  h->material_set = true;
  return PXP_OK;
}

int pxp_set_material_table(pxp_solver h, const double *delta, const double *beta, size_t n) {
  if (h == nullptr || delta == nullptr || beta == nullptr) return PXP_ERR_INVALID;
  if (n != (size_t)h->npts)
    return h->fail(PXP_ERR_INVALID, "material table length " + std::to_string(n) +
                                        " != grid points " + std::to_string(h->npts));
  PXP_TRY_CUDA(h, cudaStreamSynchronize(h->stream));
  int rc;
  switch (h->prob.kind) {
    case PXP_FFT_SOLVER_2D:
      if ((rc = fft1d_set_trans(h, delta, beta, 1, 1))) return rc;
      break;
    case PXP_CRANK_NICHOLSON:
      if ((rc = cn_set_planes(h, delta, beta, 1, 1, false))) return rc;
      break;
    case PXP_FFT_SOLVER_3D:
    case PXP_ADI:
      // z-invariant: the sampled plane serves every step and half step
      // (FFTSolver3D's z0 and z1 values agree, so no refraction integral)
      if ((rc = store_planes3(h, delta, beta, 1))) return rc;
      h->planes3_invariant = true;
      h->planes3_per = 1;
      h->plane_count = 0;
      return PXP_OK;
    default:
      return h->fail(PXP_ERR_UNSUPPORTED, "material tables not supported for this kind");
  }
  h->h_delta.assign(delta, delta + n);
  h->h_beta.assign(beta, beta + n);
  h->plane_count = 0;
  return rewrite_job(h);
}

int pxp_set_material_planes(pxp_solver h, const double *delta, const double *beta,
                            int first_step, int nsteps) {
  if (h == nullptr || delta == nullptr || beta == nullptr || nsteps <= 0 || first_step < 1)
    return PXP_ERR_INVALID;
  PXP_TRY_CUDA(h, cudaStreamSynchronize(h->stream));
  int rc;
  switch (h->prob.kind) {
    case PXP_FFT_SOLVER_2D:
      if ((rc = fft1d_set_trans(h, delta, beta, nsteps, first_step))) return rc;
      if (nsteps == 1) h->trans_stride = 0;
      break;
    case PXP_CRANK_NICHOLSON:
      if ((rc = cn_set_planes(h, delta, beta, nsteps, first_step, true))) return rc;
      break;
    case PXP_FFT_SOLVER_3D:
    case PXP_ADI: {
      const int per = h->prob.kind == PXP_ADI ? 2 : 1;
      if ((rc = store_planes3(h, delta, beta, (size_t)nsteps * per))) return rc;
      h->planes3_per = per;
      h->planes3_invariant = false;
      h->plane_first = first_step;
      h->plane_count = nsteps;
      return PXP_OK;
    }
    default:
      return h->fail(PXP_ERR_UNSUPPORTED, "material planes not supported for this kind");
  }
  h->plane_first = first_step;
  h->plane_count = nsteps;
  return rewrite_job(h);
}

int pxp_set_material_spheres(pxp_solver h, const pxp_sphere *spheres, int n) {
  if (h == nullptr || (n > 0 && spheres == nullptr) || n < 0) return PXP_ERR_INVALID;
  if (h->prob.kind != PXP_ADI && h->prob.kind != PXP_FFT_SOLVER_3D)
    return h->fail(PXP_ERR_UNSUPPORTED, "sphere materials apply to the 3-D kinds");
  PXP_TRY_CUDA(h, cudaStreamSynchronize(h->stream));
  h->plane_count = 0;  // a sphere list replaces sampled planes
  h->planes3_invariant = false;
  h->spheres.assign(spheres, spheres + n);
  free_dev(h->d_spheres, h->stream);
  free_dev(h->d_csg, h->stream);
  h->csg_nmodules = h->csg_nparts = 0;
  h->csg_zlo.clear();
  h->csg_zhi.clear();
  if (n > 0) {
    std::vector<pxp::Sphere> dev(n);
    for (int i = 0; i < n; ++i)
      dev[i] = {spheres[i].cx, spheres[i].cy, spheres[i].cz, spheres[i].radius, spheres[i].delta,
                spheres[i].beta};
    int rc;
    if ((rc = alloc(h, (void **)&h->d_spheres, sizeof(pxp::Sphere) * n, "sphere list"))) return rc;
    if (int rc_ = h2d(h, h->d_spheres, dev.data(), sizeof(pxp::Sphere) * n)) return rc_;
  }
  h->material_set = true;
  return PXP_OK;
}

namespace {

// World-space z range of a shape's local bounding box (the shape's matrix
// maps world to local: local = T * world, so world = T^-1 * local).  Returns
// false when T is not an invertible affine map (no range then: always on).
bool shape_z_range(const pxp_csg_shape &sh, double &lo, double &hi) {
  const double *T = sh.transform;
  if (T[12] != 0.0 || T[13] != 0.0 || T[14] != 0.0 || T[15] != 1.0) return false;
  const double a = T[0], b = T[1], c = T[2], d = T[4], e = T[5], f = T[6], g = T[8], h = T[9], i = T[10];
  const double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
  if (!(std::fabs(det) > 1e-300) || !std::isfinite(det)) return false;
  // row 2 of A^-1 (gives world z): (d h - e g, b g - a h, a e - b d) / det
  const double r0 = (d * h - e * g) / det, r1 = (b * g - a * h) / det, r2 = (a * e - b * d) / det;
  double ex, ey, ez;
  if (sh.kind == PXP_SHAPE_SPHERE) {
    ex = ey = ez = sh.size[0];
  } else if (sh.kind == PXP_SHAPE_BOX) {
    ex = sh.size[0] / 2; ey = sh.size[1] / 2; ez = sh.size[2] / 2;
  } else {
    ex = ey = std::max(std::fabs(sh.size[1]), std::fabs(sh.size[2]));
    ez = sh.size[0] / 2;
  }
  lo = 1e300;
  hi = -1e300;
  for (int k = 0; k < 8; ++k) {
    const double lx = (k & 1 ? ex : -ex) - T[3], ly = (k & 2 ? ey : -ey) - T[7],
                 lz = (k & 4 ? ez : -ez) - T[11];
    const double wz = r0 * lx + r1 * ly + r2 * lz;
    lo = std::min(lo, wz);
    hi = std::max(hi, wz);
  }
  const double margin = 1e-9 * (std::fabs(lo) + std::fabs(hi) + 1.0) + 1e-6;
  lo -= margin;
  hi += margin;
  return std::isfinite(lo) && std::isfinite(hi);
}

}  // namespace

int pxp_set_material_csg(pxp_solver h, const pxp_csg_module *modules, int nmodules,
                         const pxp_csg_part *parts, int nparts, const pxp_csg_shape *shapes, int nshapes) {
  if (h == nullptr || nmodules < 0 || nparts < 0 || nshapes < 0 ||
      (nmodules > 0 && modules == nullptr) || (nparts > 0 && parts == nullptr) ||
      (nshapes > 0 && shapes == nullptr))
    return PXP_ERR_INVALID;
  if (h->prob.kind != PXP_ADI && h->prob.kind != PXP_FFT_SOLVER_3D)
    return h->fail(PXP_ERR_UNSUPPORTED, "CSG materials apply to the 3-D kinds");
  if (nmodules > 64) return h->fail(PXP_ERR_UNSUPPORTED, "at most 64 CSG modules");
  for (int m = 0; m < nmodules; ++m)
    if (modules[m].first_part < 0 || modules[m].num_parts < 0 ||
        modules[m].first_part + modules[m].num_parts > nparts)
      return h->fail(PXP_ERR_INVALID, "CSG module " + std::to_string(m) + ": parts out of range");
  for (int p = 0; p < nparts; ++p)
    if (parts[p].first_shape < 0 || parts[p].num_shapes < 0 ||
        parts[p].first_shape + parts[p].num_shapes > nshapes ||
        (parts[p].operation != PXP_CSG_UNION && parts[p].operation != PXP_CSG_DIFFERENCE))
      return h->fail(PXP_ERR_INVALID, "CSG part " + std::to_string(p) + ": bad shapes or operation");
  for (int k = 0; k < nshapes; ++k)
    if (shapes[k].kind < PXP_SHAPE_SPHERE || shapes[k].kind > PXP_SHAPE_CYLINDER ||
        (shapes[k].operation != PXP_CSG_UNION && shapes[k].operation != PXP_CSG_DIFFERENCE))
      return h->fail(PXP_ERR_INVALID, "CSG shape " + std::to_string(k) + ": bad kind or operation");
  PXP_TRY_CUDA(h, cudaStreamSynchronize(h->stream));
  h->plane_count = 0;  // a CSG material replaces sampled planes
  h->planes3_invariant = false;
  // z range per module: the union of its parts' union shapes' ranges (a
  // difference shape only removes; a point outside every union shape of a
  // module's parts is claimed by none of them)
  std::vector<double> zlo(nmodules, 1e300), zhi(nmodules, -1e300);
  for (int m = 0; m < nmodules; ++m)
    for (int p = modules[m].first_part; p < modules[m].first_part + modules[m].num_parts; ++p)
      for (int k = parts[p].first_shape; k < parts[p].first_shape + parts[p].num_shapes; ++k) {
        if (shapes[k].operation != PXP_CSG_UNION) continue;
        double lo, hi;
        if (!shape_z_range(shapes[k], lo, hi)) {
          lo = -1e300;
          hi = 1e300;
        }
        zlo[m] = std::min(zlo[m], lo);
        zhi[m] = std::max(zhi[m], hi);
      }
  std::vector<char> buf(sizeof(pxp::CsgModule) * nmodules + sizeof(pxp::CsgPart) * nparts +
                        sizeof(pxp::CsgShape) * nshapes);
  pxp::CsgModule *dm = (pxp::CsgModule *)buf.data();
  pxp::CsgPart *dp = (pxp::CsgPart *)(dm + nmodules);
  pxp::CsgShape *ds = (pxp::CsgShape *)(dp + nparts);
  for (int m = 0; m < nmodules; ++m) dm[m] = {modules[m].first_part, modules[m].num_parts};
  for (int p = 0; p < nparts; ++p)
    dp[p] = {parts[p].delta, parts[p].beta, parts[p].operation, parts[p].first_shape, parts[p].num_shapes};
  for (int k = 0; k < nshapes; ++k) {
    pxp::CsgShape c{};
    for (int j = 0; j < 12; ++j) c.m[j] = shapes[k].transform[j];
    for (int j = 0; j < 3; ++j) c.size[j] = shapes[k].size[j];
    c.kind = shapes[k].kind;
    c.op = shapes[k].operation;
    ds[k] = c;
  }
  free_dev(h->d_csg, h->stream);
  h->csg_nmodules = h->csg_nparts = 0;
  if (!buf.empty()) {
    int rc;
    if ((rc = alloc(h, &h->d_csg, buf.size(), "CSG material"))) return rc;
    if ((rc = h2d(h, h->d_csg, buf.data(), buf.size()))) return rc;
  }
  h->csg_nmodules = nmodules;
  h->csg_nparts = nparts;
  h->csg_zlo = zlo;
  h->csg_zhi = zhi;
  // a CSG material replaces a sphere list
  h->spheres.clear();
  free_dev(h->d_spheres, h->stream);
  h->material_set = true;
  return PXP_OK;
}

static int upload_field(pxp_solver_s *h, void *dst, const double *src) {
  if (h->prec == pxp::kFP64) {
    PXP_TRY_CUDA(h, cudaMemcpyAsync(dst, src, 16 * h->npts, cudaMemcpyHostToDevice, h->stream));
  } else {
    std::vector<float> tmp(2 * h->npts);
    for (long long i = 0; i < 2 * h->npts; ++i) tmp[i] = (float)src[i];
    PXP_TRY_CUDA(h, cudaMemcpyAsync(dst, tmp.data(), 8 * h->npts, cudaMemcpyHostToDevice, h->stream));
    PXP_TRY_CUDA(h, cudaStreamSynchronize(h->stream));
  }
  return PXP_OK;
}

// A kernel of this device gave up a bounded wait since the handle was made:
// its results are not to be trusted.
static int check_waits(pxp_solver_s *h) {
  if (pxp::wait_timeouts(h->stream) != h->timeouts_seen)
    return h->fail(PXP_ERR_CUDA, "a kernel's bounded wait for its copies ran out on this device");
  return PXP_OK;
}

static int download_field(pxp_solver_s *h, double *dst, const void *src, long long npts = -1) {
  if (npts < 0) npts = h->npts;
  if (int rc = check_waits(h)) return rc;
  if (h->prec == pxp::kFP64) {
    PXP_TRY_CUDA(h, cudaMemcpyAsync(dst, src, 16 * npts, cudaMemcpyDeviceToHost, h->stream));
    PXP_TRY_CUDA(h, cudaStreamSynchronize(h->stream));
  } else {
    std::vector<float> tmp(2 * npts);
    PXP_TRY_CUDA(h, cudaMemcpyAsync(tmp.data(), src, 8 * npts, cudaMemcpyDeviceToHost, h->stream));
    PXP_TRY_CUDA(h, cudaStreamSynchronize(h->stream));
    for (long long i = 0; i < 2 * npts; ++i) dst[i] = (double)tmp[i];
  }
  return PXP_OK;
}

int pxp_set_initial_conditions(pxp_solver h, const double *field) {
  if (h == nullptr || field == nullptr) return PXP_ERR_INVALID;
  int rc = upload_field(h, h->d_field, field);
  if (rc) return rc;
  h->current_step = 1;
  h->ic_set = true;
  return PXP_OK;
}

int pxp_set_initial_conditions_device(pxp_solver h, const void *dfield) {
  if (h == nullptr || dfield == nullptr) return PXP_ERR_INVALID;
  PXP_TRY_CUDA(h, cudaMemcpyAsync(h->d_field, dfield, h->csize * h->npts,
                                  cudaMemcpyDeviceToDevice, h->stream));
  h->current_step = 1;
  h->ic_set = true;
  return PXP_OK;
}

int pxp_step(pxp_solver h, int nsteps) {
  if (h == nullptr) return PXP_ERR_INVALID;
  if (nsteps < 0) return h->fail(PXP_ERR_INVALID, "negative step count");
  if (!h->ic_set)
    return h->fail(PXP_ERR_INVALID, "setInitialConditions must be called before stepping");
  if (nsteps == 0) return PXP_OK;
  PXP_TRY_CUDA(h, cudaSetDevice(h->prob.device));
  const long long first = h->current_step, last = first + nsteps - 1;
  if (h->plane_count > 0 &&
      (first < h->plane_first || last >= (long long)h->plane_first + h->plane_count))
    return h->fail(PXP_ERR_INVALID, "steps " + std::to_string(first) + ".." + std::to_string(last) +
                                        " are outside the material planes provided");
  cudaError_t e = cudaSuccess;
  switch (h->prob.kind) {
    case PXP_FFT_SOLVER_2D: {
      int v = -1;
      if (int rc = variant_2d(h, &v)) return rc;
      e = pxp::launch_fft1d(h->prec, (const pxp::Fft1dJob *)h->d_job, 1, (int)h->nx,
                            (int)first, nsteps, h->stream, h->flux_count > 0, v);
      break;
    }
    case PXP_CRANK_NICHOLSON:
      if (!(h->cn_const && !h->prob.transparent_bc && h->mat_stride == 0) &&
          !pxp::cn_supported(h->prec, (int)h->nx))
        return h->fail(PXP_ERR_UNSUPPORTED,
                       "CrankNicholson at " + std::to_string(h->nx) +
                           " points runs with a z-invariant medium and Dirichlet ends only");
      if (h->cn_const && !h->prob.transparent_bc && h->mat_stride == 0) {
        int v = -1;
        if (int rc = variant_2d(h, &v)) return rc;
        e = pxp::launch_cn_const(h->prec, (const pxp::CnJob *)h->d_job, 1,
                                 pxp::cn_padded_n((int)h->nx), (int)first, nsteps, h->stream,
                                 h->flux_count > 0, v);
      }
      else
        e = pxp::launch_cn(h->prec, (const pxp::CnJob *)h->d_job, 1, pxp::cn_padded_n((int)h->nx),
                           (int)first, nsteps, h->stream, h->flux_count > 0);
      break;
    case PXP_ADI: {
      int rc = adi_steps(h, (unsigned)first, nsteps);
      if (rc) return rc;
      break;
    }
    case PXP_FFT_SOLVER_3D: {
      int rc = fft3d_steps(h, (unsigned)first, nsteps);
      if (rc) return rc;
      break;
    }
    default:
      return h->fail(PXP_ERR_UNSUPPORTED, "kind not available");
  }
  if (e != cudaSuccess) return h->cuda_fail(e, "kernel launch");
  h->current_step += (unsigned)nsteps;
  return PXP_OK;
}

int pxp_solve(pxp_solver h) {
  if (h == nullptr) return PXP_ERR_INVALID;
  if (h->current_step >= h->nz) return PXP_OK;
  return pxp_step(h, (int)(h->nz - h->current_step));
}

int pxp_synchronize(pxp_solver h) {
  if (h == nullptr) return PXP_ERR_INVALID;
  PXP_TRY_CUDA(h, cudaStreamSynchronize(h->stream));
  return check_waits(h);
}

int pxp_selftest_bounded_wait(pxp_solver h, unsigned long long limit_ns) {
  if (h == nullptr || limit_ns == 0 || limit_ns > 10000000000ull) return PXP_ERR_INVALID;
  cudaError_t e = pxp::launch_wait_selftest(limit_ns, h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "bounded-wait self-test launch");
  return PXP_OK;
}

int pxp_get_last_solution(pxp_solver h, double *field) {
  if (h == nullptr || field == nullptr) return PXP_ERR_INVALID;
  return download_field(h, field, h->d_field);
}

int pxp_get_field_device(pxp_solver h, void **dfield, int *precision) {
  if (h == nullptr || dfield == nullptr) return PXP_ERR_INVALID;
  *dfield = h->d_field;
  if (precision) *precision = h->prob.precision;
  return PXP_OK;
}

int pxp_get_stream(pxp_solver h, void **stream) {
  if (h == nullptr || stream == nullptr) return PXP_ERR_INVALID;
  *stream = (void *)h->stream;
  return PXP_OK;
}

int pxp_num_saved(pxp_solver h, int *count) {
  if (h == nullptr || count == nullptr) return PXP_ERR_INVALID;
  int c = 0;
  if (h->save_every > 0 && h->ic_set) c = (int)((h->current_step - 1) / (unsigned)h->save_every);
  if (c > h->max_slots) c = h->max_slots;
  *count = c;
  return PXP_OK;
}

int pxp_get_saved(pxp_solver h, int slot, double *field) {
  if (h == nullptr || field == nullptr) return PXP_ERR_INVALID;
  int c = 0;
  pxp_num_saved(h, &c);
  if (slot < 0 || slot >= c)
    return h->fail(PXP_ERR_INVALID, "save slot " + std::to_string(slot) + " not filled");
  const char *base = (const char *)h->d_saves + (size_t)slot * h->csize * h->save_pts;
  return download_field(h, field, base, h->save_pts);
}

int pxp_get_post(pxp_solver h, int quantity, int slot, double *out) {
  if (h == nullptr || out == nullptr) return PXP_ERR_INVALID;
  if (quantity < PXP_POST_ABS || quantity > PXP_POST_ABS2)
    return h->fail(PXP_ERR_INVALID, "unknown post-processing quantity");
  const void *src = h->d_field;
  long long n = h->npts;
  if (slot >= 0) {
    int c = 0;
    pxp_num_saved(h, &c);
    if (slot >= c) return h->fail(PXP_ERR_INVALID, "save slot " + std::to_string(slot) + " not filled");
    src = (const char *)h->d_saves + (size_t)slot * h->csize * h->save_pts;
    n = h->save_pts;
  }
  if (int rc = check_waits(h)) return rc;
  double *d_out = nullptr;
  PXP_TRY_CUDA(h, cudaMallocAsync((void **)&d_out, sizeof(double) * n, h->stream));
  cudaError_t e = pxp::launch_post(h->prec, src, d_out, n, quantity, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream);
  cudaFreeAsync(d_out, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  return e == cudaSuccess ? PXP_OK : h->cuda_fail(e, "post-processing reduction");
}

int pxp_get_post_resized(pxp_solver h, int quantity, int slot, unsigned rows, unsigned cols,
                         double *out) {
  if (h == nullptr || out == nullptr) return PXP_ERR_INVALID;
  if (h->prob.kind != PXP_FFT_SOLVER_3D && h->prob.kind != PXP_ADI)
    return h->fail(PXP_ERR_UNSUPPORTED, "resized post-processing applies to the 3-D kinds");
  if (quantity < PXP_POST_ABS || quantity > PXP_POST_ABS2)
    return h->fail(PXP_ERR_INVALID, "unknown post-processing quantity");
  if (rows == 0 || cols == 0) return h->fail(PXP_ERR_INVALID, "export dimensions must be positive");
  const void *src = h->d_field;
  long long side = h->nx;
  if (slot >= 0) {
    int c = 0;
    pxp_num_saved(h, &c);
    if (slot >= c) return h->fail(PXP_ERR_INVALID, "save slot " + std::to_string(slot) + " not filled");
    src = (const char *)h->d_saves + (size_t)slot * h->csize * h->save_pts;
    side = h->save_n;
  }
  // resizeMatrix returns the matrix unchanged unless both dimensions shrink
  if (rows >= side || cols >= side) return pxp_get_post(h, quantity, slot, out);
  if (int rc = check_waits(h)) return rc;
  const long long n = side * side;
  double *d_full = nullptr, *d_small = nullptr;
  PXP_TRY_CUDA(h, cudaMallocAsync((void **)&d_full, sizeof(double) * n, h->stream));
  cudaError_t e = cudaMallocAsync((void **)&d_small, sizeof(double) * rows * cols, h->stream);
  if (e == cudaSuccess) e = pxp::launch_post(h->prec, src, d_full, n, quantity, h->stream);
  if (e == cudaSuccess) {
    const double dX = (double)side / ((double)cols + 1.0), dY = (double)side / ((double)rows + 1.0);
    e = pxp::launch_resize(d_full, side, d_small, (int)rows, (int)cols, dY, dX, h->stream);
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, d_small, sizeof(double) * rows * cols, cudaMemcpyDeviceToHost, h->stream);
  cudaFreeAsync(d_full, h->stream);
  if (d_small) cudaFreeAsync(d_small, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  return e == cudaSuccess ? PXP_OK : h->cuda_fail(e, "resized post-processing");
}

int pxp_saved_max_abs(pxp_solver h, double *max_abs) {
  if (h == nullptr || max_abs == nullptr) return PXP_ERR_INVALID;
  int c = 0;
  pxp_num_saved(h, &c);
  if (int rc = check_waits(h)) return rc;
  unsigned long long *d_max = nullptr;
  PXP_TRY_CUDA(h, cudaMallocAsync((void **)&d_max, sizeof(unsigned long long), h->stream));
  cudaError_t e = cudaMemsetAsync(d_max, 0, sizeof(unsigned long long), h->stream);
  for (int k = 0; k < c && e == cudaSuccess; ++k)
    e = pxp::launch_max_abs(h->prec, (const char *)h->d_saves + (size_t)k * h->csize * h->save_pts,
                            h->save_pts, d_max, h->stream);
  unsigned long long bits = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, d_max, sizeof(bits), cudaMemcpyDeviceToHost, h->stream);
  cudaFreeAsync(d_max, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "max |u| over the saved fields");
  std::memcpy(max_abs, &bits, sizeof(double));
  return PXP_OK;
}

// ---- far field -------------------------------------------------------------
namespace {

// FarField::farFieldAngleToIndx (src/farFieldPost.cpp:78-101).
unsigned ff_angle_index(double angle, unsigned size, double k, double step) {
  const double angle_rad = angle * PI / 180.0;
  const double v = size * k * step * std::sin(angle_rad) / (2.0 * PI);
  // int conversion truncates; a value beyond int range is past either end
  if (!(std::fabs(v) < 2147483647.0)) return angle > 0.0 ? size - 1 : 0;
  const int n = (int)v;
  if ((unsigned)std::abs(n) >= size / 2) return angle > 0.0 ? size - 1 : 0;
  return (unsigned)(n + (int)(size / 2));
}

// Device tables of the far field, shared like the solver tables: kind 4 the
// L-entry table exp(-2 pi i m / L), kind 5 the Stockham twiddles of length q,
// kind 6 the split form of kind 4: lo[r] = exp(-2 pi i r / L) for
// r < 2^b, then hi[q] = exp(-2 pi i q 2^b / L) for q < L / 2^b.
int ff_table(pxp_solver_s *h, int kind, long long len, const double2 **out) {
  TableKey key{h->prob.device, kind, (unsigned)len, 0.0, 0.0, 0.0, 0};  // FP64 kernels
  std::lock_guard<std::mutex> lk(g_table_mutex);
  auto it = g_tables.find(key);
  if (it == g_tables.end()) {
    std::vector<cd> t;
    if (kind == 5) {
      t = twiddles((int)len);
    } else if (kind == 6) {
      const int b = pxp::farfield_split_bits(len);
      const long long nlo = 1LL << b, nhi = len >> b;
      const long double pi_l = 3.141592653589793238462643383279502884L;
      t.resize((size_t)(nlo + nhi));
      for (long long r = 0; r < nlo; ++r) {
        const long double a = -2.0L * pi_l * (long double)r / (long double)len;
        t[(size_t)r] = cd((double)cosl(a), (double)sinl(a));
      }
      for (long long q = 0; q < nhi; ++q) {
        const long double a = -2.0L * pi_l * (long double)(q * nlo) / (long double)len;
        t[(size_t)(nlo + q)] = cd((double)cosl(a), (double)sinl(a));
      }
    } else {
      t.resize((size_t)len);
      const long double pi_l = 3.141592653589793238462643383279502884L;
      for (long long m = 0; m < len; ++m) {
        const long double a = -2.0L * pi_l * (long double)m / (long double)len;
        t[(size_t)m] = cd((double)cosl(a), (double)sinl(a));
      }
    }
    void *p = nullptr;
    if (cudaMalloc(&p, sizeof(cd) * t.size()) != cudaSuccess) {
      cudaGetLastError();
      return h->fail(PXP_ERR_NOMEM, "far-field table allocation");
    }
    cudaError_t e = cudaMemcpy(p, t.data(), sizeof(cd) * t.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return h->cuda_fail(e, "far-field table upload");
    it = g_tables.emplace(key, p).first;
  }
  *out = (const double2 *)it->second;
  return PXP_OK;
}

struct FfPlan {
  bool three_d = false;
  long long L = 0;
  unsigned y0 = 0, y1 = 0, x0 = 0, x1 = 0;  // windows (3-D: y along columns, x along rows)
  unsigned rows = 0, cols = 0;              // result before resizing
  unsigned out_rows = 0, out_cols = 0;      // returned shape
  bool resize = false;
};

int ff_plan(pxp_solver_s *h, const pxp_farfield_params *p, FfPlan &f) {
  if (p == nullptr) return h->fail(PXP_ERR_INVALID, "far-field parameters missing");
  f.three_d = h->prob.kind == PXP_FFT_SOLVER_3D || h->prob.kind == PXP_ADI;
  const double k = h->prob.wavenumber;
  const long long n = h->nx;
  if (!f.three_d) {
    f.L = p->pad_length < n ? n : p->pad_length;
  } else {
    if (p->padding == PXP_PAD_LINEAR_FIT)
      return h->fail(PXP_ERR_UNSUPPORTED, "linear-fit padding is not provided");
    if (p->padding != PXP_PAD_ZERO && p->padding != PXP_PAD_CONSTANT)
      return h->fail(PXP_ERR_INVALID, "unknown far-field padding");
    f.L = std::max<long long>({(long long)p->pad_length, (long long)h->ny, n});
  }
  if (f.L > (1LL << 22)) return h->fail(PXP_ERR_UNSUPPORTED, "far-field pad length above 2^22");
  const unsigned L = (unsigned)f.L;
  f.x0 = ff_angle_index(p->phi_min, L, k, h->prob.x.step);
  f.x1 = ff_angle_index(p->phi_max, L, k, h->prob.x.step);
  if (f.x1 < f.x0) return h->fail(PXP_ERR_INVALID, "empty far-field angular range");
  if (!f.three_d) {
    f.rows = f.out_rows = f.x1 - f.x0 + 1;
    f.cols = f.out_cols = 1;
    return PXP_OK;
  }
  f.y0 = ff_angle_index(p->phi_min, L, k, h->prob.y.step);
  f.y1 = ff_angle_index(p->phi_max, L, k, h->prob.y.step);
  if (f.y1 < f.y0) return h->fail(PXP_ERR_INVALID, "empty far-field angular range");
  f.rows = f.y1 - f.y0 + 1;
  f.cols = f.x1 - f.x0 + 1;
  f.resize = p->export_rows != 0 && p->export_cols != 0 && p->export_rows < f.rows &&
             p->export_cols < f.cols;
  f.out_rows = f.resize ? p->export_rows : f.rows;
  f.out_cols = f.resize ? p->export_cols : f.cols;
  return PXP_OK;
}

// The pruned transform unless computing the kept outputs directly is cheaper.
// PXP_FARFIELD_PATH=direct or =pruned pins the choice (the pruned transform
// where the length allows it).
int ff_choose_q(long long n, long long L, long long window) {
  const int q = pxp::farfield_pruned_q(n, L);
  if (q == 0) return 0;
  if (const char *v = std::getenv("PXP_FARFIELD_PATH")) {
    if (std::strcmp(v, "direct") == 0) return 0;
    if (std::strcmp(v, "pruned") == 0) return q;
  }
  int lg = 0;
  while ((1 << lg) < q) ++lg;
  const long long passes = std::min(L / q, window);
  return n * window < passes * q * lg ? 0 : q;
}

}  // namespace

void pxp_farfield_defaults(pxp_farfield_params *p) {
  if (p == nullptr) return;
  *p = pxp_farfield_params{};
  p->phi_min = -90.0;
  p->phi_max = 90.0;
  p->padding = PXP_PAD_ZERO;
}

int pxp_farfield_shape(pxp_solver h, const pxp_farfield_params *p, unsigned *rows, unsigned *cols) {
  if (h == nullptr) return PXP_ERR_INVALID;
  FfPlan f;
  if (int rc = ff_plan(h, p, f)) return rc;
  if (rows) *rows = f.out_rows;
  if (cols) *cols = f.out_cols;
  return PXP_OK;
}

int pxp_farfield(pxp_solver h, const pxp_farfield_params *p, double *out) {
  if (h == nullptr || out == nullptr) return PXP_ERR_INVALID;
  FfPlan f;
  if (int rc = ff_plan(h, p, f)) return rc;
  if (!h->ic_set) return h->fail(PXP_ERR_INVALID, "no field: set the initial conditions first");
  if (f.three_d && p->subtract_reference && h->d_ref == nullptr)
    return h->fail(PXP_ERR_INVALID, "no reference field set");
  if (int rc = check_waits(h)) return rc;
  const double2 *wL = nullptr;
  if (int rc = ff_table(h, 4, f.L, &wL)) return rc;
  cudaStream_t s = h->stream;
  const bool c64 = h->prec != pxp::kFP64;
  std::vector<void *> tmp;
  auto release = [&]() {
    for (void *t : tmp) cudaFreeAsync(t, s);
  };
  auto dalloc = [&](size_t bytes) -> void * {
    void *q = nullptr;
    if (cudaMallocAsync(&q, bytes, s) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    tmp.push_back(q);
    return q;
  };
  const double2 *wsplit = nullptr;
  const int split_bits = pxp::farfield_split_bits(f.L);
  auto lines_for = [&](long long n, long long window, int *q, const double2 **twq) -> int {
    *q = ff_choose_q(n, f.L, window);
    *twq = nullptr;
    if (*q == 0) return PXP_OK;
    if (wsplit == nullptr)
      if (int rc = ff_table(h, 6, f.L, &wsplit)) return rc;
    return ff_table(h, 5, *q, twq);
  };
  cudaError_t e = cudaSuccess;
  double *d_res = nullptr;
  const size_t out_elems = (size_t)f.out_rows * f.out_cols;
  if (!f.three_d) {
    pxp::FarFieldLines ln{};
    ln.in = h->d_field;
    ln.in_c64 = c64;
    ln.line_stride = h->nx;
    ln.n = (int)h->nx;
    ln.nlines = 1;
    ln.pad_value = (p->pad_length < h->nx) ? make_double2(0.0, 0.0)
                                           : make_double2(p->pad_value_re, p->pad_value_im);
    ln.L = f.L;
    ln.i0 = f.x0;
    ln.i1 = f.x1;
    ln.mode = 2;
    ln.divisor = std::sqrt((double)f.L);
    ln.out_stride = 1;
    ln.wL = wL;
    int q;
    if (int rc = lines_for(ln.n, f.rows, &q, &ln.twQ)) return rc;
    ln.wsplit = wsplit;
    ln.split_bits = split_bits;
    d_res = (double *)dalloc(sizeof(double) * out_elems);
    if (d_res == nullptr) return h->fail(PXP_ERR_NOMEM, "far-field buffers");
    ln.out = d_res;
    e = pxp::launch_farfield_lines(ln, q, s);
  } else {
    const unsigned rows = h->ny, cols = h->nx;
    if (p->padding == PXP_PAD_CONSTANT && rows != cols)
      return h->fail(PXP_ERR_UNSUPPORTED, "constant padding needs a square field");
    double2 *d_t = (double2 *)dalloc(sizeof(double2) * (size_t)f.rows * cols);
    d_res = (double *)dalloc(sizeof(double) * (size_t)f.rows * f.cols);
    double *d_small = f.resize ? (double *)dalloc(sizeof(double) * out_elems) : nullptr;
    if (d_t == nullptr || d_res == nullptr || (f.resize && d_small == nullptr)) {
      release();
      return h->fail(PXP_ERR_NOMEM, "far-field buffers");
    }
    // columns, cut along y -> d_t[(i - y0) * cols + c]
    pxp::FarFieldLines a{};
    a.in = h->d_field;
    a.in_c64 = c64;
    a.ref = p->subtract_reference ? (const double2 *)h->d_ref : nullptr;
    a.line_stride = rows;
    a.n = (int)rows;
    a.nlines = cols;
    a.pad_const = p->padding == PXP_PAD_CONSTANT;
    a.L = f.L;
    a.i0 = f.y0;
    a.i1 = f.y1;
    a.mode = 0;
    a.out = d_t;
    a.out_stride = cols;
    a.wL = wL;
    int qa;
    if (int rc = lines_for(a.n, f.rows, &qa, &a.twQ)) {
      release();
      return rc;
    }
    a.wsplit = wsplit;
    a.split_bits = split_bits;
    e = pxp::launch_farfield_lines(a, qa, s);
    // conjugated rows, cut along x -> d_res[r + (i - x0) * rows], |X|^2 / L
    pxp::FarFieldLines b{};
    b.in = d_t;
    b.line_stride = cols;
    b.n = (int)cols;
    b.nlines = f.rows;
    b.conj_in = 1;
    b.pad_const = a.pad_const;
    b.L = f.L;
    b.i0 = f.x0;
    b.i1 = f.x1;
    b.mode = 1;
    b.divisor = (double)f.L;
    b.out = d_res;
    b.out_stride = f.rows;
    b.wL = wL;
    int qb;
    if (int rc = lines_for(b.n, f.cols, &qb, &b.twQ)) {
      release();
      return rc;
    }
    b.wsplit = wsplit;
    b.split_bits = split_bits;
    if (e == cudaSuccess) e = pxp::launch_farfield_lines(b, qb, s);
    if (e == cudaSuccess && f.resize) {
      const double dX = (double)f.cols / ((double)p->export_cols + 1.0);
      const double dY = (double)f.rows / ((double)p->export_rows + 1.0);
      e = pxp::launch_resize(d_res, f.rows, d_small, (int)p->export_rows, (int)p->export_cols, dY,
                             dX, s);
      d_res = d_small;
    }
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, d_res, sizeof(double) * out_elems, cudaMemcpyDeviceToHost, s);
  release();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? PXP_OK : h->cuda_fail(e, "far field");
}

int pxp_set_reference(pxp_solver h, const double *field) {
  if (h == nullptr) return PXP_ERR_INVALID;
  if (field == nullptr) {
    free_dev(h->d_ref, h->stream);
    return PXP_OK;
  }
  if (h->d_ref == nullptr)
    if (int rc = alloc(h, &h->d_ref, sizeof(cd) * h->npts, "reference field")) return rc;
  return h2d(h, h->d_ref, field, sizeof(cd) * h->npts);
}

int pxp_set_reference_from(pxp_solver h, pxp_solver src) {
  if (h == nullptr || src == nullptr) return PXP_ERR_INVALID;
  if (src->npts != h->npts || src->prob.device != h->prob.device)
    return h->fail(PXP_ERR_INVALID, "reference handle has another grid size or device");
  if (!src->ic_set) return h->fail(PXP_ERR_INVALID, "reference handle holds no field");
  if (int rc = check_waits(src)) return rc;
  if (h->d_ref == nullptr)
    if (int rc = alloc(h, &h->d_ref, sizeof(cd) * h->npts, "reference field")) return rc;
  // the source's pending steps finish before this handle's stream reads its field
  PXP_TRY_CUDA(h, cudaStreamSynchronize(src->stream));
  cudaError_t e = src->prec == pxp::kFP64
                      ? cudaMemcpyAsync(h->d_ref, src->d_field, sizeof(cd) * h->npts,
                                        cudaMemcpyDeviceToDevice, h->stream)
                      : pxp::launch_widen(src->d_field, h->d_ref, h->npts, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  return e == cudaSuccess ? PXP_OK : h->cuda_fail(e, "copying the reference field");
}

// ---- per-step flux (post::Transmittivity) -----------------------------------
int pxp_set_flux_windows(pxp_solver h, int first_step, int count, const unsigned *start,
                         const unsigned *end) {
  if (h == nullptr || count < 0) return PXP_ERR_INVALID;
  if (h->prob.kind != PXP_FFT_SOLVER_2D && h->prob.kind != PXP_CRANK_NICHOLSON)
    return h->fail(PXP_ERR_UNSUPPORTED, "flux windows apply to the 2-D kinds");
  PXP_TRY_CUDA(h, cudaStreamSynchronize(h->stream));
  free_dev(h->d_flux_win, h->stream);
  free_dev(h->d_flux, h->stream);
  h->flux_step0 = 0;
  h->flux_count = 0;
  if (count > 0) {
    if (first_step < 1 || start == nullptr || end == nullptr) return PXP_ERR_INVALID;
    std::vector<int2> w((size_t)count);
    for (int k = 0; k < count; ++k) {
      if (start[k] > end[k] || end[k] >= h->nx)
        return h->fail(PXP_ERR_INVALID, "flux window " + std::to_string(k) + " is not a <= b < Nx");
      w[(size_t)k] = make_int2((int)start[k], (int)end[k]);
    }
    const std::vector<double> nan((size_t)count, std::nan(""));
    int rc;
    if ((rc = alloc(h, (void **)&h->d_flux_win, sizeof(int2) * count, "flux windows"))) return rc;
    if ((rc = alloc(h, (void **)&h->d_flux, sizeof(double) * count, "flux sums"))) return rc;
    if ((rc = h2d(h, h->d_flux_win, w.data(), sizeof(int2) * count))) return rc;
    if ((rc = h2d(h, h->d_flux, nan.data(), sizeof(double) * count))) return rc;
    h->flux_step0 = first_step;
    h->flux_count = count;
  }
  return rewrite_job(h);
}

int pxp_get_flux(pxp_solver h, int first_step, int count, double *out) {
  if (h == nullptr || out == nullptr || count < 0) return PXP_ERR_INVALID;
  if (first_step < h->flux_step0 || (long long)first_step + count > (long long)h->flux_step0 + h->flux_count)
    return h->fail(PXP_ERR_INVALID, "steps outside the flux windows set");
  if (count == 0) return PXP_OK;
  if (int rc = check_waits(h)) return rc;
  PXP_TRY_CUDA(h, cudaMemcpyAsync(out, h->d_flux + (first_step - h->flux_step0), sizeof(double) * count,
                                  cudaMemcpyDeviceToHost, h->stream));
  PXP_TRY_CUDA(h, cudaStreamSynchronize(h->stream));
  return PXP_OK;
}

int pxp_field_flux(pxp_solver h, unsigned start, unsigned end, double *sum) {
  if (h == nullptr || sum == nullptr) return PXP_ERR_INVALID;
  if (h->prob.kind != PXP_FFT_SOLVER_2D && h->prob.kind != PXP_CRANK_NICHOLSON)
    return h->fail(PXP_ERR_UNSUPPORTED, "flux sums apply to the 2-D kinds");
  if (start > end || end >= h->nx) return h->fail(PXP_ERR_INVALID, "flux window is not a <= b < Nx");
  if (!h->ic_set) return h->fail(PXP_ERR_INVALID, "no field: set the initial conditions first");
  if (int rc = check_waits(h)) return rc;
  double *d = nullptr;
  PXP_TRY_CUDA(h, cudaMallocAsync((void **)&d, sizeof(double), h->stream));
  cudaError_t e = pxp::launch_flux_sum(h->prec, h->d_field, (int)start, (int)end, d, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sum, d, sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  cudaFreeAsync(d, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  return e == cudaSuccess ? PXP_OK : h->cuda_fail(e, "flux sum");
}

int pxp_reset(pxp_solver h) {
  if (h == nullptr) return PXP_ERR_INVALID;
  h->current_step = 1;
  return PXP_OK;
}

int pxp_current_step(pxp_solver h, unsigned *step) {
  if (h == nullptr || step == nullptr) return PXP_ERR_INVALID;
  *step = h->current_step;
  return PXP_OK;
}

int pxp_shape(pxp_solver h, unsigned *nx, unsigned *ny, unsigned *nz) {
  if (h == nullptr) return PXP_ERR_INVALID;
  if (nx) *nx = h->nx;
  if (ny) *ny = h->ny;
  if (nz) *nz = h->nz;
  return PXP_OK;
}

int pxp_device_bytes(pxp_solver h, size_t *bytes) {
  if (h == nullptr || bytes == nullptr) return PXP_ERR_INVALID;
  *bytes = h->dev_bytes;
  return PXP_OK;
}

int pxp_get_intensity(pxp_solver h, double *intensity) {
  if (h == nullptr || intensity == nullptr) return PXP_ERR_INVALID;
  std::vector<double> f(2 * h->npts);
  int rc = download_field(h, f.data(), h->d_field);
  if (rc) return rc;
  for (long long i = 0; i < h->npts; ++i)
    intensity[i] = f[2 * i] * f[2 * i] + f[2 * i + 1] * f[2 * i + 1];
  return PXP_OK;
}

}  // extern "C"

// ============================================================== batches ==
struct pxp_batch_s {
  int device = 0;
  size_t budget = 0, used = 0;
  cudaStream_t stream = nullptr;  // job uploads; joins the group streams
  // 2-D groups of different (kind, size) run concurrently, one stream each,
  // started after the round's upload and joined back into `stream`
  std::vector<cudaStream_t> gstreams;
  std::vector<cudaEvent_t> gdone;
  cudaEvent_t uploaded = nullptr;
  // one job counter per group: FFTSolver2D groups run persistent CTAs that
  // take their next job from it (persistent.cuh)
  unsigned *d_queue = nullptr;
  size_t queue_cap = 0;
  std::vector<pxp_solver_s *> active;
  void *d_jobs = nullptr;
  size_t d_jobs_cap = 0;
  void *h_jobs = nullptr;  // pinned staging of the job descriptors
  size_t h_jobs_cap = 0;
  std::string err;
  int fail(int code, const std::string &m) {
    err = m;
    set_global_error(m);
    return code;
  }
};

namespace {

bool is_2d(const pxp_solver_s *h) {
  return h->prob.kind == PXP_FFT_SOLVER_2D || h->prob.kind == PXP_CRANK_NICHOLSON;
}
bool cn_uses_const(const pxp_solver_s *h) {
  return h->cn_const && !h->prob.transparent_bc && h->mat_stride == 0;
}

int grow(pxp_batch_s *b, size_t bytes) {
  if (bytes <= b->d_jobs_cap) return PXP_OK;
  size_t cap = std::max(bytes, 2 * b->d_jobs_cap);
  if (b->d_jobs) cudaFreeAsync(b->d_jobs, b->stream);
  if (b->h_jobs) {
    cudaStreamSynchronize(b->stream);
    cudaFreeHost(b->h_jobs);
  }
  b->d_jobs = nullptr;
  b->h_jobs = nullptr;
  cudaError_t e = cudaMallocAsync(&b->d_jobs, cap, b->stream);
  if (e == cudaSuccess) e = cudaMallocHost(&b->h_jobs, cap);
  if (e != cudaSuccess) return b->fail(PXP_ERR_NOMEM, "batch job arrays");
  b->d_jobs_cap = b->h_jobs_cap = cap;
  return PXP_OK;
}

}  // namespace

extern "C" {

int pxp_batch_create(int device, size_t budget, pxp_batch *out) {
  if (out == nullptr) return PXP_ERR_INVALID;
  *out = nullptr;
  pxp_batch_s *b = new (std::nothrow) pxp_batch_s();
  if (!b) return PXP_ERR_NOMEM;
  b->device = device;
  b->budget = budget;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) retain_pool(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    set_global_error(std::string("batch stream: ") + cudaGetErrorString(e));
    delete b;
    return PXP_ERR_CUDA;
  }
  *out = b;
  return PXP_OK;
}

int pxp_batch_destroy(pxp_batch b) {
  if (b == nullptr) return PXP_OK;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  if (b->d_jobs) cudaFreeAsync(b->d_jobs, b->stream);
  cudaStreamSynchronize(b->stream);
  if (b->h_jobs) cudaFreeHost(b->h_jobs);
  if (b->d_queue) cudaFree(b->d_queue);
  for (cudaStream_t g : b->gstreams) cudaStreamDestroy(g);
  for (cudaEvent_t e : b->gdone) cudaEventDestroy(e);
  if (b->uploaded) cudaEventDestroy(b->uploaded);
  cudaStreamDestroy(b->stream);
  delete b;
  return PXP_OK;
}

int pxp_batch_admit(pxp_batch b, pxp_solver h, int nsteps) {
  if (b == nullptr || h == nullptr || nsteps < 0) return PXP_ERR_INVALID;
  if (h->prob.device != b->device) return b->fail(PXP_ERR_INVALID, "solver on another device");
  if (!h->ic_set) return b->fail(PXP_ERR_INVALID, "solver has no initial conditions");
  for (pxp_solver_s *a : b->active)
    if (a == h) return b->fail(PXP_ERR_INVALID, "solver already admitted");
  if (h->plane_count > 0 &&
      (h->current_step < (unsigned)h->plane_first ||
       (long long)h->current_step + nsteps > (long long)h->plane_first + h->plane_count))
    return b->fail(PXP_ERR_INVALID, "steps outside the material planes provided");
  if (h->prob.kind == PXP_CRANK_NICHOLSON && !cn_uses_const(h) &&
      !pxp::cn_supported(h->prec, (int)h->nx))
    return b->fail(PXP_ERR_UNSUPPORTED, "CrankNicholson at this size needs a z-invariant medium "
                                        "and Dirichlet ends");
  if (b->used + h->dev_bytes > b->budget) return PXP_ERR_NOT_READY;
  cudaSetDevice(b->device);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess)
    return b->fail(PXP_ERR_CUDA, "solver stream");
  h->batch_remaining = nsteps;
  b->active.push_back(h);
  b->used += h->dev_bytes;
  return PXP_OK;
}

int pxp_batch_round(pxp_batch b, int max_steps) {
  if (b == nullptr || max_steps <= 0) return PXP_ERR_INVALID;
  cudaSetDevice(b->device);
  // the staging buffer of the previous round must be consumed
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return b->fail(PXP_ERR_CUDA, "batch stream");
  // ---- 2-D groups: key (kind, n, precision, CN matrix path)
  struct Key {
    int kind, n, prec, cpath;
    bool operator<(const Key &o) const {
      return std::tie(kind, n, prec, cpath) < std::tie(o.kind, o.n, o.prec, o.cpath);
    }
  };
  std::map<Key, std::vector<pxp_solver_s *>> groups;
  for (pxp_solver_s *h : b->active) {
    if (!is_2d(h) || h->batch_remaining <= 0) continue;
    Key k{h->prob.kind, (int)h->nx, (int)h->prec, h->prob.kind == PXP_CRANK_NICHOLSON ? (int)cn_uses_const(h) : 0};
    groups[k].push_back(h);
  }
  // Within a group the CTA index follows the job order, and the block
  // scheduler starts CTAs in index order as SMs free up: with the jobs that
  // have the most steps this round first (longest processing time first),
  // a launch with more jobs than resident CTAs fills the freed slots with
  // the shorter jobs and ends close to the longest job's time.
  for (auto &g : groups)
    std::stable_sort(g.second.begin(), g.second.end(),
                     [max_steps](const pxp_solver_s *a, const pxp_solver_s *c) {
                       return std::min(a->batch_remaining, max_steps) >
                              std::min(c->batch_remaining, max_steps);
                     });
  // each group's kernel variant, the one every solver of its key runs alone
  // (tuned here, before this round launches anything, if no solver of the
  // key has stepped yet)
  std::vector<int> gvariant;
  for (auto &g : groups) {
    int v = -1;
    if (int rc = variant_2d(g.second.front(), &v)) return b->fail(rc, g.second.front()->err);
    gvariant.push_back(v);
  }
  size_t total = 0;
  for (auto &g : groups)
    total += g.second.size() * (g.first.kind == PXP_FFT_SOLVER_2D ? sizeof(pxp::Fft1dJob) : sizeof(pxp::CnJob));
  if (total > 0) {
    int rc = grow(b, total);
    if (rc) return rc;
  }
  size_t off = 0;
  std::vector<std::pair<size_t, const std::pair<const Key, std::vector<pxp_solver_s *>> *>> offs;
  for (auto &g : groups) {
    offs.push_back({off, &g});
    for (pxp_solver_s *h : g.second) {
      const int n = std::min(h->batch_remaining, max_steps);
      if (g.first.kind == PXP_FFT_SOLVER_2D) {
        pxp::Fft1dJob j = h->job_fft;
        j.step0 = (int)h->current_step;
        j.nsteps = n;
        std::memcpy((char *)b->h_jobs + off, &j, sizeof(j));
        off += sizeof(j);
      } else {
        pxp::CnJob j = h->job_cn;
        j.step0 = (int)h->current_step;
        j.nsteps = n;
        std::memcpy((char *)b->h_jobs + off, &j, sizeof(j));
        off += sizeof(j);
      }
    }
  }
  if (total > 0 &&
      cudaMemcpyAsync(b->d_jobs, b->h_jobs, total, cudaMemcpyHostToDevice, b->stream) != cudaSuccess)
    return b->fail(PXP_ERR_CUDA, "job upload");
  // one stream per group (created as needed), each starting after the upload
  // and joined back into the batch stream
  if (!offs.empty()) {
    if (!b->uploaded && cudaEventCreateWithFlags(&b->uploaded, cudaEventDisableTiming) != cudaSuccess)
      return b->fail(PXP_ERR_CUDA, "batch event");
    while (b->gstreams.size() < offs.size()) {
      cudaStream_t st;
      cudaEvent_t ev;
      if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
        return b->fail(PXP_ERR_CUDA, "batch group stream");
      if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaStreamDestroy(st);
        return b->fail(PXP_ERR_CUDA, "batch group event");
      }
      b->gstreams.push_back(st);
      b->gdone.push_back(ev);
    }
    if (cudaEventRecord(b->uploaded, b->stream) != cudaSuccess)
      return b->fail(PXP_ERR_CUDA, "batch event record");
  }
  if (b->queue_cap < offs.size()) {
    if (b->d_queue) cudaFree(b->d_queue);
    b->d_queue = nullptr;
    b->queue_cap = 0;
    if (cudaMalloc(&b->d_queue, sizeof(unsigned) * offs.size()) != cudaSuccess) {
      cudaGetLastError();
      return b->fail(PXP_ERR_NOMEM, "batch job counters");
    }
    b->queue_cap = offs.size();
  }
  for (size_t gi = 0; gi < offs.size(); ++gi) {
    auto &o = offs[gi];
    cudaStream_t gst = b->gstreams[gi];
    if (cudaStreamWaitEvent(gst, b->uploaded, 0) != cudaSuccess)
      return b->fail(PXP_ERR_CUDA, "batch group wait");
    const Key &k = o.second->first;
    const auto &list = o.second->second;
    const void *jobs = (const char *)b->d_jobs + o.first;
    bool any_flux = false;
    for (const pxp_solver_s *h : list) any_flux = any_flux || h->flux_count > 0;
    const int variant = gvariant[gi];
    cudaError_t e;
    if (k.kind == PXP_FFT_SOLVER_2D) {
      e = cudaMemsetAsync(b->d_queue + gi, 0, sizeof(unsigned), gst);
      if (e == cudaSuccess)
        e = pxp::launch_fft1d((pxp::Precision)k.prec, (const pxp::Fft1dJob *)jobs,
                              (int)list.size(), k.n, -1, -1, gst, any_flux, variant,
                              b->d_queue + gi);
    }
    else if (k.cpath)
      e = pxp::launch_cn_const((pxp::Precision)k.prec, (const pxp::CnJob *)jobs, (int)list.size(),
                               pxp::cn_padded_n(k.n), -1, -1, gst, any_flux, variant);
    else
      e = pxp::launch_cn((pxp::Precision)k.prec, (const pxp::CnJob *)jobs, (int)list.size(),
                         pxp::cn_padded_n(k.n), -1, -1, gst, any_flux);
    if (e != cudaSuccess) return b->fail(PXP_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    if (cudaEventRecord(b->gdone[gi], gst) != cudaSuccess ||
        cudaStreamWaitEvent(b->stream, b->gdone[gi], 0) != cudaSuccess)
      return b->fail(PXP_ERR_CUDA, "batch group join");
    for (pxp_solver_s *h : list) {
      const int n = std::min(h->batch_remaining, max_steps);
      h->current_step += (unsigned)n;
      h->batch_remaining -= n;
    }
  }
  // ---- 3-D solvers on their own streams
  for (pxp_solver_s *h : b->active) {
    if (is_2d(h) || h->batch_remaining <= 0) continue;
    const int n = std::min(h->batch_remaining, max_steps);
    int rc = pxp_step(h, n);
    if (rc) return b->fail(rc, h->err);
    h->batch_remaining -= n;
  }
  return PXP_OK;
}

int pxp_batch_collect(pxp_batch b, pxp_solver *done, int cap, int *count) {
  if (b == nullptr || count == nullptr || (cap > 0 && done == nullptr)) return PXP_ERR_INVALID;
  cudaSetDevice(b->device);
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return b->fail(PXP_ERR_CUDA, "batch stream");
  int c = 0;
  std::vector<pxp_solver_s *> keep;
  for (pxp_solver_s *h : b->active) {
    if (!is_2d(h) && cudaStreamSynchronize(h->stream) != cudaSuccess)
      return b->fail(PXP_ERR_CUDA, "solver stream");
    if (h->batch_remaining <= 0 && c < cap) {
      done[c++] = h;
      b->used -= h->dev_bytes;
    } else {
      keep.push_back(h);
    }
  }
  b->active.swap(keep);
  *count = c;
  return PXP_OK;
}

int pxp_batch_status(pxp_batch b, int *active, size_t *bytes) {
  if (b == nullptr) return PXP_ERR_INVALID;
  if (active) *active = (int)b->active.size();
  if (bytes) *bytes = b->used;
  return PXP_OK;
}

}  // extern "C"
