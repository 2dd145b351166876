// fft3d.cu -- K-FFT2: FFTSolver3D split step as two HBM line passes.
//
// Replaces FFTSolver3D::solveStep (src/fftSolver3D.cpp:52-85): the 2-D FFTW
// transforms of propagate (:87-120) are split into 1-D transforms along x and
// along y and regrouped so that each step reads and writes the field twice:
//   x pass  (lines of fixed row index, stride n):  F_x, * K(kx, ky), F_x^-1
//   y pass  (contiguous lines of fixed x):          F_y^-1, refraction, F_y
// where the y pass's trailing F_y is the next step's first transform.
// Persistent CTAs stream lines through two shared-memory buffers with
// cp.async prefetch of the next line; each line is transformed in place in a
// bank-conflict-free swizzled layout with the twiddles held in shared memory.
//
// FP64 pointwise arithmetic follows the reference op by op: the propagator
// argument fl(a * fl(fl(kx*kx) + fl(ky*ky))) with kx, ky from
// spatialFreqX/Y (:32-50), the refraction (prev * t) / (n*n) with t =
// exp(-k (beta + i delta) dz) (:154), the refraction integral (:253-273) when
// the material at z0 and z1 differs by more than 1e-10, and the absorber
// bands (Absorber::apply, src/absorber.cpp:3-12: y bands, then x bands).
// The propagator's sin/cos come from pxp_sincos.h (within 1 ulp of 1.0 on
// the argument range), exp in the refraction is CUDA's; everything else is
// rounded as the reference rounds it.
#include "fft3d_point.cuh"

namespace pxp {

// ---- asynchronous global -> shared copies (cp.async, 8 or 16 bytes)
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Issue the copy of line `line` into the swizzled buffer `dst`.
template <typename C, int N, int T>
__device__ __forceinline__ void load_line(C *dst, const C *field, int line, bool strided) {
  if (strided) {
    // element j of row `line` is at j*N + line
    for (int j = threadIdx.x; j < N; j += T) {
      if constexpr (sizeof(C) == 16) cp_async16(dst + sw<C>(j), field + (long long)j * N + line);
      else cp_async8(dst + sw<C>(j), field + (long long)j * N + line);
    }
  } else {
    const C *src = field + (long long)line * N;
    constexpr int per16 = 16 / (int)sizeof(C);  // elements per 16-byte chunk
    for (int c = threadIdx.x; c < N / per16; c += T)
      cp_async16(dst + sw<C>(c * per16), src + c * per16);
  }
}

template <typename C, int N, int T>
__device__ __forceinline__ void store_line(const C *src, C *field, int line, bool strided) {
  if (strided) {
    for (int j = threadIdx.x; j < N; j += T) field[(long long)j * N + line] = src[sw<C>(j)];
  } else {
    C *dst = field + (long long)line * N;
    for (int j = threadIdx.x; j < N; j += T) dst[j] = src[sw<C>(j)];
  }
}

// Persistent CTAs walk the n lines of one pass.  Variants (the same
// arithmetic per radix; radix 16 changes the FFT's rounding pattern, within
// the parity tolerance):
//   DB = true : two line buffers; the copy of the next line is in flight while
//               the current one is transformed; twiddles and kx^2 in shared
//               memory (one CTA per SM at large n);
//   DB = false: one line buffer, twiddles and kx^2 read through L1, registers
//               capped so that two CTAs share an SM and overlap each other's
//               copies;
//   MAXR = 16 : radix-16 Stockham passes (three passes for 4096 points),
//               N/16 threads per line, single buffer.
// The launcher times the variants on the first steps and keeps the fastest.
template <typename R, int N, int T, bool DB, int MAXR>
__global__ void __launch_bounds__(T, (DB || MAXR == 16 || T >= 1024) ? 1 : 2)
    fft3d_pass_kernel(const Fft3dPass q, const double *__restrict__ gkx2,
                      const Tw<typename Cx<R>::T> *__restrict__ gtw) {
  using C = typename Cx<R>::T;
  using W = Tw<C>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf0 = reinterpret_cast<C *>(smem_raw);
  C *buf1 = DB ? buf0 + N : buf0;
  W *stw = reinterpret_cast<W *>(buf0 + (DB ? 2 * N : N));
  double *skx2 = reinterpret_cast<double *>(stw + N);
  C *field = reinterpret_cast<C *>(q.field);
  const bool strided = q.mode == 1;
  const int tid = threadIdx.x;
  const W *tw = gtw;
  const double *kx2 = gkx2;

  int line = blockIdx.x;
  if (line < N) load_line<C, N, T>(buf0, field, line, strided);
  cp_async_commit();
  if constexpr (DB) {
    for (int i = tid; i < N; i += T) stw[i] = gtw[i];
    if (strided)
      for (int i = tid; i < N; i += T) skx2[i] = gkx2[i];
    tw = stw;
    kx2 = skx2;
  }
  const double inv_norm = 1.0 / q.norm;  // n*n is a power of two: exact
  C *save = reinterpret_cast<C *>(q.save);

  for (int it = 0; line < N; ++it, line += gridDim.x) {
    C *u = (it & 1) ? buf1 : buf0;
    C *nxt = (it & 1) ? buf0 : buf1;
    const int next = line + gridDim.x;
    if constexpr (DB) {
      if (next < N) load_line<C, N, T>(nxt, field, next, strided);
      cp_async_commit();
      cp_async_wait1();
    } else {
      asm volatile("cp.async.wait_all;\n" ::: "memory");
    }
    __syncthreads();

    if (q.mode == 1) {
      fft_smem<C, N, T, -1, MAXR>(u, tw, tid);
      const double ky = kfreq(line, N, q.two_pi, q.stepn_y);
      const double ky2 = __dmul_rn(ky, ky);
      for (int j = tid; j < N; j += T) u[sw<C>(j)] = prop3(q, u[sw<C>(j)], kx2[j], ky2, j, line);
      __syncthreads();
      fft_smem<C, N, T, +1, MAXR>(u, tw, tid);
    } else {
      if (q.mode >= 2) {
        fft_smem<C, N, T, +1, MAXR>(u, tw, tid);
        for (int j = tid; j < N; j += T) {
          const C v = refract3<R>(q, u[sw<C>(j)], line, j, inv_norm);
          u[sw<C>(j)] = v;
          if (save) save[(long long)line * N + j] = v;
        }
        __syncthreads();
      }
      if (q.mode != 3) fft_smem<C, N, T, -1, MAXR>(u, tw, tid);
    }
    store_line<C, N, T>(u, field, line, strided);
    __syncthreads();  // the buffer is refilled next
    if constexpr (!DB) {
      if (next < N) load_line<C, N, T>(u, field, next, strided);
      cp_async_commit();
    }
  }
  cp_async_commit();
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// x pass over W adjacent lines at a time: the strided lines are columns of
// the field, so W adjacent columns make each row's segment W elements long
// (32 bytes: W = 2 for complex128, 4 for complex64) and every DRAM/L2 sector
// a copy touches is used whole; the W transforms share each pass (ILP W).
// Line w sits at w*LD, LD = N + 1 (complex128) or N + 4 (complex64)
// elements, so that the W threads staging one row land in different banks;
// twiddles and kx^2 are loaded into shared memory once per CTA.
template <typename C, int N>
constexpr int xpass_ld() { return N + (sizeof(C) == 16 ? 1 : 4); }

template <typename R, int N, int T, int W>
__global__ void __launch_bounds__(T, 1) fft3d_xpass_w_kernel(const Fft3dPass q,
                                                            const double *__restrict__ gkx2,
                                                            const Tw<typename Cx<R>::T> *__restrict__ gtw) {
  using C = typename Cx<R>::T;
  constexpr int LD = xpass_ld<C, N>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Tw<C> *tw = reinterpret_cast<Tw<C> *>(smem_raw);
  double *kx2 = reinterpret_cast<double *>(tw + N);
  C *u = reinterpret_cast<C *>(kx2 + N);
  C *field = reinterpret_cast<C *>(q.field);
  const int tid = threadIdx.x;
  for (int i = tid; i < N; i += T) {
    tw[i] = gtw[i];
    kx2[i] = gkx2[i];
  }
  constexpr int NBLK = N / W;
  for (int blk = blockIdx.x; blk < NBLK; blk += gridDim.x) {
    const int line0 = blk * W;
    // element (j, w): field[j*N + line0 + w] -> u[w*LD + sw(j)]; w fastest
    for (int idx = tid; idx < W * N; idx += T) {
      const int w = idx % W, j = idx / W;
      if constexpr (sizeof(C) == 16) cp_async16(u + w * LD + sw<C>(j), field + (long long)j * N + line0 + w);
      else cp_async8(u + w * LD + sw<C>(j), field + (long long)j * N + line0 + w);
    }
    cp_async_commit();
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    fft_smem_w<C, N, T, -1, W, LD>(u, tw, tid);
#pragma unroll
    for (int w = 0; w < W; ++w) {
      const double ky = kfreq(line0 + w, N, q.two_pi, q.stepn_y);
      const double ky2 = __dmul_rn(ky, ky);
      for (int j = tid; j < N; j += T)
        u[w * LD + sw<C>(j)] = prop3(q, u[w * LD + sw<C>(j)], kx2[j], ky2, j, line0 + w);
    }
    __syncthreads();
    fft_smem_w<C, N, T, +1, W, LD>(u, tw, tid);
    for (int idx = tid; idx < W * N; idx += T) {
      const int w = idx % W, j = idx / W;
      field[(long long)j * N + line0 + w] = u[w * LD + sw<C>(j)];
    }
    __syncthreads();  // the buffer is refilled next
  }
}

template <typename R, int N>
static cudaError_t fft3d_xpass_w_launch(const Fft3dPass &q, const double *kx2, const void *twv,
                                        cudaStream_t s) {
  using C = typename Cx<R>::T;
  const Tw<C> *tw = reinterpret_cast<const Tw<C> *>(twv);
  constexpr int W = 32 / (int)sizeof(C);
  constexpr int T = N / 8 < 32 ? 32 : (N / 8 > 1024 ? 1024 : N / 8);
  constexpr size_t smem = sizeof(double2) * N + sizeof(double) * N + sizeof(C) * W * xpass_ld<C, N>();
  static_assert(smem + 16 <= 227 * 1024, "wide x pass exceeds shared memory");
  auto k = fft3d_xpass_w_kernel<R, N, T, W>;
  {
    const cudaError_t e = raise_dynamic_smem((const void *)k, (int)smem);
    if (e != cudaSuccess) return e;
  }
  static int grid = 0;  // CTAs per wave (same SM count on every B200)
  if (grid == 0) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, T, smem);
    if (e != cudaSuccess) return e;
    grid = sms * (per > 0 ? per : 1);
  }
  k<<<grid < N / W ? grid : N / W, T, smem, s>>>(q, kx2, tw);
  return cudaGetLastError();
}

static bool fft3d_wide_x() {
  static const bool on = [] {
    const char *e = std::getenv("PXP_FFT3D_WIDE_X");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <int N, int MAXR> constexpr int pass_threads() {
  return N / MAXR < 32 ? 32 : (N / MAXR > 1024 ? 1024 : N / MAXR);
}

template <typename R, int N, bool DB, int MAXR>
static cudaError_t fft3d_launch_v(const Fft3dPass &q, const double *kx2, const void *twv,
                                  cudaStream_t s) {
  using C = typename Cx<R>::T;
  const Tw<C> *tw = reinterpret_cast<const Tw<C> *>(twv);
  constexpr int T = pass_threads<N, MAXR>();
  constexpr size_t smem = DB ? 2 * sizeof(C) * N + sizeof(double2) * N + sizeof(double) * N
                             : sizeof(C) * N;
  auto k = fft3d_pass_kernel<R, N, T, DB, MAXR>;
  {
    const cudaError_t e = raise_dynamic_smem((const void *)k, (int)smem);
    if (e != cudaSuccess) return e;
  }
  static int grid = 0;  // CTAs per wave (same SM count on every B200)
  if (grid == 0) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, T, smem);
    if (e != cudaSuccess) return e;
    grid = sms * (per > 0 ? per : 1);
  }
  k<<<grid < N ? grid : N, T, smem, s>>>(q, kx2, tw);
  return cudaGetLastError();
}

template <typename R, int N>
static cudaError_t fft3d_launch_n(const Fft3dPass &q, int variant, const double *kx2,
                                  const void *tw16, cudaStream_t s) {
  using C = typename Cx<R>::T;
  const void *tw8 = q.twiddle;
  // x pass: W adjacent columns per CTA where their buffer fits
  // (measured: faster from 1024 points, slower at 512)
  constexpr bool wide_fits = N >= 1024 && N <= 4096;
  if constexpr (wide_fits)
    if (q.mode == 1 && fft3d_wide_x()) return fft3d_xpass_w_launch<R, N>(q, kx2, tw8, s);
  // two line buffers plus tables exceed a CTA's shared memory above 4096
  // points (FP64) / 8192 (FP32): the single-buffer form stands in
  constexpr bool db_fits = (2 * sizeof(C) + sizeof(double2) + sizeof(double)) * N <= 227 * 1024;
  if constexpr (db_fits)
    if (variant == 0) return fft3d_launch_v<R, N, true, 8>(q, kx2, tw8, s);
  if (variant <= 1) return fft3d_launch_v<R, N, false, 8>(q, kx2, tw8, s);
  return fft3d_launch_v<R, N, false, 16>(q, kx2, tw16, s);
}

int fft1d_bluestein_m(int n);

bool fft3d_supported(Precision p, int n) {
  if (n & (n - 1))  // Bluestein line transforms (fft3d_blu.cu)
    return n >= 8 && fft1d_bluestein_m(n) <= (p == kFP64 ? 8192 : 16384);
  return n >= 64 && n <= 8192;
}

cudaError_t launch_fft3d_pass(Precision p, const Fft3dPass &q, int variant, const double *kx2,
                              const void *tw16, const void *wn, cudaStream_t s) {
  if (q.n & (q.n - 1)) return launch_fft3d_bluestein(p, q, kx2, s);
  if (variant == 3) {
    if (fft3d_lines_supported(p, q.n) && wn != nullptr) return launch_fft3d_lines(p, q, kx2, wn, s);
    variant = 0;
  }
  if (variant == 4 || variant == 5) {
    const bool single = variant == 5;
    if (fft3d_r16_supported(p, q.n, single) && wn != nullptr)
      return launch_fft3d_r16(p, q, kx2, wn, s, single);
    variant = 0;
  }
#define PXP_C3(NN)                                                                  \
  case NN:                                                                          \
    return p == kFP64 ? fft3d_launch_n<double, NN>(q, variant, kx2, tw16, s) \
                      : fft3d_launch_n<float, NN>(q, variant, kx2, tw16, s);
  switch (q.n) {
    PXP_C3(64) PXP_C3(128) PXP_C3(256) PXP_C3(512) PXP_C3(1024) PXP_C3(2048) PXP_C3(4096)
    PXP_C3(8192)
    default:
      return cudaErrorInvalidValue;
  }
#undef PXP_C3
}

}  // namespace pxp
