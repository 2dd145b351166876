// farfield.cu -- post::FarField on the device.
//
// The reference (src/farFieldPost.cpp:22-62, 141-247) pads each line of the
// exit field to L entries (FarField::setPadLength; the examples use 32768),
// transforms it with FFTW, fftshifts and keeps the window of angles that
// farFieldAngleToIndx (:78-101) gives.  3-D: every column of the field
// (minus the reference run's field) is transformed and cropped along y,
// then every row of that -- conjugated, as Armadillo's `.t()` of a complex
// row is -- is transformed and cropped along x, keeping |X|^2 / L.
//
// A padded line holds data in only n << L entries, so a transform of length
// L = P * Q with n <= Q splits into P transforms of length Q:
//   X[k1 + P k2] = sum_{j<n} (x_j w_L^{j k1}) w_Q^{j k2},   k1 < P, k2 < Q,
// each a shared-memory Stockham FFT of the line times a twiddle (pruned
// input, L log Q work instead of L log L, the line read from HBM once).  The
// fftshift and the angular window are applied as the outputs are written.
// Constant padding (the padded entries equal a value c) is handled by
// linearity: padded = c + (x - c) on the data, so X = c L [k = 0] + DFT of
// (x - c).  The same identity places the 2-D exit field in the middle of the
// padded line: a shift changes only the phase of X, and the 2-D far field
// keeps |X|.
//
// A direct DFT (one output per thread, exact integer index j k mod L into an
// L-entry twiddle table) covers lengths that are not powers of two and
// windows narrow enough that computing only the kept outputs is cheaper.
#include "fft_smem.cuh"
#include "pxp_complex.cuh"
#include "pxp_kernels.h"

namespace pxp {

namespace {

__device__ __forceinline__ double2 ff_load(const FarFieldLines &p, long long line, int j) {
  const long long off = line * p.line_stride + j;
  double2 v = p.in_c64 ? to_d(reinterpret_cast<const float2 *>(p.in)[off])
                       : reinterpret_cast<const double2 *>(p.in)[off];
  if (p.ref != nullptr) {
    const double2 r = p.ref[off];
    v = make_double2(v.x - r.x, v.y - r.y);
  }
  if (p.conj_in) v.y = -v.y;
  return v;
}

// Value of the padded entries of a line (see the header comment).
__device__ __forceinline__ double2 ff_pad(const FarFieldLines &p, long long line) {
  return p.pad_const ? ff_load(p, line, 0) : p.pad_value;
}

__device__ __forceinline__ void ff_store(const FarFieldLines &p, long long line, long long i,
                                         double2 X) {
  const long long o = line + (i - p.i0) * p.out_stride;
  if (p.mode == 0) {
    reinterpret_cast<double2 *>(p.out)[o] = X;
  } else {
    const double a = hypot(X.x, X.y);  // std::abs(complex)
    reinterpret_cast<double *>(p.out)[o] = p.mode == 1 ? a * a / p.divisor : a / p.divisor;
  }
}

// Index k of the unshifted transform that lands at i after fftshift
// (entry i swapped with i + L/2 for i < L/2; an odd length keeps its last
// entry in place).
__device__ __forceinline__ long long ff_unshift(long long i, long long L) {
  const long long h = L / 2;
  if (i < h) return i + h;
  if (i < 2 * h) return i - h;
  return i;
}

}  // namespace

// G lines per CTA, T threads, sub-transform length Q (power of two, n <= Q,
// Q | L); blockIdx.y selects a share of the k1 range.  With REG, each thread keeps its S = Q / T entries of (x - c) in
// registers for the P passes over k1; without (Q = 8192, where registers
// would spill), it reads them again each pass (from L2 after the first).
template <int Q, int T, int G, bool REG>
__global__ void __launch_bounds__(T) ff_pruned_kernel(FarFieldLines p) {
  constexpr int LD = Q + 1;
  constexpr int S = Q / T;
  constexpr int SR = REG ? S : 1;
  static_assert(S * T == Q, "Q must be a multiple of T");
  extern __shared__ double2 ff_smem[];
  double2 *x = ff_smem;
  // twiddle factors exp(-2 pi i m / L) as lo[m mod B] * hi[m / B], B = 2^split_bits:
  // two tables of about sqrt(L) entries each, held in shared memory
  const int sb = p.split_bits;
  const int nlo = 1 << sb, nhi = (int)(p.L >> sb);
  double2 *wlo = x + G * LD;
  double2 *whi = wlo + nlo;
  const int tid = threadIdx.x;
  for (int i = tid; i < nlo + nhi; i += T) wlo[i] = p.wsplit[i];
  const long long line0 = (long long)blockIdx.x * G;
  double2 c[G];
  double2 v[G][SR];
  auto src = [&](int g, int j) {
    const long long line = line0 + g;
    double2 a = make_double2(0.0, 0.0);
    if (line < p.nlines && j < p.n) {
      const double2 u = ff_load(p, line, j);
      a = make_double2(u.x - c[g].x, u.y - c[g].y);
    }
    return a;
  };
#pragma unroll
  for (int g = 0; g < G; ++g) {
    const long long line = line0 + g;
    c[g] = line < p.nlines ? ff_pad(p, line) : make_double2(0.0, 0.0);
    if constexpr (REG) {
#pragma unroll
      for (int s = 0; s < S; ++s) v[g][s] = src(g, tid + s * T);
    }
  }
  __syncthreads();  // the twiddle tables are in place
  const long long L = p.L, P = L / Q, h = L / 2, mask = L - 1;
  const long long win = p.i1 - p.i0 + 1;
  // blockIdx.y takes one contiguous share of the P sub-transforms
  const long long kchunk = (P + gridDim.y - 1) / gridDim.y;
  const long long k1_end = min(P, (long long)(blockIdx.y + 1) * kchunk);
  for (long long k1 = (long long)blockIdx.y * kchunk; k1 < k1_end; ++k1) {
    // outputs of this k1 sit at i = (k1 + P k2 + h) mod L: one residue class mod P
    if (win < P) {
      const long long r = (k1 + h) % P;
      const long long first = p.i0 + ((r - p.i0 % P) % P + P) % P;
      if (first > p.i1) continue;
    }
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int j = tid + s * T;
      const long long m = ((long long)j * k1) & mask;
      const double2 w = cmul(whi[m >> sb], wlo[m & (nlo - 1)]);
#pragma unroll
      for (int g = 0; g < G; ++g) {
        double2 a;
        if constexpr (REG) a = v[g][s]; else a = src(g, j);
        x[g * LD + sw<double2>(j)] = cmul(a, w);
      }
    }
    __syncthreads();
    fft_smem_w<double2, Q, T, -1, G, LD>(x, p.twQ, tid);
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int k2 = tid + s * T;
      const long long k = k1 + P * k2;
      const long long i = (k + h) & mask;
      if (i < p.i0 || i > p.i1) continue;
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const long long line = line0 + g;
        if (line >= p.nlines) continue;
        double2 X = x[g * LD + sw<double2>(k2)];
        if (k == 0) X = make_double2(X.x + c[g].x * (double)L, X.y + c[g].y * (double)L);
        ff_store(p, line, i, X);
      }
    }
    __syncthreads();
  }
}

// One line per blockIdx.x, T consecutive outputs per blockIdx.y; the line
// (minus its pad value) staged in shared memory when it fits.
template <int T, bool STAGED>
__global__ void __launch_bounds__(T) ff_direct_kernel(FarFieldLines p) {
  extern __shared__ double2 ff_smem[];
  const long long line = blockIdx.x;
  const double2 c = ff_pad(p, line);
  if (STAGED) {
    for (int j = threadIdx.x; j < p.n; j += T) {
      const double2 u = ff_load(p, line, j);
      ff_smem[j] = make_double2(u.x - c.x, u.y - c.y);
    }
    __syncthreads();
  }
  const long long i = p.i0 + (long long)blockIdx.y * T + threadIdx.x;
  if (i > p.i1) return;
  const long long L = p.L;
  const long long k = ff_unshift(i, L);
  double2 acc = make_double2(0.0, 0.0);
  long long m = 0;  // j k mod L
  for (int j = 0; j < p.n; ++j) {
    double2 u;
    if (STAGED) {
      u = ff_smem[j];
    } else {
      const double2 a = ff_load(p, line, j);
      u = make_double2(a.x - c.x, a.y - c.y);
    }
    acc = cfma(u, p.wL[m], acc);
    m += k;
    if (m >= L) m -= L;
  }
  if (k == 0) acc = make_double2(acc.x + c.x * (double)L, acc.y + c.y * (double)L);
  ff_store(p, line, i, acc);
}

// PostProcessingModule::resizeMatrix (src/postProcessing.cpp:29-49): export
// cell (j, i) is the mean of the column means of the block with inclusive
// bounds (j dY .. (j+1) dY, i dX .. (i+1) dX), each truncated to an index.
// Column means add even and odd entries in two sums, as Armadillo's mean
// does.
__global__ void ff_resize_kernel(const double *__restrict__ in, long long rows, double *__restrict__ out,
                                 int er, int ec, double dY, double dX) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)er * ec) return;
  const int j = (int)(idx % er), i = (int)(idx / er);
  const long long r0 = (long long)(j * dY), r1 = (long long)((j + 1) * dY);
  const long long c0 = (long long)(i * dX), c1 = (long long)((i + 1) * dX);
  const long long nr = r1 - r0 + 1, nc = c1 - c0 + 1;
  double a1 = 0.0, a2 = 0.0;
  long long q = 0;
  for (long long col = c0; col <= c1; ++col, ++q) {
    const double *colp = in + col * rows + r0;
    double s1 = 0.0, s2 = 0.0;
    long long r = 0;
    for (; r + 1 < nr; r += 2) {
      s1 += colp[r];
      s2 += colp[r + 1];
    }
    if (r < nr) s1 += colp[r];
    const double m = (s1 + s2) / (double)nr;
    if (q & 1) a2 += m; else a1 += m;
  }
  out[j + (long long)i * er] = (a1 + a2) / (double)nc;
}

__global__ void ff_widen_kernel(const float2 *__restrict__ in, double2 *__restrict__ out, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = to_d(in[i]);
}

namespace {

template <int Q, int T, int G>
cudaError_t ff_pruned_launch(const FarFieldLines &p, cudaStream_t s) {
  constexpr bool REG = Q <= 4096;
  const size_t smem =
      sizeof(double2) * (G * (Q + 1) + (1LL << p.split_bits) + (p.L >> p.split_bits));
  cudaError_t e = cudaFuncSetAttribute(ff_pruned_kernel<Q, T, G, REG>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long long blocks = (p.nlines + G - 1) / G;
  // few lines (or many sub-transforms per line): split each line's
  // sub-transforms over blockIdx.y until about 8 CTAs per SM are in flight
  const long long P = p.L / Q;
  long long ky = (148LL * 8 + blocks - 1) / blocks;
  ky = ky < 1 ? 1 : (ky > P ? P : ky);
  ff_pruned_kernel<Q, T, G, REG><<<dim3((unsigned)blocks, (unsigned)ky), T, smem, s>>>(p);
  return cudaGetLastError();
}

}  // namespace

int farfield_split_bits(long long L) {
  int lg = 0;
  while ((1LL << lg) < L) ++lg;
  return (lg + 1) / 2;
}

int farfield_pruned_q(long long n, long long L) {
  long long q = 64;
  while (q < n) q *= 2;
  if (q > L || q > 8192 || (L & (L - 1)) != 0 || L % q != 0) return 0;
  return (int)q;
}

cudaError_t launch_farfield_lines(const FarFieldLines &p, int q, cudaStream_t s) {
  if (p.nlines <= 0 || p.i1 < p.i0) return cudaSuccess;
  switch (q) {
    case 0: break;
    case 64: return ff_pruned_launch<64, 64, 2>(p, s);
    case 128: return ff_pruned_launch<128, 64, 2>(p, s);
    case 256: return ff_pruned_launch<256, 64, 2>(p, s);
    case 512: return ff_pruned_launch<512, 64, 2>(p, s);
    case 1024: return ff_pruned_launch<1024, 128, 2>(p, s);
    case 2048: return ff_pruned_launch<2048, 256, 2>(p, s);
    case 4096: return ff_pruned_launch<4096, 512, 1>(p, s);
    case 8192: return ff_pruned_launch<8192, 1024, 1>(p, s);
    default: return cudaErrorInvalidValue;
  }
  constexpr int T = 256;
  const long long win = p.i1 - p.i0 + 1;
  const dim3 grid((unsigned)p.nlines, (unsigned)((win + T - 1) / T));
  const size_t smem = sizeof(double2) * (size_t)p.n;
  if (smem <= 160 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(ff_direct_kernel<T, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    ff_direct_kernel<T, true><<<grid, T, smem, s>>>(p);
  } else {
    ff_direct_kernel<T, false><<<grid, T, 0, s>>>(p);
  }
  return cudaGetLastError();
}

cudaError_t launch_resize(const double *in, long long rows, double *out, int er, int ec, double dY,
                          double dX, cudaStream_t s) {
  const long long n = (long long)er * ec;
  if (n <= 0) return cudaSuccess;
  ff_resize_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(in, rows, out, er, ec, dY, dX);
  return cudaGetLastError();
}

cudaError_t launch_widen(const void *in, void *out, long long n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const long long b = (n + 255) / 256;
  ff_widen_kernel<<<(unsigned)(b < 148 * 8 ? b : 148 * 8), 256, 0, s>>>(
      (const float2 *)in, (double2 *)out, n);
  return cudaGetLastError();
}

}  // namespace pxp
