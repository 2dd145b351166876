// fft3d_r16.cu -- FFTSolver3D line passes with 16 points per thread
// (n = 512 .. 4096), two line slots per CTA.
//
// The step is the two-pass scheme of fft3d.cu (src/fftSolver3D.cpp:52-156):
//   x pass (mode 1): lines of fixed y (stride n): F_x, * K(kx, ky), F_x^-1
//   y pass (mode 2): contiguous lines of fixed x: F_y^-1, refraction, F_y
// (mode 0: F_y only; mode 3: F_y^-1 and refraction only).  What this
// variant changes is how much shared memory a transform moves, the resource
// that bounds the register-resident line kernels:
//
//  * Thread j of a line slot holds the 16 points j + s*n/16 (s = 0..15) in
//    registers.  A transform is a first pass of radix R0 = 16, 8, 4 or 2 on
//    the thread's own points (n = R0 * 16^k; 16/R0 butterflies, no
//    twiddles) and k radix-16 Stockham passes, so a 4096-point transform
//    crosses shared memory twice (radix 8 needs three crossings).  The last
//    pass leaves thread j with outputs j + r*n/16 in natural order, the
//    first pass's inputs of the next transform: the forward and inverse
//    transforms meet in registers, and lines are loaded from and stored to
//    global memory straight from registers (no staging copy through shared
//    memory).
//  * An exchange element is 16 bytes: one complex128 point, or the same
//    point of two adjacent lines in complex64 (a complex64 thread carries
//    two lines, which also makes each strided x-pass access 16 contiguous
//    bytes).  The exchange buffer is XOR-swizzled, element i at
//    i ^ (((i >> 3) ^ (i >> 4)) & 7), so that every access of 8 consecutive
//    threads -- the reads at stride 1, the first-pass writes at stride 16,
//    8, 4 or 2, the radix-16 passes' writes -- hits 8 different 16-byte bank
//    groups.
//  * Twiddles come from a shared table in pass order (entry (r-1)*NS + k of
//    the pass with sub-transform length NS), built once per CTA from the
//    exp(-2 pi i m / n) table; a complex64 thread applies each twiddle to
//    both of its lines.
//  * A CTA holds two line slots with their own exchange buffers and named
//    barriers, each walking its own sequence of lines: while one slot waits
//    for its loads or a barrier, the other computes.  No copy is
//    asynchronous, so nothing waits on an mbarrier.
//
// Per-point arithmetic (propagator, refraction, absorber, save) is
// fft3d_point.cuh's, shared with the other FFTSolver3D kernels.  The
// transforms round like the radix-16 variant of fft3d.cu up to the order of
// their passes (within the parity tolerance); complex64 data compute in FP32
// with split twiddles and constants (fft_smem.cuh).
#include <cuda.h>

#include <cstring>

#include "bulk_copy.cuh"
#include "fft3d_point.cuh"
#include "fft_r16.cuh"

namespace pxp {

// waits of the radix-16 line kernel that ran out on this device, read by
// the host
__device__ unsigned int g_r16_wait_timeouts = 0;

cudaError_t encode_field_tmap(void *field, int n, int real_bytes, int box_reals, int box_rows,
                              CUtensorMap *out);
namespace r16 {

using r16c::tw_offset;

// LP lines a slot (2 for complex64 by default, which makes every exchange
// element 16 bytes; 1 gives complex64 8-byte elements and half the
// registers), SL slots a CTA.
template <typename R, int N, int LP = (sizeof(typename Cx<R>::T) == 8 ? 2 : 1), int SL = 2>
struct Cfg {
  using C = typename Cx<R>::T;
  static constexpr int TL = N / 16;                       // threads per slot
  static constexpr int S = SL;                            // line slots per CTA
  static constexpr int T = S * TL;                        // threads per CTA
  static constexpr int LPT = LP;                          // lines per slot
  static constexpr int EB = (int)sizeof(C) * LP;          // exchange element bytes
  static constexpr int R0 = r16c::Plan<N>::R0;             // first-pass radix
  static constexpr int NP16 = r16c::Plan<N>::NP16;         // radix-16 passes
  static constexpr int TWN = r16c::Plan<N>::TWN;           // twiddle entries
  static constexpr int GROUPS = N / LPT;                  // line groups per pass
  static constexpr size_t XBYTES = (size_t)EB * N;        // one slot's buffer
  // FP64 keeps kx^2 per column in shared memory for the x pass
  static constexpr size_t KXBYTES = sizeof(R) == 8 ? 8 * (size_t)N : 0;
  // x lines by TMA tiles (loads into and stores from the slot's buffer)
  // where an exchange element is 16 bytes
  static constexpr bool XTMA = EB == 16;
  static constexpr size_t SMEM = 128 + S * XBYTES + 16 * (size_t)TWN + KXBYTES + 16 * S;
  static constexpr int BOX = N < 256 ? N : 256;  // rows of one L2 prefetch tile
  // lines one prefetch tile covers (16-byte rows: complex64 single lines are
  // prefetched in pairs)
  static constexpr int PFL = EB == 8 ? 2 : LP;
  // CTAs per SM: as many as shared memory holds, at most 128 registers a
  // thread
  static constexpr int SMEM_FIT = (int)((227 * 1024) / SMEM);
  static constexpr int RPT = EB == 8 ? 64 : 128;          // registers a thread
  static constexpr int REG_FIT = 65536 / (T * RPT);
  static constexpr int MINB = SMEM_FIT < REG_FIT ? SMEM_FIT : REG_FIT;
  static_assert(N % 16 == 0 && TL % 32 == 0, "whole warps per slot");
};

// Exchange-buffer position of element i (elements of EB bytes).
template <int EB> __device__ __forceinline__ int xsw(int i) { return r16c::xsw<EB>(i); }

__device__ __forceinline__ void slot_sync(int slot, int count) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(1 + slot), "r"(count) : "memory");
}

// Exchange element of a thread's LPT lines at one position.
template <typename C, int LP> struct Xe;
template <> struct Xe<double2, 1> {
  using T = double2;
  static __device__ __forceinline__ T pack(const double2 (&v)[1][16], int s) { return v[0][s]; }
  static __device__ __forceinline__ void unpack(double2 (&v)[1][16], int s, T e) { v[0][s] = e; }
};
template <> struct Xe<float2, 1> {
  using T = float2;
  static __device__ __forceinline__ T pack(const float2 (&v)[1][16], int s) { return v[0][s]; }
  static __device__ __forceinline__ void unpack(float2 (&v)[1][16], int s, T e) { v[0][s] = e; }
};
template <> struct Xe<float2, 2> {
  using T = float4;
  static __device__ __forceinline__ T pack(const float2 (&v)[2][16], int s) {
    return make_float4(v[0][s].x, v[0][s].y, v[1][s].x, v[1][s].y);
  }
  static __device__ __forceinline__ void unpack(float2 (&v)[2][16], int s, T e) {
    v[0][s] = make_float2(e.x, e.y);
    v[1][s] = make_float2(e.z, e.w);
  }
};


// Radix-16 passes P .. NP16-1 of a transform: read the pass's inputs
// j + r*TL, twiddles W_{16 NS}^(r k) (k = j mod NS), 16-point DFT, write the
// outputs to (j - k)*16 + k + r*NS -- except the last pass, which keeps
// them in registers (natural order).
template <int SIGN, typename R, int N, int LP, int SL, int P>
__device__ __forceinline__ void r16_passes(typename Cx<R>::T (&v)[LP][16],
                                           typename Xe<typename Cx<R>::T, LP>::T *X,
                                           const Tw<typename Cx<R>::T> *tws, int slot, int j) {
  using K = Cfg<R, N, LP, SL>;
  using C = typename Cx<R>::T;
  using E = Xe<C, LP>;
  if constexpr (P < K::NP16) {
    constexpr int NS = K::R0 << (4 * P);
    constexpr int OFF = tw_offset<K::R0, P>();
    slot_sync(slot, K::TL);  // the writes of the previous pass are done
#pragma unroll
    for (int r = 0; r < 16; ++r) E::unpack(v, r, X[xsw<K::EB>(j + r * K::TL)]);
    const int k = j & (NS - 1);
#pragma unroll
    for (int r = 1; r < 16; ++r) {
      const Tw<C> w = tws[OFF + (r - 1) * NS + k];
#pragma unroll
      for (int t = 0; t < K::LPT; ++t)
        v[t][r] = SIGN < 0 ? tw_mul(v[t][r], w) : tw_mulc(v[t][r], w);
    }
#pragma unroll
    for (int t = 0; t < K::LPT; ++t) dft16<SIGN>(v[t]);
    if constexpr (P < K::NP16 - 1) {
      slot_sync(slot, K::TL);  // every read of this pass is done
      const int base = (j - k) * 16 + k;
#pragma unroll
      for (int r = 0; r < 16; ++r) X[xsw<K::EB>(base + r * NS)] = E::pack(v, r);
    }
    r16_passes<SIGN, R, N, LP, SL, P + 1>(v, X, tws, slot, j);
  }
}

// One transform of the thread's LPT lines, points v[t][s] = j + s*TL before
// and after (natural order).  X: the slot's exchange buffer; every write to
// it follows a barrier that ends the previous reads, every read follows the
// barrier that ends the writes.
template <int SIGN, typename R, int N, int LP, int SL>
__device__ __forceinline__ void line_fft(typename Cx<R>::T (&v)[LP][16],
                                         typename Xe<typename Cx<R>::T, LP>::T *X,
                                         const Tw<typename Cx<R>::T> *tws, int slot, int j) {
  using K = Cfg<R, N, LP, SL>;
  using C = typename Cx<R>::T;
  using E = Xe<C, LP>;
  constexpr int TL = K::TL, R0 = K::R0;
  // first pass: radix R0 over the thread's own points; butterfly
  // b = j + u*TL takes points s = u + r*(16/R0) and writes b*R0 + r
#pragma unroll
  for (int t = 0; t < K::LPT; ++t) r16c::first_pass<SIGN, R0>(v[t]);
  slot_sync(slot, TL);  // the previous reads of X are done
#pragma unroll
  for (int u = 0; u < 16 / R0; ++u)
#pragma unroll
    for (int r = 0; r < R0; ++r) X[xsw<K::EB>((j + u * TL) * R0 + r)] = E::pack(v, u + r * (16 / R0));
  r16_passes<SIGN, R, N, LP, SL, 0>(v, X, tws, slot, j);
}

template <typename R, int N, int LP, int SL>
__global__ void __launch_bounds__(Cfg<R, N, LP, SL>::T, Cfg<R, N, LP, SL>::MINB)
    fft3d_r16_kernel(const __grid_constant__ Fft3dPass q,
                     const __grid_constant__ CUtensorMap tmap, const double *__restrict__ gkx2,
                     const Tw<typename Cx<R>::T> *__restrict__ wn) {
  using K = Cfg<R, N, LP, SL>;
  using C = typename Cx<R>::T;
  using E = Xe<C, LP>;
  using W = Tw<C>;
  constexpr int TL = K::TL, LPT = K::LPT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  const int tid = threadIdx.x;
  const int slot = tid / TL, j = tid % TL;
  typename E::T *X = reinterpret_cast<typename E::T *>(base + slot * K::XBYTES);
  W *tws = reinterpret_cast<W *>(base + K::S * K::XBYTES);
  double *skx2 = reinterpret_cast<double *>(base + K::S * K::XBYTES + 16 * (size_t)K::TWN);
  uint64_t *sbar = reinterpret_cast<uint64_t *>(base + K::S * K::XBYTES + 16 * (size_t)K::TWN +
                                                K::KXBYTES) + 2 * slot;
  __shared__ int slot_fail[K::S];
  if (j == 0) {
    mbar_init(sbar, 1);
    slot_fail[slot] = 0;
  }
  // twiddles of every radix-16 pass: entry off + (r-1)*NS + k = W_{16 NS}^(r k)
  r16c::load_twiddles<N>(tws, wn, tid, K::T);
  if constexpr (sizeof(R) == 8) {
    if (q.mode == 1 && q.prop_x == nullptr)  // FP64's joint argument per point
      for (int i = tid; i < N; i += K::T) skx2[i] = gkx2[i];
  }
  __syncthreads();
  // the field is read only after the previous kernel in the stream is done
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");

  const bool xpass = q.mode == 1;
  C *field = reinterpret_cast<C *>(q.field);
  C *save = reinterpret_cast<C *>(q.save);
  const double inv_norm = 1.0 / q.norm;  // n*n is a power of two: exact
  const bool scale_only = refract3_is_scale(q, inv_norm);
  const int nslots = gridDim.x * K::S;
  // L2 prefetch of a slot's lines (one thread each): the y lines of a group
  // are one contiguous block; the x lines are columns, N/BOX tiles of the
  // tensor map (16-byte rows: one complex128 column, or two complex64)
  auto prefetch = [&](int gp) {
    if (gp >= K::GROUPS) return;
    if (xpass) {
      for (int b = 0; b < N / K::BOX; ++b)
        asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];\n" ::"l"(&tmap),
                     "r"(2 * ((gp * LPT) & ~(K::PFL - 1))), "r"(b * K::BOX)
                     : "memory");
    } else {
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(field + (long long)gp * LPT * N),
                   "r"((unsigned)(sizeof(C) * LPT * N))
                   : "memory");
    }
  };
  if (j == 0) prefetch(blockIdx.x * K::S + slot);
  int it = 0;
  for (int g = blockIdx.x * K::S + slot; g < K::GROUPS; g += nslots, ++it) {
    const int line0 = g * LPT;
    if (j == 0) prefetch(g + nslots);  // this slot's next group, while this one computes
    C v[LPT][16];
    if (K::XTMA && xpass) {
      // the columns arrive by N/BOX TMA tiles into the slot's buffer, in
      // natural order (element e at X[e]), once every thread of the slot is
      // past its reads of the buffer; one thread arms the slot's mbarrier
      // and waits (bounded), a slot barrier publishes the line
      slot_sync(slot, TL);
      if (j == 0) {
        mbar_arrive_expect_tx(sbar, (unsigned)(K::EB * N));
        const unsigned dst = smem_u32(X);
        for (int b = 0; b < N / K::BOX; ++b)
          asm volatile(
              "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
              " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst + (unsigned)(b * K::BOX * K::EB)),
              "l"(&tmap), "r"(2 * line0), "r"(b * K::BOX), "r"(smem_u32(sbar))
              : "memory");
        if (!mbar_wait_bounded(sbar, it & 1, 2000000000ull)) {
          atomicAdd(&g_r16_wait_timeouts, 1u);
          mbar_wait_bounded(sbar, it & 1, 2000000000ull);  // the copy may still be in flight
          slot_fail[slot] = 1;
        }
      }
      slot_sync(slot, TL);
      if (slot_fail[slot]) break;
      (void)mbar_try_wait(sbar, it & 1);  // completed phase: orders the line for this thread
#pragma unroll
      for (int s = 0; s < 16; ++s) E::unpack(v, s, X[j + s * TL]);
    } else {
      // x lines are columns (element e of line l at e*N + l; a complex64
      // thread's two lines are adjacent), y lines are rows
#pragma unroll
      for (int s = 0; s < 16; ++s) {
        const int e = j + s * TL;
        if (xpass) {
          E::unpack(v, s,
                    *reinterpret_cast<const typename E::T *>(field + (long long)e * N + line0));
        } else {
#pragma unroll
          for (int t = 0; t < LPT; ++t) v[t][s] = field[(long long)(line0 + t) * N + e];
        }
      }
    }
    if (xpass) {
      line_fft<-1, R, N, LP, SL>(v, X, tws, slot, j);
      // propagator K = exp(-i a (kx^2 + ky^2)) (src/fftSolver3D.cpp:24-30, 87-120)
#pragma unroll
      for (int t = 0; t < LPT; ++t) {
        const int line = line0 + t;  // y index
        double ky2 = 0.0;
        if constexpr (sizeof(R) == 8) {
          const double ky = kfreq(line, N, q.two_pi, q.stepn_y);
          ky2 = __dmul_rn(ky, ky);
        }
#pragma unroll
        for (int s = 0; s < 16; ++s) {
          const int e = j + s * TL;
          v[t][s] = prop3(q, v[t][s], sizeof(R) == 8 ? skx2[e] : 0.0, ky2, e, line);
        }
      }
      line_fft<+1, R, N, LP, SL>(v, X, tws, slot, j);
    } else {
      if (q.mode >= 2) {
        line_fft<+1, R, N, LP, SL>(v, X, tws, slot, j);
        if (scale_only) {
#pragma unroll
          for (int t = 0; t < LPT; ++t)
#pragma unroll
            for (int s = 0; s < 16; ++s) v[t][s] = scale_point(v[t][s], inv_norm);
        } else {
          // material or absorber in this step: the thread's own points go
          // through its exchange-buffer slots (each thread touches only its
          // own, so the one barrier ends the other threads' last reads) and
          // one non-unrolled refract3 loop
          slot_sync(slot, TL);
#pragma unroll
          for (int s = 0; s < 16; ++s) X[xsw<K::EB>(j + s * TL)] = E::pack(v, s);
#pragma unroll 1
          for (int s = 0; s < 16; ++s) {
            const int e = j + s * TL;  // y index
            C w[LPT][16];
            E::unpack(w, 0, X[xsw<K::EB>(e)]);
#pragma unroll
            for (int t = 0; t < LPT; ++t) w[t][0] = refract3<R>(q, w[t][0], line0 + t, e, inv_norm);
            X[xsw<K::EB>(e)] = E::pack(w, 0);
          }
#pragma unroll
          for (int s = 0; s < 16; ++s) E::unpack(v, s, X[xsw<K::EB>(j + s * TL)]);
        }
        if (save) {
#pragma unroll
          for (int t = 0; t < LPT; ++t)
#pragma unroll
            for (int s = 0; s < 16; ++s) save[(long long)(line0 + t) * N + j + s * TL] = v[t][s];
        }
      }
      if (q.mode != 3) line_fft<-1, R, N, LP, SL>(v, X, tws, slot, j);
    }
    if (K::XTMA && xpass) {
      // the columns leave by TMA tile stores from the slot's buffer (natural
      // order) once every thread is past the last pass's reads; the issuing
      // thread waits until the copies have read the buffer before it joins
      // the next line's first slot barrier
      slot_sync(slot, TL);
#pragma unroll
      for (int s = 0; s < 16; ++s) X[j + s * TL] = E::pack(v, s);
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      slot_sync(slot, TL);
      if (j == 0) {
        const unsigned src = smem_u32(X);
        for (int b = 0; b < N / K::BOX; ++b)
          asm volatile(
              "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(
                  &tmap),
              "r"(2 * line0), "r"(b * K::BOX), "r"(src + (unsigned)(b * K::BOX * K::EB))
              : "memory");
        asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
        asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
      }
    } else {
#pragma unroll
      for (int s = 0; s < 16; ++s) {
        const int e = j + s * TL;
        if (xpass) {
          *reinterpret_cast<typename E::T *>(field + (long long)e * N + line0) = E::pack(v, s);
        } else {
#pragma unroll
          for (int t = 0; t < LPT; ++t) field[(long long)(line0 + t) * N + e] = v[t][s];
        }
      }
    }
  }
  // the slot's last tile stores complete before its threads leave
  if (j == 0) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
}

template <typename R, int N, int LP, int SL>
cudaError_t launch(const Fft3dPass &q, const double *kx2, const void *wnv, cudaStream_t s) {
  using K = Cfg<R, N, LP, SL>;
  using W = Tw<typename Cx<R>::T>;
  static_assert(K::SMEM <= 227 * 1024, "line slots exceed shared memory");
  auto k = fft3d_r16_kernel<R, N, LP, SL>;
  {
    const cudaError_t e = raise_dynamic_smem((const void *)k, (int)K::SMEM);
    if (e != cudaSuccess) return e;
  }
  // CTAs per wave, once per instantiation (the same SM count on every B200)
  static int per = 0, sms = 0;
  if (per == 0) {
    int dev = 0, p = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, k, K::T, K::SMEM);
    if (e != cudaSuccess) return e;
    per = p < 1 ? 1 : p;
  }
  const int ctas = (K::GROUPS + K::S - 1) / K::S;
  const int grid = ctas < sms * per ? ctas : sms * per;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(K::T);
  cfg.dynamicSmemBytes = K::SMEM;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // x pass: the tensor map of the field for the L2 prefetches (16-byte rows)
  CUtensorMap tmap;
  std::memset(&tmap, 0, sizeof(tmap));
  if (q.mode == 1) {
    const cudaError_t te = encode_field_tmap(q.field, N, (int)sizeof(R), 2 * K::PFL, K::BOX, &tmap);
    if (te != cudaSuccess) return te;
  }
  return cudaLaunchKernelEx(&cfg, k, q, tmap, kx2, reinterpret_cast<const W *>(wnv));
}

}  // namespace r16

unsigned fft3d_r16_wait_timeouts(cudaStream_t s) {
  unsigned v = 0;
  if (cudaMemcpyFromSymbolAsync(&v, g_r16_wait_timeouts, sizeof(v), 0, cudaMemcpyDeviceToHost,
                                s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return 0;
  return v;
}

bool fft3d_r16_supported(Precision p, int n, bool single) {
  if (single && p != kFP32) return false;
  return n >= 512 && n <= 4096 && !(n & (n - 1));
}

cudaError_t launch_fft3d_r16(Precision p, const Fft3dPass &q, const double *kx2, const void *wn,
                             cudaStream_t s, bool single) {
#define PXP_R16(NN)                                                                      \
  case NN:                                                                               \
    if (p == kFP64) return r16::launch<double, NN, 1, 2>(q, kx2, wn, s);                 \
    return single ? r16::launch<float, NN, 1, 4>(q, kx2, wn, s)                          \
                  : r16::launch<float, NN, 2, 2>(q, kx2, wn, s);
  switch (q.n) {
    PXP_R16(512) PXP_R16(1024) PXP_R16(2048) PXP_R16(4096)
    default:
      return cudaErrorInvalidValue;
  }
#undef PXP_R16
}

}  // namespace pxp
