// fft3d_lines.cu -- FFTSolver3D line passes with register-resident transforms
// and TMA-staged lines (n = 64 .. 4096).
//
// The step is the two-pass scheme of fft3d.cu (src/fftSolver3D.cpp:52-156):
//   x pass (mode 1): lines of fixed y (stride n): F_x, * K(kx, ky), F_x^-1
//   y pass (mode 2): contiguous lines of fixed x: F_y^-1, refraction, F_y
// (mode 0: F_y only; mode 3: F_y^-1 and refraction only).  What differs is
// where the data live while a line is transformed:
//
//  * Each line of n points belongs to n/8 threads; thread j holds the points
//    j + s*n/8 (s = 0..7) in registers.  A transform is a first pass of
//    radix R0 = 8, 4 or 2 (n = R0 * 8^k; no twiddles, the thread's 8 points
//    are exactly its butterflies' inputs) and k radix-8 Stockham passes.  In
//    every radix-8 pass thread j owns butterfly j, so its seven twiddles
//    W_n^(r * (j mod NS) * n/(8 NS)) are the same for every line: they are
//    read once per launch into registers, and no twiddle is read from memory
//    during the transforms.
//  * The last radix-8 pass leaves thread j holding outputs j + r*n/8 in
//    natural order -- the inputs of its first butterflies of the next
//    transform.  So the forward and inverse transforms of a pass meet in
//    registers (the propagator or the refraction is applied there), the line
//    is read from the staging buffer straight into registers and written to
//    global memory straight from them, and shared memory is touched only by
//    the exchanges between passes: two ping-pong buffers, one barrier per
//    pass.
//  * Lines arrive by TMA into a staging buffer while the previous line group
//    is transformed: a contiguous group of y lines is one bulk copy; a group
//    of x lines (adjacent rows of the column-major field) is n/256 tiles of
//    a 2-D tensor map over this GPU's own field (no multicast).  x lines
//    also leave by tile stores, from the exchange buffer the last pass
//    read (issued by one thread for the CTA, or, with one complex128 line a
//    group, by each warp for its own rows); y lines leave by coalesced
//    stores from registers.  One thread arms an mbarrier for the group's
//    bytes and issues the copies; it waits with a bounded wait (about 2 s;
//    a wait that runs out is counted, the copy drained and the CTA leaves)
//    and a CTA barrier publishes the line.
//
// A CTA holds LG line slots of n/8 threads; a complex64 thread carries two
// lines (the tensor tiles then start on 16-byte boundaries).  Per-point
// arithmetic (propagator factors or argument and sincos, refraction,
// absorber, save) is fft3d_point.cuh's, shared with fft3d.cu.  The
// transforms round like the other kernels' up to the order of their passes
// (within the parity tolerance); complex64 data compute in FP32 with split
// twiddles as fft_smem.cuh does.
#include <cuda.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "bulk_copy.cuh"
#include "fft3d_point.cuh"

namespace pxp {

// waits of these kernels that ran out on this device, read by the host
__device__ unsigned int g_lines_wait_timeouts = 0;

namespace lines {

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }

template <typename R, int N, int LG> struct Cfg {
  using C = typename Cx<R>::T;
  static constexpr int TL = N / 8;                          // threads per line
  static constexpr int T = TL * LG;                         // threads per CTA
  static constexpr int LPT = sizeof(C) == 8 ? 2 : 1;        // lines per thread
  static constexpr int L = LG * LPT;                        // lines per group
  static constexpr int LOG = ilog2c(N);
  static constexpr int R0 = LOG % 3 == 0 ? 8 : (LOG % 3 == 1 ? 2 : 4);
  static constexpr int NP8 = (LOG - ilog2c(R0)) / 3;        // radix-8 passes
  static constexpr int XS = N + 16 / (int)sizeof(C);        // exchange stride per line
  static constexpr int BC = N < 256 ? N : 256;              // tensor tile: positions
  static constexpr int GROUPS = N / L;
  // x pass stores by warp (one complex128 line a group, n >= 256): see the
  // kernel's epilogue
  static constexpr bool WARP_ST = L == 1 && N >= 256;
  static constexpr int BCS = 32;                            // rows a warp's tile store

  // radix-8 passes whose twiddles sit in registers: all of them, except at
  // 512 threads per CTA and for complex128 lines at 256, where only the
  // last pass's do and the earlier passes' -- few distinct values, 7 * NS
  // of them -- come from a small table in global memory
  // (Fft3dPass::tw_lines) through L1.  That keeps a thread at 128
  // registers: one CTA an SM at 512 threads, two at 256 (16 warps instead
  // of 8; complex64 lines, two a thread, would spill there); and outside
  // shared memory the table leaves the SM 60 KB of L1 (a 196 KB carve-out)
  // for it and the propagator's x factors
  static constexpr bool TW_TABLE = T >= 512 || (T == 256 && sizeof(C) == 16);
  static constexpr int TWR = TW_TABLE ? 1 : NP8;
  static constexpr int MINB = T == 256 && TW_TABLE ? 2 : 1;  // CTAs an SM
  static constexpr int TWS_N = [] {  // entries of that table
    int n = 0;
    for (int p = 0; p < NP8 - TWR; ++p) n += 7 * (R0 << (3 * p));
    return n;
  }();
  static constexpr size_t STAGE = sizeof(C) * (size_t)L * N;
  static constexpr size_t XBYTES = sizeof(C) * (size_t)L * XS;
  static constexpr size_t SMEM = 128 + STAGE + 2 * ((XBYTES + 127) & ~size_t(127)) + 128;
  static_assert(N % 8 == 0 && T <= 1024, "line slots");
};

template <typename C, typename W> __device__ __forceinline__ C twm(C v, W w, bool fwd) {
  return fwd ? tw_mul(v, w) : tw_mulc(v, w);
}

// First pass (NS = 1, radix R0) on the thread's 8 points j + s*n/8, result
// to exchange buffer X at the Stockham positions b*R0 + r of its butterflies
// b = j + q*n/8.
template <int SIGN, int R0, int TL, typename C>
__device__ __forceinline__ void first_pass(C (&v)[8], C *X, int j) {
  if constexpr (R0 == 8) {
    dft8<SIGN>(v);
#pragma unroll
    for (int r = 0; r < 8; ++r) X[sw<C>(8 * j + r)] = v[r];
  } else if constexpr (R0 == 4) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      C a = v[q], b = v[q + 2], c = v[q + 4], d = v[q + 6];
      dft4<SIGN>(a, b, c, d);
      const int b0 = 4 * (j + q * TL);
      X[sw<C>(b0)] = a;
      X[sw<C>(b0 + 1)] = b;
      X[sw<C>(b0 + 2)] = c;
      X[sw<C>(b0 + 3)] = d;
    }
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      C a = v[q], b = v[q + 4];
      dft2<SIGN>(a, b);
      const int b0 = 2 * (j + q * TL);
      X[sw<C>(b0)] = a;
      X[sw<C>(b0 + 1)] = b;
    }
  }
}

// Radix-8 pass with sub-transform length NS: thread j takes butterfly j
// (inputs j + r*n/8), twiddles tw[0..6], outputs to (j - k)*8 + k + r*NS,
// k = j mod NS; the last pass (NS = n/8) keeps them in registers.
template <int SIGN, int N, int NS, typename C>
__device__ __forceinline__ void r8_pass(C (&v)[8], const C *Xin, C *Xout, const Tw<C> (&tw)[7],
                                        int j) {
  constexpr int TL = N / 8;
#pragma unroll
  for (int r = 0; r < 8; ++r) v[r] = Xin[sw<C>(j + r * TL)];
#pragma unroll
  for (int r = 1; r < 8; ++r) v[r] = twm(v[r], tw[r - 1], SIGN < 0);
  dft8<SIGN>(v);
  if constexpr (NS < TL) {
    const int k = j & (NS - 1);
    const int base = (j - k) * 8 + k;
#pragma unroll
    for (int r = 0; r < 8; ++r) Xout[sw<C>(base + r * NS)] = v[r];
  }
}

// Offset of radix-8 pass P's entries in the shared twiddle table: entry
// off + (r - 1) * NS + k = W_n^(r k n / (8 NS)).
template <int R0, int P> __host__ __device__ constexpr int tws_offset() {
  int off = 0;
  for (int p = 0; p < P; ++p) off += 7 * (R0 << (3 * p));
  return off;
}

// The radix-8 passes P .. NP8-1 of a transform of this thread's LPT lines.
// Passes below NP8 - TWR take their twiddles from the shared table tws, the
// others from the registers twr (one set per pass, tw index P - (NP8 - TWR)).
template <int SIGN, typename R, int N, int LG, int P>
__device__ __forceinline__ void r8_passes(typename Cx<R>::T (&v)[Cfg<R, N, LG>::LPT][8],
                                          typename Cx<R>::T *X0, typename Cx<R>::T *X1, int &cur,
                                          const Tw<typename Cx<R>::T> (&twr)[Cfg<R, N, LG>::TWR][7],
                                          const Tw<typename Cx<R>::T> *tws, int slot, int j) {
  using K = Cfg<R, N, LG>;
  using C = typename Cx<R>::T;
  if constexpr (P < K::NP8) {
    constexpr int NS = K::R0 << (3 * P);
    constexpr int FIRST_REG = K::NP8 - K::TWR;
    Tw<C> tw[7];
    if constexpr (P >= FIRST_REG) {
#pragma unroll
      for (int r = 0; r < 7; ++r) tw[r] = twr[P - FIRST_REG][r];
    } else {
      const int k = j & (NS - 1);
#pragma unroll
      for (int r = 0; r < 7; ++r) tw[r] = tws[tws_offset<K::R0, P>() + r * NS + k];
    }
    const C *in = cur ? X1 : X0;
    C *out = cur ? X0 : X1;
#pragma unroll
    for (int t = 0; t < K::LPT; ++t) {
      const int off = (slot * K::LPT + t) * K::XS;
      r8_pass<SIGN, N, NS>(v[t], in + off, out + off, tw, j);
    }
    if constexpr (P < K::NP8 - 1) {
      cur ^= 1;
      __syncthreads();
    }
    r8_passes<SIGN, R, N, LG, P + 1>(v, X0, X1, cur, twr, tws, slot, j);
  }
}

// One transform of the LPT lines of this thread, points in v[t][0..7]
// before and after (natural order).  cur: the exchange buffer holding the
// current data (0 or 1, updated); every write goes to the other one, so one
// barrier per pass suffices.  hook() runs once, right after the first
// barrier (every thread has then consumed its inputs).
template <int SIGN, typename R, int N, int LG, typename Hook>
__device__ __forceinline__ void line_fft(typename Cx<R>::T (&v)[Cfg<R, N, LG>::LPT][8],
                                         typename Cx<R>::T *X0, typename Cx<R>::T *X1, int &cur,
                                         const Tw<typename Cx<R>::T> (&tw)[Cfg<R, N, LG>::TWR][7],
                                         const Tw<typename Cx<R>::T> *tws, int slot, int j, Hook hook) {
  using K = Cfg<R, N, LG>;
  using C = typename Cx<R>::T;
  C *out = cur ? X0 : X1;
#pragma unroll
  for (int t = 0; t < K::LPT; ++t)
    first_pass<SIGN, K::R0, K::TL>(v[t], out + (slot * K::LPT + t) * K::XS, j);
  cur ^= 1;
  __syncthreads();
  hook();
  r8_passes<SIGN, R, N, LG, 0>(v, X0, X1, cur, tw, tws, slot, j);
}

template <typename R, int N, int LG>
__global__ void __launch_bounds__(Cfg<R, N, LG>::T, Cfg<R, N, LG>::MINB)
    fft3d_lines_kernel(const __grid_constant__ Fft3dPass q, const __grid_constant__ CUtensorMap tmap,
                       const __grid_constant__ CUtensorMap tmap_st,
                       const double *__restrict__ gkx2,
                       const Tw<typename Cx<R>::T> *__restrict__ wn) {
  using K = Cfg<R, N, LG>;
  using C = typename Cx<R>::T;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  C *S = reinterpret_cast<C *>(base);
  C *X0 = reinterpret_cast<C *>(base + K::STAGE);
  C *X1 = reinterpret_cast<C *>(base + K::STAGE + ((K::XBYTES + 127) & ~size_t(127)));
  uint64_t *bar =
      reinterpret_cast<uint64_t *>(base + K::STAGE + 2 * ((K::XBYTES + 127) & ~size_t(127)));
  const Tw<C> *tws = reinterpret_cast<const Tw<C> *>(q.tw_lines);
  __shared__ int s_ok;

  const int tid = threadIdx.x;
  const int slot = tid / K::TL, j = tid % K::TL;
  const bool xpass = q.mode == 1;
  C *field = reinterpret_cast<C *>(q.field);
  C *save = reinterpret_cast<C *>(q.save);

  // twiddles of the last TWR radix-8 passes, constant for this thread (the
  // earlier passes' come from tws, entry (r-1)*NS + k of pass p)
  Tw<C> tw[K::TWR][7];
#pragma unroll
  for (int pr = 0; pr < K::TWR; ++pr) {
    const int ns = K::R0 << (3 * (K::NP8 - K::TWR + pr));
    const int k = j & (ns - 1);
    const int stride = N / (8 * ns);
#pragma unroll
    for (int r = 1; r < 8; ++r) tw[pr][r - 1] = wn[r * k * stride];
  }
  double kx2[8] = {};
  if (sizeof(R) == 8 && xpass && q.prop_x == nullptr) {  // FP64's joint argument per point
#pragma unroll
    for (int s = 0; s < 8; ++s) kx2[s] = gkx2[j + s * K::TL];
  }
  const double inv_norm = 1.0 / q.norm;  // n*n is a power of two: exact
  const bool scale_only = refract3_is_scale(q, inv_norm);
  if (tid == 0) mbar_init(bar, 1);
  __syncthreads();
  // the field is read only after the previous kernel in the stream is done
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");

  auto issue = [&](int g) {
    const int line0 = g * K::L;
    mbar_arrive_expect_tx(bar, (unsigned)K::STAGE);
    if (xpass) {
      const unsigned dst = smem_u32(S);
      for (int b = 0; b < N / K::BC; ++b) {
        const int c0 = 2 * line0, c1 = b * K::BC;
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst + (unsigned)(b * K::BC * K::L * sizeof(C))),
            "l"(&tmap), "r"(c0), "r"(c1), "r"(smem_u32(bar))
            : "memory");
      }
    } else {
      bulk_load(S, field + (long long)line0 * N, (unsigned)K::STAGE, bar);
    }
  };

  int g = blockIdx.x;
  if (tid == 0 && g < K::GROUPS) issue(g);
  int cur = 1;
  for (int it = 0; g < K::GROUPS; ++it, g += gridDim.x) {
    // the previous group's tile stores have read their buffer (x pass; with
    // per-warp stores each warp's lane 0 issued its own)
    if (K::WARP_ST ? (tid & 31) == 0 : tid == 0)
      asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
    if (tid == 0) {
      const bool ok = mbar_wait_bounded(bar, it & 1, 2000000000ull);
      if (!ok) {
        atomicAdd(&g_lines_wait_timeouts, 1u);
        mbar_wait_bounded(bar, it & 1, 2000000000ull);  // the copy may still be in flight
      }
      s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) {
      if ((tid & 31) == 0) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
      return;
    }
    (void)mbar_try_wait(bar, it & 1);  // completed phase: orders the staged line for this thread
    const int line0 = g * K::L;
    C v[K::LPT][8];
#pragma unroll
    for (int t = 0; t < K::LPT; ++t) {
      const int l = slot * K::LPT + t;
#pragma unroll
      for (int s = 0; s < 8; ++s) {
        const int e = j + s * K::TL;
        v[t][s] = xpass ? S[e * K::L + l] : S[l * N + e];
      }
    }
    // The staging buffer is free once every thread has read it, which the
    // first exchange barrier of the group's first transform guarantees:
    // thread 0 then issues the next group's copy (its latency hides behind
    // the rest of this group's work).
    const int gn = g + gridDim.x;
    auto issue_next = [&] {
      if (tid == 0 && gn < K::GROUPS) issue(gn);
    };
    auto nothing = [] {};

    if (q.mode == 1) {
      line_fft<-1, R, N, LG>(v, X0, X1, cur, tw, tws, slot, j, issue_next);
      // propagator K = exp(-i a (kx^2 + ky^2)) (src/fftSolver3D.cpp:24-30, 87-120)
#pragma unroll
      for (int t = 0; t < K::LPT; ++t) {
        const int line = line0 + slot * K::LPT + t;  // y index
        const double ky = kfreq(line, N, q.two_pi, q.stepn_y);
        const double ky2 = __dmul_rn(ky, ky);
#pragma unroll
        for (int s = 0; s < 8; ++s) v[t][s] = prop3(q, v[t][s], kx2[s], ky2, j + s * K::TL, line);
      }
      line_fft<+1, R, N, LG>(v, X0, X1, cur, tw, tws, slot, j, nothing);
    } else if (q.mode == 0) {
      line_fft<-1, R, N, LG>(v, X0, X1, cur, tw, tws, slot, j, issue_next);
    } else {
      line_fft<+1, R, N, LG>(v, X0, X1, cur, tw, tws, slot, j, issue_next);
      if (scale_only) {
#pragma unroll
        for (int t = 0; t < K::LPT; ++t)
#pragma unroll
          for (int s = 0; s < 8; ++s) v[t][s] = scale_point(v[t][s], inv_norm);
      } else {
        // material or absorber in this step: the thread's own points go
        // through the exchange buffer the last pass did not read (every
        // thread is past its reads) and one non-unrolled refract3 loop; the
        // barrier after it keeps the next transform's first writes to that
        // buffer behind every thread's use of it
        C *scr = (cur ? X0 : X1) + slot * K::LPT * K::XS;
#pragma unroll
        for (int t = 0; t < K::LPT; ++t)
#pragma unroll
          for (int s = 0; s < 8; ++s) scr[t * K::XS + j + s * K::TL] = v[t][s];
#pragma unroll 1
        for (int i = 0; i < 8 * K::LPT; ++i) {
          const int t = i / 8, e = j + (i % 8) * K::TL;  // e: y index
          C *p = scr + t * K::XS + e;
          *p = refract3<R>(q, *p, line0 + slot * K::LPT + t, e, inv_norm);
        }
#pragma unroll
        for (int t = 0; t < K::LPT; ++t)
#pragma unroll
          for (int s = 0; s < 8; ++s) v[t][s] = scr[t * K::XS + j + s * K::TL];
        __syncthreads();
      }
      if (save) {
#pragma unroll
        for (int t = 0; t < K::LPT; ++t)
#pragma unroll
          for (int s = 0; s < 8; ++s)
            save[(long long)(line0 + slot * K::LPT + t) * N + j + s * K::TL] = v[t][s];
      }
      if (q.mode != 3) line_fft<-1, R, N, LG>(v, X0, X1, cur, tw, tws, slot, j, nothing);
    }
    if (xpass && K::WARP_ST) {
      // one line a group: the last pass left thread j with outputs j + s*TL
      // and read them from F at sw(j + s*TL), which stays inside the aligned
      // 8-element block of j + s*TL, so a warp's outputs go back to exactly
      // the slots that warp read -- no CTA barrier, only the warp's own --
      // and leave by the warp's tile stores of its 8 runs of 32 rows
      C *F = cur ? X1 : X0;
      const int lane = tid & 31, w0 = tid & ~31;
      __syncwarp();
#pragma unroll
      for (int s = 0; s < 8; ++s) F[j + s * K::TL] = v[0][s];
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncwarp();
      if (lane == 0) {
#pragma unroll
        for (int s = 0; s < 8; ++s) {
          const int e0 = w0 + s * K::TL;
          asm volatile(
              "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(
                  &tmap_st),
              "r"(2 * line0), "r"(e0), "r"(smem_u32(F + e0))
              : "memory");
        }
        asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
      }
    } else if (xpass) {
      // columns leave by TMA tile stores (the staging layout: element e of
      // line l at e*L + l), instead of 16-byte stores strided by the row
      // length, from the exchange buffer the last pass read, once every
      // thread is past those reads: the next group writes that buffer only
      // in its second pass, after its first-pass barrier, and thread 0 waits
      // for the copies' reads at the top of the next group, beside its wait
      // for the staged line -- off the critical path
      __syncthreads();
      C *F = cur ? X1 : X0;
#pragma unroll
      for (int t = 0; t < K::LPT; ++t)
#pragma unroll
        for (int s = 0; s < 8; ++s) F[(j + s * K::TL) * K::L + slot * K::LPT + t] = v[t][s];
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        const unsigned src = smem_u32(F);
        for (int b = 0; b < N / K::BC; ++b)
          asm volatile(
              "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(
                  &tmap),
              "r"(2 * line0), "r"(b * K::BC), "r"(src + (unsigned)(b * K::BC * K::L * sizeof(C)))
              : "memory");
        asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
      }
    } else {
      // rows: natural-order outputs straight to global memory (coalesced)
#pragma unroll
      for (int t = 0; t < K::LPT; ++t) {
        const int line = line0 + slot * K::LPT + t;
#pragma unroll
        for (int s = 0; s < 8; ++s) field[(long long)line * N + j + s * K::TL] = v[t][s];
      }
    }
  }
  // the last group's tile stores complete before the CTA leaves
  if ((tid & 31) == 0) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
}

// ---- host side -------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &qr) ==
            cudaSuccess &&
        qr == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// Tensor map of the field as rows of 2n reals (re, im) x n columns; tiles
// of 2L reals x rows positions (the x lines row0 .. row0+L-1 at that many
// positions: BC for the loads and the CTA's stores, BCS for a warp's).
template <typename R, int N, int LG>
cudaError_t make_tmap(void *field, CUtensorMap *out, int rows) {
  using K = Cfg<R, N, LG>;
  EncodeTiledFn enc = encode_fn();
  if (enc == nullptr) return cudaErrorNotSupported;
  const cuuint64_t dims[2] = {(cuuint64_t)2 * N, (cuuint64_t)N};
  const cuuint64_t strides[1] = {(cuuint64_t)2 * N * sizeof(R)};
  const cuuint32_t box[2] = {(cuuint32_t)(2 * K::L), (cuuint32_t)rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(out, sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                         2, field, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <typename R, int N, int LG>
cudaError_t launch(const Fft3dPass &q, const double *kx2, const void *wnv, cudaStream_t s) {
  const Tw<typename Cx<R>::T> *wn = reinterpret_cast<const Tw<typename Cx<R>::T> *>(wnv);
  using K = Cfg<R, N, LG>;
  static_assert(K::SMEM <= 227 * 1024, "line pass exceeds shared memory");
  CUtensorMap tmap, tmap_st;
  std::memset(&tmap, 0, sizeof(tmap));
  std::memset(&tmap_st, 0, sizeof(tmap_st));
  if (q.mode == 1) {
    cudaError_t e = make_tmap<R, N, LG>(q.field, &tmap, K::BC);
    if (e == cudaSuccess && K::WARP_ST) e = make_tmap<R, N, LG>(q.field, &tmap_st, K::BCS);
    if (e != cudaSuccess) return e;
  }
  if (K::TWS_N > 0 && q.tw_lines == nullptr) return cudaErrorInvalidValue;
  auto k = fft3d_lines_kernel<R, N, LG>;
  {
    const cudaError_t e = raise_dynamic_smem((const void *)k, (int)K::SMEM);
    if (e != cudaSuccess) return e;
  }
  if constexpr (K::TW_TABLE) {
    // MINB CTAs an SM: the rest of the SM's 256 KB serves as L1 (the
    // propagator's x factors and the twiddle table are read through it)
    const cudaError_t e = prefer_smem_carveout((const void *)k, (int)K::SMEM, K::MINB);
    if (e != cudaSuccess) return e;
  }
  static int per_sm = 0, sms = 0;
  if (per_sm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, K::T, K::SMEM);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
  }
  const int grid = K::GROUPS < sms * per_sm ? K::GROUPS : sms * per_sm;
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
  return cudaLaunchKernelEx(&cfg, k, q, tmap, tmap_st, kx2, wn);
}

}  // namespace lines

// Tensor map of an n x n complex field as rows of 2n reals (real_bytes 8:
// complex128, 4: complex64), tiles of box_reals x box_rows; shared with the
// radix-16 line kernel's L2 prefetches (fft3d_r16.cu).
cudaError_t encode_field_tmap(void *field, int n, int real_bytes, int box_reals, int box_rows,
                              CUtensorMap *out) {
  lines::EncodeTiledFn enc = lines::encode_fn();
  if (enc == nullptr) return cudaErrorNotSupported;
  std::memset(out, 0, sizeof(*out));
  const cuuint64_t dims[2] = {(cuuint64_t)2 * n, (cuuint64_t)n};
  const cuuint64_t strides[1] = {(cuuint64_t)2 * n * real_bytes};
  const cuuint32_t box[2] = {(cuuint32_t)box_reals, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r =
      enc(out, real_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
          field, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

namespace lines {
template <int N, int LG> int tw_exponents(int *out, int cap) {
  using K = Cfg<double, N, LG>;  // the complex64 kernel reads the same table or none
  static_assert(Cfg<float, N, LG>::TWS_N == 0 || Cfg<float, N, LG>::TWS_N == K::TWS_N,
                "one table for both precisions");
  if (K::TWS_N > cap) return -1;
  int i = 0;
  for (int p = 0; p < K::NP8 - K::TWR; ++p) {
    const int ns = K::R0 << (3 * p);
    for (int e = 0; e < 7 * ns; ++e) {
      const int r = e / ns + 1, kk = e % ns;
      out[i++] = r * kk * (N / (8 * ns));
    }
  }
  return i;
}
}  // namespace lines

int fft3d_lines_tw_exponents(int n, int *out, int cap) {
  switch (n) {  // the line slots launch_fft3d_lines uses for n
    case 1024: return lines::tw_exponents<1024, 2>(out, cap);
    case 2048: return lines::tw_exponents<2048, 1>(out, cap);
    case 4096: return lines::tw_exponents<4096, 1>(out, cap);
    default: return 0;
  }
}

bool fft3d_lines_supported(Precision p, int n) {
  (void)p;
  return n >= 64 && n <= 4096 && !(n & (n - 1));
}

cudaError_t launch_fft3d_lines(Precision p, const Fft3dPass &q, const double *kx2,
                               const void *wn, cudaStream_t s) {
  const void *w = wn;
#define PXP_L3(NN, LGD, LGF)                                                          \
  case NN:                                                                            \
    return p == kFP64 ? lines::launch<double, NN, LGD>(q, kx2, w, s)                  \
                      : lines::launch<float, NN, LGF>(q, kx2, w, s);
  switch (q.n) {
    // line slots per CTA: 256 threads (255 registers each) from n = 1024,
    // 512 at n = 4096 (one line); fewer at small n so that the groups
    // spread over the SMs
    PXP_L3(64, 8, 8) PXP_L3(128, 4, 4) PXP_L3(256, 2, 2) PXP_L3(512, 2, 2)
    PXP_L3(1024, 2, 2) PXP_L3(2048, 1, 1) PXP_L3(4096, 1, 1)
    default:
      return cudaErrorInvalidValue;
  }
#undef PXP_L3
}

unsigned fft3d_lines_wait_timeouts(cudaStream_t s) {
  unsigned v = 0;
  if (cudaMemcpyFromSymbolAsync(&v, g_lines_wait_timeouts, sizeof(v), 0, cudaMemcpyDeviceToHost,
                                s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return 0;
  return v;
}

}  // namespace pxp
