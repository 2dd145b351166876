// pxp_kernels.h -- host-side launch interface of the CUDA kernels.
// Plain structs of device pointers; shared by the C-ABI layer (capi.cu) and
// the kernel translation units.  No torch types anywhere.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace pxp {

enum Precision { kFP64 = 0, kFP32 = 1 };

// Record the message pxp_last_error(NULL, ...) returns (capi.cu).
void set_last_error(const char *msg);

// Raise the dynamic shared-memory limit of `kernel` to at least `bytes` on the
// current device (smem_attr.cu).  The attribute is per device context, so a
// process driving several GPUs needs it set on each; this records what was
// set per (kernel, device) and calls cudaFuncSetAttribute only when needed.
cudaError_t raise_dynamic_smem(const void *kernel, int bytes);
// Ask, once per kernel and device, for the smallest shared-memory carve-out
// that holds `ctas` CTAs of `bytes` dynamic shared memory each, leaving the
// rest of the SM's unified L1/shared storage to L1.
cudaError_t prefer_smem_carveout(const void *kernel, int bytes, int ctas);

// ---------------------------------------------------------------- FFT 1-D --
// One split-step problem with one transverse dimension (FFTSolver2D).
// All complex arrays are interleaved and in the solver's precision.
// Per-step flux integrals of the 2-D step kernels (flux.cuh): for steps
// step0 .. step0 + count - 1 the kernel stores out[step - step0] = the
// trapezoid sum of |u|^2 over win[step - step0] = (a, b), a <= b.
struct FluxSpec {
  const int2 *win;
  double *out;
  int step0, count;
};

struct Fft1dJob {
  void *field;             // N complex: field after the previous step
  // Constant-factor tables hold complex128 entries in FP64 and split
  // complex64 pairs (fft_smem.cuh) in FP32.
  const void *kern;        // N entries: propagator exp(-i (dz/2k) kx^2)
  const void *trans;       // N entries per table: transmission (FP64: t,
                           // applied as (u*t)/N; FP32: t/N, applied as u*t)
  long long trans_stride;  // complex elements between per-step tables; 0 =
                           // z-invariant medium (one table)
  const void *twiddle;     // N entries: radix-8 Stockham twiddles (pass order)
  void *saves;             // save slots, N complex each (may be null)
  int n;                   // transverse points (power of two)
  int step0;               // 1-based index of the first step of this launch
  int nsteps;              // steps to take
  int save_every;          // save when step % save_every == 0 (0 = never)
  int max_slots;           // capacity of saves
  int trans_step0;         // step that per-step table 0 belongs to
  FluxSpec flux;           // per-step flux integrals (out == null: none)
  // n not a power of two (Bluestein): twiddle holds the Stockham twiddles of
  // the power-of-two length m >= 2n - 1; chirp: n complex128
  // exp(-i pi j^2 / n); bconv: m complex128, the transform of the
  // conjugate chirp filter divided by m
  const void *chirp;
  const void *bconv;
  int m;
  // powers of two 512 .. 4096 (fft1d_r16.cu): N entries exp(-2 pi i m / N)
  const void *wn;
};

// Launch nj jobs that all share one transform length n (one CTA per job).
// step0/nsteps >= 0 override every job's own values (single-problem use).
// flux: some job has flux windows (the kernel variant that sums them).
// Register-resident radix-16 FFTSolver2D kernel (fft1d_r16.cu): whether it
// takes size n (powers of two 512 .. 4096), and its launch.
bool fft1d_r16_enabled(int n);
cudaError_t launch_fft1d_r16(Precision p, const Fft1dJob *d_jobs, int nj, int n, int step0,
                             int nsteps, cudaStream_t s, bool flux, unsigned *queue = nullptr);
// Launch variants of the 2-D step kernels, chosen per (device, precision,
// size) by the tuner in capi.cu: FFTSolver2D 0 = shared-memory Stockham
// kernel, 1 = register-resident radix-16 kernel; CrankNicholson's
// step-invariant path at 4096 rows 0 = one CTA, 1 = a cluster of two CTAs.
// *_variants returns how many a size has (1: nothing to choose); variant
// -1 is the default (the radix-16 kernel where it runs; one CTA).
int fft1d_variants(Precision p, int n);
int cn_const_variants(Precision p, int n);
// queue: a device counter (zero at launch) that makes the power-of-two
// kernels persistent -- at most one wave of CTAs, each taking its next job
// from the counter (persistent.cuh); null: one CTA per job.
cudaError_t launch_fft1d(Precision p, const Fft1dJob *d_jobs, int nj, int n,
                         int step0, int nsteps, cudaStream_t s, bool flux = false,
                         int variant = -1, unsigned *queue = nullptr);
bool fft1d_supported(Precision p, int n);
// complex128 lines of 16384 points (fft1d_pair.cu): a cluster of two CTAs per
// job, each holding the points of one parity; the job's twiddle is the
// 8192-point Stockham table and its chirp the table exp(-2 pi i k / 16384).
cudaError_t launch_fft1d_pair(Precision p, const Fft1dJob *d_jobs, int nj, int n, int step0,
                              int nsteps, cudaStream_t s, bool flux);
inline bool fft1d_pair_size(Precision p, int n) { return p == kFP64 && n == 16384; }
// Length of the power-of-two transforms of the Bluestein path for n (the
// smallest power of two >= 2n - 1); n itself for powers of two.
int fft1d_bluestein_m(int n);

// ------------------------------------------------------------ CN 1-D ------
// Crank-Nicolson problem (CrankNicholson with default F=G=H=1, J=0).
struct CnJob {
  void *field;                 // N complex (solver precision)
  const double *delta, *beta;  // material at z (per x), FP64
  const double *delta_prev, *beta_prev;  // material at z - dz
  long long mat_stride;        // doubles between per-step planes (0 = z-invariant)
  void *saves;
  double rho, r;               // dz/(k dx^2), k dz
  int n;                       // rows solved: Nx, or Nx padded to M*T (cn_padded_n)
  int n_real;                  // Nx; rows n_real..n-1 are decoupled padding
  int step0, nsteps, save_every, max_slots, mat_step0;
  int transparent;             // BC_t::TRANSPARENT
  int status;                  // unused (reserved)
  const void *lu_g, *lu_h;     // factor tables of the step matrix (const path)
  FluxSpec flux;               // per-step flux integrals (out == null: none)
};
cudaError_t launch_cn(Precision p, const CnJob *d_jobs, int nj, int n, int step0,
                      int nsteps, cudaStream_t s, bool flux = false);
bool cn_supported(Precision p, int n);
// Rows the CN kernels solve for Nx = n: n itself when n/8 is a power of
// two, else n padded up to 8 times the next power of two.
int cn_padded_n(int n);
// Diagonal of the padding rows (zero right-hand side and field), in the
// kernels' rows and in the host's factor tables of the step-invariant path.
constexpr double kCnPad = 1e30;
// z-invariant medium and Dirichlet ends: the step matrix never changes; the
// job's lu_g / lu_h hold its Thomas factor tables (n complex128 each).
cudaError_t launch_cn_const(Precision p, const CnJob *d_jobs, int nj, int n, int step0,
                            int nsteps, cudaStream_t s, bool flux = false, int variant = -1);
bool cn_const_supported(Precision p, int n);

// ------------------------------------------------------------- ADI ------
struct Sphere {
  double cx, cy, cz, r, delta, beta;
};
constexpr int kInlineSpheres = 16;

// Constructive solid geometry on the device (the reference's CSGMaterial
// flattened, see pxp_set_material_csg): shapes hold rows 0-2 of their 4x4
// transformation.  `active` marks the modules that can contain a point of
// the planes the launch samples (the others are skipped: they claim no such
// point); modules == nullptr or active == 0 means no CSG material.
struct CsgShape {
  double m[12];
  double size[3];
  int kind, op;
};
struct CsgPart {
  double delta, beta;
  int op, first, count;
};
struct CsgModule {
  int first, count;
};
struct Csg {
  const CsgModule *modules;
  const CsgPart *parts;
  const CsgShape *shapes;
  int nmodules;
  unsigned long long active;
};

// One half step of ADI (ADI::xImplicit / yImplicit,
// src/alternatingDirectionSolver.cpp:8-134) on an n x n field.  Systems run
// along the implicit direction ("position"); the explicit stencil couples
// neighbouring systems.  Element (system s, position p) is at
// p * stride_pos + s * stride_sys.
struct AdiHalf {
  const void *in;
  void *out;
  void *save;              // optional extra copy of the output (save slot)
  long long stride_pos, stride_sys;
  int n;                   // Nx = Ny: positions per system and number of systems
  int n_pad;               // 0, or the padded system length the general kernel
                           // solves (adi_padded_n; rows n..n_pad-1 decoupled)
  int y_implicit;          // 1: y-implicit diagonal formula (reference :103)
  int use_tbc;             // ADI::useTBC
  int nspheres;            // active spheres; > kInlineSpheres: use spheres_all
  double inv_dzh;          // 1.0 / (dz/2)
  double kd2_impl;         // k*d*d along the implicit direction
  double kd2_expl;         // k*d*d along the explicit direction
  double k;
  double xmin, dx, ymin, dy;
  double z;                // material plane of this half step
  // one-wave vacuum kernel: chunks tab_c0 < c < tab_c1 of the staged tables
  // hold bit for bit the entries of chunk tab_c0 and read those (0, 0: none)
  int tab_c0, tab_c1;
  Csg csg;                 // CSG material (instead of spheres) when csg.active
  // sampled material of this half step's plane (instead of spheres or CSG)
  // when plane_delta is set: n*n doubles each, the field's layout (x index *
  // n + y index)
  const double *plane_delta, *plane_beta;
  const Sphere *spheres_all;
  Sphere spheres[kInlineSpheres];
};
cudaError_t launch_adi_half(Precision p, const AdiHalf &h, cudaStream_t s);
bool adi_supported(Precision p, int n);
// System length the general ADI kernel solves for Nx = n (n itself for the
// powers of two adi_supported takes, else 8 times the next power of two),
// and whether that kernel runs n.
int adi_padded_n(int n);
bool adi_padded_supported(Precision p, int n);
// Half step whose plane holds no material and no transparent boundary: the
// matrix is the same for every system and every step; g/h are its Thomas
// factor tables (n complex128 each, see scan_solve.cuh; read by the FP32
// kernel, which takes powers of two only).
// `staged`: the factor tables of the FP64 one-wave kernel, for its padded
// system length adi_wave_n(n), with their in-chunk products, in the layout
// it copies into shared memory (adi_const_staged_tables).  FP64 runs any
// n with adi_wave_n(n) > 0 here.
cudaError_t launch_adi_half_const(Precision p, const AdiHalf &h, const void *g, const void *hh,
                                  const void *staged, cudaStream_t s);
// System length of the FP64 one-wave vacuum kernel for a grid of n nodes
// (64, 128, 256, 512, 768 or 1024, the smallest that holds n), 0 when n is
// outside 4 .. 1024.  Rows n .. length-1 are decoupled padding.
int adi_wave_n(int n);
// Host: fills out[0 .. 4n) complex128 with [g | h | pf | pb] in the
// chunk-transposed slots of the one-wave vacuum kernel for system length n
// (pf, pb: products of h over each chunk's rows up to / from a row) and
// returns true; false when no one-wave kernel solves length n (out
// untouched).  g, h, out: interleaved (re, im); for a padded grid, g and h
// already hold the padding rows (g = 1, h = 0).  run[0..1]: the longest
// run [c0, c1) of consecutive chunks whose entries (g, h, pf and pb at every
// row of the chunk) are bit for bit equal, for AdiHalf::tab_c0 / tab_c1.
bool adi_const_staged_tables(int n, const double *g, const double *h, double *out, int run[2]);
// Saved-slice downsampling of the 3-D solvers (Solver3D::copyCurrentSolution,
// src/solver3D.cpp:94-112): n x n field -> m x m block averages.
cudaError_t launch_block_average(Precision p, const void *full, void *out, int n, int m,
                                 cudaStream_t s);

// Post-processing quantities of n complex values into n doubles:
// 0 = |u|, 1 = arg u, 2 = Re u, 3 = |u|^2 (post.cu).
cudaError_t launch_post(Precision p, const void *field, double *out, long long n, int quantity,
                        cudaStream_t s);
// Running max of |u| over n values into *result (the bits of a double,
// start from 0).
cudaError_t launch_max_abs(Precision p, const void *field, long long n, unsigned long long *result,
                           cudaStream_t s);

// Lines of a far-field transform (farfield.cu): line l, entry j at
// in[l * line_stride + j] (complex64 when in_c64, else complex128), minus
// ref (complex128, same layout) when ref is set, conjugated when conj_in;
// padded to L entries with pad_value (or, when pad_const, with the line's
// entry 0).  Kept: outputs i0..i1 of the fftshifted transform, written to
// out[l + (i - i0) * out_stride] as complex128 (mode 0), |X|^2 / divisor
// (mode 1) or |X| / divisor (mode 2).  wL: L entries exp(-2 pi i m / L);
// twQ: Stockham twiddles of the sub-transform length; wsplit: the same
// factors as two short tables (see below).
struct FarFieldLines {
  const void *in;
  const double2 *ref;
  long long line_stride;
  int in_c64, conj_in, pad_const, mode;
  int n;
  long long nlines;
  double2 pad_value;
  long long L, i0, i1;
  void *out;
  long long out_stride;
  double divisor;
  const double2 *wL;
  const double2 *twQ;
  // pruned transform: exp(-2 pi i m / L) = hi[m >> split_bits] * lo[m & (2^split_bits - 1)],
  // wsplit = lo (2^split_bits entries) followed by hi (L >> split_bits entries)
  const double2 *wsplit;
  int split_bits;
};

// Sub-transform length of the pruned transform for lines of n entries
// padded to L, or 0 when L is not a power of two or n needs more than 8192
// (the direct DFT then runs).
int farfield_pruned_q(long long n, long long L);
// split_bits of the pruned transform's twiddle tables for length L.
int farfield_split_bits(long long L);
// q: farfield_pruned_q's choice, or 0 for the direct DFT.
cudaError_t launch_farfield_lines(const FarFieldLines &p, int q, cudaStream_t s);
// resizeMatrix of a column-major rows-row matrix to er x ec.
cudaError_t launch_resize(const double *in, long long rows, double *out, int er, int ec, double dY,
                          double dX, cudaStream_t s);
// Trapezoid sum of |u|^2 over [a, b] of a field of n points (one CTA).
cudaError_t launch_flux_sum(Precision p, const void *field, int a, int b, double *out,
                            cudaStream_t s);
// complex64 -> complex128, n entries.
cudaError_t launch_widen(const void *in, void *out, long long n, cudaStream_t s);

// Kernel waits on the current device that ran out (bounded mbarrier waits),
// read on stream s (synchronises s).
unsigned wait_timeouts(cudaStream_t s);
// One-thread kernel whose bounded wait (limit_ns of global time) runs out on
// purpose and is counted like the propagation kernels' (adi.cu).
cudaError_t launch_wait_selftest(unsigned long long limit_ns, cudaStream_t s);

// --------------------------------------------------------------- FFT 3-D --
// FFTSolver3D (src/fftSolver3D.cpp:52-156, 327-374) on an n x n field in the
// reference's column-major layout (element (y, x) at x*n + y).  A step is two
// line passes over HBM:
//   x pass: each line of fixed y index (stride n): forward FFT along x,
//           propagator multiply, backward FFT along x;
//   y pass: each contiguous line of fixed x: backward FFT along y,
//           transmission / normalisation / absorber (refraction of this
//           step), then the next step's forward FFT along y.
// The field between pxp_step calls is in real space; the first step of a call
// starts with a forward-only y pass and the last ends without the forward.
struct Fft3dPass {
  void *field;             // n*n complex (solver precision), in place
  void *save;              // optional: real-space copy after refraction
  const void *twiddle;     // n complex128
  int n;
  int mode;                // 0: forward y only; 1: x pass; 2: y pass (inverse,
                           // refraction, forward); 3: y pass without forward
  // propagator (x pass): K = exp(-A (kx^2 + ky^2)), A = (0, 0.5*dz/k)
  double a;                // 0.5*dz/k
  double two_pi;           // 2.0*PI
  double stepn_x, stepn_y; // step*n per axis (FFTSolver3D::spatialFreqX/Y)
  // refraction (y pass)
  double k, dz, xmin, dx, ymin, dy, z1, z0, norm;
  int nspheres;
  Csg csg;                 // CSG material (instead of spheres) when csg.active
  // sampled material of this step (instead of spheres or CSG) when
  // plane_delta is set: the (delta, beta) FFTSolver3D::refraction applies at
  // each point, n*n doubles each in the field's layout
  const double *plane_delta, *plane_beta;
  const Sphere *spheres_all;
  Sphere spheres[kInlineSpheres];
  // n not a power of two (fft3d_blu.cu): twiddle holds the Stockham
  // twiddles of the Bluestein length m >= 2n - 1; chirp: n complex128
  // exp(-i pi j^2 / n); bconv: m complex128, the filter's transform over m
  const void *chirp, *bconv;
  int m;
  // absorber (FFTSolver3D::absorbingBC): thickness in pixels and inverse
  // damping length per axis (0 thickness = off)
  int thick_x, thick_y;
  double inv_damp_x, inv_damp_y;
  // the propagator as the product of its x and y factors, prop_x[i] =
  // exp(-i a kx_i^2) and prop_y[i] = exp(-i a ky_i^2) (n entries each,
  // complex128 in FP64, split complex64 in FP32; phases reduced on the host
  // in extended precision; k_i folds, so entry i equals entry n - i and the
  // kernels read entries 0 .. n/2 only); null in FP64 when the reference's
  // joint argument is asked for (PXP_FFT3D_JOINT_PROP=1)
  const void *prop_x, *prop_y;
  // twiddles of the register-line kernel's radix-8 passes before its last
  // (fft3d_lines.cu, n = 1024 .. 4096): entry i = exp(-2 pi i m_i / n), m_i from
  // fft3d_lines_tw_exponents, in the solver's table form
  const void *tw_lines;
};
// Exponents m_i of the twiddle table Fft3dPass::tw_lines for length n (out:
// room for cap entries); returns the entry count (0: the kernel for n reads
// no table).
int fft3d_lines_tw_exponents(int n, int *out, int cap);
// variant: 0 = radix 8, double-buffered, tables in shared memory; 1 = radix
// 8, single buffer, tables through L1; 2 = radix 16, single buffer; 3 =
// register-resident transforms with TMA-staged lines (fft3d_lines.cu; n up
// to 4096); 4 = 16 points per thread, radix-16 passes, two line slots per
// CTA (fft3d_r16.cu; n = 512 .. 4096); 5 = the same with complex64 lines
// one a slot and four slots a CTA (FP32 only: half the registers, twice the
// warps).  Sizes a variant does not take run variant 0.
// kx2: n doubles, fl(kx*kx) per column index; q.twiddle / tw16: Stockham
// twiddles for radix 8 / radix 16 pass orders; wn: n complex128
// exp(-2 pi i m / n), m < n.
cudaError_t launch_fft3d_pass(Precision p, const Fft3dPass &q, int variant, const double *kx2,
                              const void *tw16, const void *wn, cudaStream_t s);
constexpr int kFft3dVariants = 6;
bool fft3d_supported(Precision p, int n);
bool fft3d_lines_supported(Precision p, int n);
// single: complex64 lines one a slot, four slots a CTA (variant 5)
bool fft3d_r16_supported(Precision p, int n, bool single = false);
cudaError_t launch_fft3d_r16(Precision p, const Fft3dPass &q, const double *kx2, const void *wn,
                             cudaStream_t s, bool single = false);
// Line passes of a size that is not a power of two (Bluestein transforms,
// fft3d_blu.cu); q.chirp, q.bconv, q.m and q.twiddle as described above.
cudaError_t launch_fft3d_bluestein(Precision p, const Fft3dPass &q, const double *kx2,
                                   cudaStream_t s);
cudaError_t launch_fft3d_lines(Precision p, const Fft3dPass &q, const double *kx2, const void *wn,
                               cudaStream_t s);
// Bounded waits of the line-pass kernels that ran out on the current device.
unsigned fft3d_lines_wait_timeouts(cudaStream_t s);
unsigned fft3d_r16_wait_timeouts(cudaStream_t s);

}  // namespace pxp
