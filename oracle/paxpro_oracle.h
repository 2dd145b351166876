/*
 * paxpro_oracle.h -- CPU oracle for the paraxial propagation step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates, on the CPU and in FP64,
 * the arithmetic of the reference solvers (FFTSolver2D, FFTSolver3D with its
 * refraction integral and absorber, CrankNicholson, ADI, ThomasAlgorithm) so
 * that the CUDA product can be checked against it.  Only tests/, the smoke
 * check and bench.py's CPU-baseline leg may load it; the product never does.
 *
 * Parity status: the tridiagonal solve is pinned bit-for-bit against the
 * reference's own ThomasAlgorithm template compiled from its source
 * (oracle/ref_pin.cpp).  The rest of the path depends on FFTW3 / Armadillo /
 * HDF5, which are absent here, so those parts are "parity unpinned": they are
 * checked against known-answer tests (analytic Gaussian beam, plane wave in a
 * uniform medium, unitarity) and against numpy/pocketfft for the FFT.
 *
 * All complex arrays are interleaved (re, im) doubles.  2-transverse-dim
 * fields use the reference's Armadillo column-major layout: element
 * (row = y index, col = x index) lives at col*Ny + row.
 */
#ifndef PAXPRO_ORACLE_H
#define PAXPRO_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Grid, as ParaxialSimulation's three Disctretization records plus k. */
typedef struct {
  double xmin, xmax, dx;
  double ymin, ymax, dy;
  double zmin, zmax, dz;
  double wavenumber;
} orc_grid;

/* One sphere of a first-hit sphere list (materials of the 3-D configs). */
typedef struct {
  double cx, cy, cz, radius, delta, beta;
} orc_sphere;

enum {
  ORC_MAT_VACUUM = 0,
  ORC_MAT_WAVEGUIDE = 1, /* planar core + cladding + index-based beta ramp */
  ORC_MAT_SPHERES = 2,   /* first sphere with r^2 < R^2 wins */
  ORC_MAT_XTABLE = 3,    /* z-invariant delta/beta per x index (2-D only) */
  ORC_MAT_CSG = 4        /* CSGMaterial over geom::Module / Part / Shape */
};

/* CSGMaterial (src/materialFunction.cpp:3-13) flattened: modules in order,
 * each a range of parts, each part a range of shapes.  kind: 0 sphere, 1
 * box, 2 cylinder; operation: 0 union (add), 1 difference; transform: the
 * shape's 4x4 geom::Shape::transformation, row-major; size: sphere radius /
 * box Lx, Ly, Lz / cylinder height, r1, r2. */
typedef struct {
  int kind, operation;
  double transform[16];
  double size[3];
} orc_csg_shape;
typedef struct {
  int operation, first_shape, num_shapes;
  double delta, beta;
} orc_csg_part;
typedef struct {
  int first_part, num_parts;
} orc_csg_module;

typedef struct {
  int kind;
  /* waveguide */
  double core_half_width, delta_clad, beta_clad, ramp_beta;
  int ramp_points;
  int n_transverse;
  /* spheres */
  const orc_sphere *spheres;
  int n_spheres;
  /* x table */
  const double *delta_table, *beta_table;
  /* constructive solid geometry */
  const orc_csg_module *csg_modules;
  int n_csg_modules;
  const orc_csg_part *csg_parts;
  const orc_csg_shape *csg_shapes;
} orc_material;

/* Node count exactly as the reference computes it (truncating cast). */
unsigned orc_node_count(double mn, double mx, double step);

/* In-place complex DFT of length n (radix-2 FFT for powers of two, a direct
 * DFT otherwise); sign -1 = forward
 * exp(-2 pi i jk/n), +1 = backward exp(+2 pi i jk/n); unnormalised. */
int orc_fft1d(double *data, int n, int sign);

/* Material lookup at (x, y, z). */
void orc_material_eval(const orc_material *m, const orc_grid *g, double x,
                       double y, double z, double *delta, double *beta);

/* The reference's tridiagonal solve (symmetric off-diagonals, no pivoting).
 * Solution overwrites diag; rhs is modified.  n >= 2. */
void orc_thomas(double *diag, const double *subdiag, double *rhs, int n);

/* Runs of the four solvers from the initial field u0 (already the field at
 * z = zmin, as after setInitialConditions).  Steps 1..nsteps are taken as
 * Solver::step() would.  Every save_every steps (if > 0) the current field
 * is appended to saves.  The final field goes to u_out.  Return 0 on
 * success, negative on bad input. */
int orc_fft2d_run(const orc_grid *g, const orc_material *m, const double *u0,
                  int nsteps, int save_every, double *saves, double *u_out);

int orc_cn2d_run(const orc_grid *g, const orc_material *m, int transparent_bc,
                 const double *u0, int nsteps, int save_every, double *saves,
                 double *u_out);

/* The per-step material planes the reference samples, as the C ABI's
 * pxp_set_material_planes takes them for the 3-D kinds: kind 3
 * (FFTSolver3D): one plane per step, the (delta, beta) refraction applies
 * (refraction integral included); kind 4 (ADI): two planes per step, at
 * getZ(step) and getZ(step) + dz/2.  Steps first_step .. +nsteps-1; each
 * plane Nx*Ny doubles in the field's column-major layout. */
int orc_material_planes(const orc_grid *g, const orc_material *m, int kind, int first_step,
                        int nsteps, double *delta, double *beta);

int orc_fft3d_run(const orc_grid *g, const orc_material *m,
                  double absorber_width, double absorber_damping,
                  const double *u0, int nsteps, int save_every, double *saves,
                  double *u_out);

int orc_adi3d_run(const orc_grid *g, const orc_material *m, int use_tbc,
                  const double *u0, int nsteps, int save_every, double *saves,
                  double *u_out);

/* Sources (initial fields), evaluated as the reference's source classes. */
void orc_gaussian_beam_2d(const orc_grid *g, double wavelength, double waist,
                          double center, double amplitude, double z,
                          double *out /* Nx complex */);
void orc_gaussian_beam_3d(const orc_grid *g, double wavelength, double waist,
                          double cx, double cy, double amplitude, double z,
                          double *out /* Ny x Nx column-major */);
void orc_plane_wave(int n, double value_re, double value_im, double *out);

/* Transverse downsampling of a saved 3-D field as Solver3D::
 * copyCurrentSolution does it (src/solver3D.cpp:94-112): the saved slice has
 * m = n / ratio rows and columns (src/solver3D.cpp:26, 36); with
 * delta = n / m (a double), entry (row, col) is the sum of the n x n field's
 * block rows [row*delta, row*delta + delta - 1] and columns [col*delta,
 * col*delta + delta - 1] (bounds truncated to unsigned, as the submat
 * arguments are), summed column by column, divided by delta*delta.
 * full: n x n column-major complex; out: m x m column-major complex. */
void orc_block_average(const double *full, int n, int m, double *out);

/* Run the lines of 2-D transforms on all OpenMP threads (1) or on one
 * thread as the reference's FFTW plans do (0, default).  Results are the
 * same either way: each line's transform is computed identically. */
void orc_set_fft_parallel(int on);

/* Number of OpenMP threads the oracle uses (0 = library default). */
void orc_set_threads(int n);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
