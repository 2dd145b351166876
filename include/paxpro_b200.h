/*
 * paxpro_b200.h -- C ABI of the B200 propagation solvers.
 *
 * The reference exposes its solvers through C++ classes (include/solver.hpp,
 * include/solver2D.hpp, include/solver3D.hpp, include/paraxialSimulation.hpp)
 * and a SWIG module (pypaxpro/pypaxpro.i).  This header is the plain-C
 * boundary those classes sit on in this build: opaque handles, plain
 * pointers and sizes, int status codes, no exceptions and no C++ or torch
 * types.  The C++ mirror of the reference API (the headers in include/paxpro) and the
 * Python package call only these functions.
 *
 * Conventions
 *  - Complex arrays are interleaved (re, im) doubles on the host.
 *  - 1-transverse-dim fields are Nx values (arma::cx_vec).  2-transverse-dim
 *    fields are Ny x Nx in Armadillo column-major order: element (row = y
 *    index, col = x index) at col*Ny + row (arma::cx_mat, as the reference's
 *    Solver3D stores prevSolution/currentSolution, src/solver3D.cpp:33-34).
 *  - Steps are numbered from 1 as Solver::currentStep (include/solver.hpp:73).
 *  - Every function returns PXP_OK (0) or a negative status; the handle keeps
 *    a message for pxp_last_error.
 */
#ifndef PAXPRO_B200_H
#define PAXPRO_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PXP_OK 0
#define PXP_ERR_INVALID (-1)     /* bad argument / call order */
#define PXP_ERR_NOMEM (-2)       /* device or host allocation failed */
#define PXP_ERR_CUDA (-3)        /* CUDA runtime error */
#define PXP_ERR_ABORTED (-4)     /* job cancelled */
#define PXP_ERR_BUDGET (-5)      /* step / wait budget exceeded */
#define PXP_ERR_NOT_READY (-6)   /* result not available yet */
#define PXP_ERR_UNSUPPORTED (-7) /* size/precision this build does not run */

/* ---- solver kinds (the reference's Solver2D / Solver3D subclasses) ------ */
#define PXP_FFT_SOLVER_2D 1   /* FFTSolver2D, include/fftSolver2D.hpp:13 */
#define PXP_CRANK_NICHOLSON 2 /* CrankNicholson, include/crankNicholson.hpp:16 */
#define PXP_FFT_SOLVER_3D 3   /* FFTSolver3D, include/fftSolver3D.hpp:16 */
#define PXP_ADI 4             /* ADI, include/alternatingDirectionSolver.hpp:15 */

#define PXP_FP64 0 /* plain mode: complex128 fields, reference parity */
#define PXP_FP32 1 /* served mode: complex64 fields, FP64-reduced phase tables */

/* Disctretization (include/paraxialSimulation.hpp:20-26). */
typedef struct {
  double min, max, step;
  unsigned downsampling_ratio;
} pxp_discretization;

/* Everything ParaxialSimulation hands a solver in setSolver/solve
 * (src/paraxialSimulation.cpp:67-131, 398). */
typedef struct {
  int kind;            /* PXP_FFT_SOLVER_2D ... PXP_ADI */
  int precision;       /* PXP_FP64 / PXP_FP32 */
  pxp_discretization x; /* setTransverseDiscretization */
  pxp_discretization y; /* setVerticalDiscretization (3-D kinds) */
  pxp_discretization z; /* setLongitudinalDiscretization */
  double wavenumber;   /* setWavenumber / setWaveLength: k = 2 pi / lambda */
  int transparent_bc;  /* CrankNicholson BC_t::TRANSPARENT; ADI::useTBC */
  double absorber_width, absorber_damping; /* FFTSolver3D::absorbingBC (0 = off) */
  int save_every;      /* save a field every n steps (0 = never; the
                          reference's 2-D solvers keep every step, its 3-D
                          solvers every z.downsampling_ratio steps) */
  int device;          /* CUDA device ordinal */
} pxp_problem;

/* One sphere of a first-hit sphere material (sphere r^2 < R^2 test as in
 * Examples/sphere.cpp:13-14, shapes evaluated in list order as
 * CSGMaterial::getXrayMatProp, src/materialFunction.cpp:3-13). */
typedef struct {
  double cx, cy, cz, radius, delta, beta;
} pxp_sphere;

typedef struct pxp_solver_s *pxp_solver;

/* Node count exactly as ParaxialSimulation::nodeNumber* computes it
 * (src/paraxialSimulation.cpp:107-120). */
unsigned pxp_node_count(double min, double max, double step);

/* Solver::setSimulator + ParaxialSimulation::setSolver
 * (src/paraxialSimulation.cpp:122-131, src/solver2D.cpp:21-42,
 * src/solver3D.cpp:19-44): allocate device state for the problem.
 * Transverse sizes: CrankNicholson any Nx >= 16 up to 16384 (above 4096 in
 * FP64 and 8192 in FP32 for z-invariant media with Dirichlet ends only, on
 * clusters of CTAs; transparent ends need Nx / 8 to be a power of two); ADI
 * any Nx >= 4 up to 2048 (vacuum planes of FP64 grids up to 1024 nodes of
 * any size run the one-wave fast path, padded to 64 .. 1024 rows; other
 * sizes that are not powers of two run the general kernel); FFTSolver2D any
 * Nx >= 8 up to 16384 for powers of two (FP64 16384 on a cluster of two
 * CTAs), and up to 4096 (FP64) / 8192 (FP32) for other sizes (Bluestein's
 * transform); FFTSolver3D powers of two from 64 to 8192 and other sizes up
 * to 4096 (FP64) / 8192 (FP32) (Bluestein line transforms).  Other sizes
 * return PXP_ERR_UNSUPPORTED. */
int pxp_solver_create(const pxp_problem *problem, pxp_solver *out);

/* Solver destructor (src/solver2D.cpp:10-19, src/solver3D.cpp:11-17). */
int pxp_solver_destroy(pxp_solver s);

/* Material hook, z-invariant medium sampled per transverse point
 * (ParaxialSimulation::getXrayMatProp, src/paraxialSimulation.cpp:513-537):
 * delta[i], beta[i] at x_i for the 2-D kinds (n = Nx), or at (x_col, y_row)
 * column-major for the 3-D kinds (n = Nx*Ny). */
int pxp_set_material_table(pxp_solver s, const double *delta, const double *beta, size_t n);

/* Material hook, sampled per step for z-varying media (any MaterialFunction
 * the host evaluates): for each step s = first_step .. first_step+nsteps-1
 * the planes of that step, in step order:
 *   FFTSolver2D: delta/beta at z = getZ(s) + dz/2 (src/fftSolver2D.cpp:38);
 *   CrankNicholson: at z and z - dz (src/crancNicholson.cpp:37-38), two
 *     planes per step (z first);
 *   FFTSolver3D: the delta/beta FFTSolver3D::refraction applies at each
 *     point (src/fftSolver3D.cpp:122-156): the values at z1 = getZ(s), or,
 *     where they differ from those at z0 = getZ(s-1) by more than 1e-10, the
 *     refractionIntegral of the two (:253-273); one plane per step;
 *   ADI: at getZ(s) (x half step, src/alternatingDirectionSolver.cpp:21) and
 *     getZ(s) + dz/2 (y half step, :91), two planes per step.
 * Layout [plane][point]: x for the 2-D kinds; x index * Ny + y index (the
 * field's column-major layout) for the 3-D kinds.  The planes replace a
 * table, sphere or CSG material; stepping outside first_step ..
 * first_step+nsteps-1 then fails with PXP_ERR_INVALID. */
int pxp_set_material_planes(pxp_solver s, const double *delta, const double *beta,
                            int first_step, int nsteps);

/* Material hook, first-hit sphere list evaluated on the device
 * (3-D kinds; 2-D kinds take y = 0). */
int pxp_set_material_spheres(pxp_solver s, const pxp_sphere *spheres, int n);

/* Material hook, constructive solid geometry evaluated on the device
 * (3-D kinds): the CSGMaterial of the reference (src/materialFunction.cpp:3-13)
 * flattened.  A point's material comes from the first module (in order)
 * that claims it; a module scans its parts from the last to the first and
 * the first part containing the point decides: a union part gives its
 * (delta, beta), a difference part gives vacuum (geom::Module::
 * getXrayMatProp, src/geometry.cpp:212-234); a part contains the point when,
 * scanning its shapes from the last to the first, the first shape containing
 * it was added as a union (geom::Part::isInside, src/geometry.cpp:91-108).
 * A shape tests the point after applying its 4x4 transformation
 * (geom::Shape::transform, src/shape.cpp:59-70): sphere sqrt(x^2+y^2+z^2) <
 * R; box |x| < Lx/2, |y| < Ly/2, |z| < Lz/2 (strict); cylinder
 * -h/2 < z < h/2 and sqrt(x^2+y^2) < r1 + (r2-r1)/h*(z+h/2)
 * (src/shape.cpp:146-187).  Up to 64 modules. */
#define PXP_SHAPE_SPHERE 0
#define PXP_SHAPE_BOX 1
#define PXP_SHAPE_CYLINDER 2
#define PXP_CSG_UNION 0
#define PXP_CSG_DIFFERENCE 1
typedef struct {
  int kind;             /* PXP_SHAPE_* */
  int operation;        /* joins its part as PXP_CSG_UNION (geom::Part::add) or
                           PXP_CSG_DIFFERENCE (geom::Part::difference) */
  double transform[16]; /* geom::Shape::transformation, row-major 4x4 */
  double size[3];       /* sphere: radius; box: Lx, Ly, Lz; cylinder: height, r1, r2 */
} pxp_csg_shape;
typedef struct {
  int operation;        /* joins its module: geom::Module::add / difference */
  int first_shape, num_shapes;
  double delta, beta;   /* geom::Part::delta, beta */
} pxp_csg_part;
typedef struct {
  int first_part, num_parts;
} pxp_csg_module;
int pxp_set_material_csg(pxp_solver s, const pxp_csg_module *modules, int nmodules,
                         const pxp_csg_part *parts, int nparts, const pxp_csg_shape *shapes,
                         int nshapes);

/* Solver::setInitialConditions (include/solver.hpp:54,57): the field at
 * z = zmin; host array.  Resets the step counter to 1 and clears saves. */
int pxp_set_initial_conditions(pxp_solver s, const double *field);
/* Same from a device array of the solver's storage precision. */
int pxp_set_initial_conditions_device(pxp_solver s, const void *dfield);

/* Solver::step repeated nsteps times (src/solver2D.cpp:243-250,
 * src/solver3D.cpp:148-166).  Asynchronous on the solver's stream. */
int pxp_step(pxp_solver s, int nsteps);

/* Solver::solve: all remaining steps up to nodeNumberLongitudinal()-1
 * (src/solver2D.cpp:224-241, src/solver3D.cpp:168-199). */
int pxp_solve(pxp_solver s);

/* Wait for the solver's queued work; returns the first error seen. */
int pxp_synchronize(pxp_solver s);

/* Solver::getLastSolution / getLastSolution3D (include/solver2D.hpp:78,
 * include/solver3D.hpp:38): copy the current field to the host (complex128). */
int pxp_get_last_solution(pxp_solver s, double *field);
/* Device pointer to the resident field (solver precision), valid until the
 * next call on the handle. */
int pxp_get_field_device(pxp_solver s, void **dfield, int *precision);

/* The CUDA stream (cudaStream_t) the solver launches its kernels and copies
 * on, for callers that order their own work or events against it.  No
 * reference counterpart: the reference runs on the host. */
int pxp_get_stream(pxp_solver s, void **stream);

/* Saved fields (the columns of Solver2D::solution / slices of
 * Solver3D::solution, include/solver2D.hpp:121, include/solver3D.hpp:52):
 * number of slots filled and one slot copied to the host.  A slot of the
 * 3-D solvers holds m x m complex values, m = Nx / x.downsampling_ratio,
 * the block averages Solver3D::copyCurrentSolution stores
 * (src/solver3D.cpp:94-112); with ratio 1, the field.  The 2-D solvers
 * accept ratio 1 only (their reference downsampling is the VISA low-pass
 * filter): pxp_solver_create returns PXP_ERR_UNSUPPORTED otherwise. */
int pxp_num_saved(pxp_solver s, int *count);
int pxp_get_saved(pxp_solver s, int slot, double *field);

/* Post-processing quantities computed on the device (post:: modules,
 * src/postProcessMod.cpp:7-150): out receives one double per point of a
 * saved slot (slot >= 0; its layout and size as pxp_get_saved) or of the
 * last solution (slot = -1; the layout of pxp_get_last_solution). */
#define PXP_POST_ABS 0  /* |u|: post::Intensity (:7-15), IntensityUint8's scale (:17-30) */
#define PXP_POST_ARG 1  /* arg u: post::Phase (:86-100), post::ExitPhase (:134-150) */
#define PXP_POST_REAL 2 /* Re u: post::ExitField (:102-116) */
#define PXP_POST_ABS2 3 /* pow(|u|, 2): post::ExitIntensity (:118-132) */
int pxp_get_post(pxp_solver s, int quantity, int slot, double *out);
/* The same quantity of a 3-D field resized to rows x cols by
 * PostProcessingModule::resizeMatrix (src/postProcessing.cpp:29-49: block
 * means, the matrix unchanged unless both dimensions shrink), as the
 * modules do after setExportDimensions; out holds rows x cols doubles
 * (column-major), or the full field when it is not resized. */
int pxp_get_post_resized(pxp_solver s, int quantity, int slot, unsigned rows, unsigned cols,
                         double *out);
/* Largest |u| over the filled save slots (0 when none): the scale of
 * post::IntensityUint8 (src/postProcessMod.cpp:23, abs of the complex
 * maximum by modulus). */
int pxp_saved_max_abs(pxp_solver s, double *max_abs);

/* post::FarField (src/farFieldPost.cpp:22-62, 141-247; include/postProcessMod.hpp:68-123)
 * of the last solution, computed on the device.
 *   2-D kinds: the exit field centred in a line of pad_length entries filled
 *     with pad_value (ParaxialSimulation::setFarFieldPadValue; the bare field
 *     when pad_length is below Nx), |FFT| / sqrt(L), fftshift, the angular
 *     window along x: rows = window length, cols = 1.  `padding` and the
 *     export and reference fields are not used (the reference's 2-D result
 *     does not use them).
 *   3-D kinds: L = max(pad_length, Ny, Nx); the field minus the reference
 *     (when subtract_reference; see pxp_set_reference); columns padded to L
 *     (zero or constant padding), transformed, fftshifted and cut to the
 *     window along y; then the conjugated rows of that (Armadillo's .t() of
 *     a complex row) likewise along x; |.|^2 / L; then
 *     PostProcessingModule::resizeMatrix (src/postProcessing.cpp:29-49) to
 *     export_rows x export_cols when both are set and both smaller.
 * The window of an axis is farFieldAngleToIndx(phi_min) ..
 * farFieldAngleToIndx(phi_max) (:78-101) with that axis' step.  Output:
 * rows x cols doubles, column-major (an arma::mat), shape from
 * pxp_farfield_shape.  PXP_PAD_LINEAR_FIT (GSL fits, marked untested in the
 * reference) and L above 2^22 return PXP_ERR_UNSUPPORTED; an empty window
 * (phi_max below phi_min) PXP_ERR_INVALID. */
#define PXP_PAD_ZERO 0
#define PXP_PAD_LINEAR_FIT 1
#define PXP_PAD_CONSTANT 2
typedef struct pxp_farfield_params {
  unsigned pad_length;       /* FarField::setPadLength (default 0) */
  double phi_min, phi_max;   /* FarField::setAngleRange, degrees (-90, 90) */
  int padding;               /* FarField::setPadding, 3-D (PXP_PAD_ZERO) */
  double pad_value_re, pad_value_im; /* 2-D padded entries (0) */
  unsigned export_rows, export_cols; /* setExportDimensions, 3-D (0, 0: none) */
  int subtract_reference;    /* FarField::setReference, 3-D (0) */
} pxp_farfield_params;
/* Fills pxp_farfield_params with the reference's defaults. */
void pxp_farfield_defaults(pxp_farfield_params *p);
int pxp_farfield_shape(pxp_solver s, const pxp_farfield_params *p, unsigned *rows, unsigned *cols);
int pxp_farfield(pxp_solver s, const pxp_farfield_params *p, double *out);
/* The field FarField subtracts (GenericScattering's reference run,
 * src/genericScattering.cpp:160-178): a host array in the layout of
 * pxp_get_last_solution (Nx*Ny complex128), or NULL to clear. */
int pxp_set_reference(pxp_solver s, const double *field);
/* The same, from another handle's current field on the same device (same
 * grid size), copied on the device. */
int pxp_set_reference_from(pxp_solver s, pxp_solver src);

/* post::Transmittivity (src/transmittivity.cpp:30-83) for the 2-D kinds:
 * the trapezoid sum of pow(|u|, 2) over an index window [a, b] (weights 1
 * at a and b, 2 between: trapezoidalIntegrateIntensityZ, :30-41, without
 * its factor dx/2), computed by the step kernels as they store each new
 * field.  pxp_set_flux_windows gives one window per step for steps
 * first_step .. first_step + count - 1 (count = 0 clears; a <= b < Nx);
 * pxp_get_flux returns the sums of those steps (NaN for steps not run
 * yet); pxp_field_flux sums the current field over one window. */
int pxp_set_flux_windows(pxp_solver s, int first_step, int count, const unsigned *start,
                         const unsigned *end);
int pxp_get_flux(pxp_solver s, int first_step, int count, double *out);
int pxp_field_flux(pxp_solver s, unsigned start, unsigned end, double *sum);

/* Solver::reset (include/solver.hpp:30): step counter back to 1. */
int pxp_reset(pxp_solver s);

/* Next step index (Solver::currentStep). */
int pxp_current_step(pxp_solver s, unsigned *step);

/* Grid shape of the handle: Nx, Ny (1 for 2-D kinds), Nz. */
int pxp_shape(pxp_solver s, unsigned *nx, unsigned *ny, unsigned *nz);

/* ---- batching and serving (no reference counterpart: the reference runs
 * one problem at a time on the host) ------------------------------------- */

/* Device memory a solver holds (field, saves, tables). */
int pxp_device_bytes(pxp_solver s, size_t *bytes);

/* |u|^2 of the current field, Nx (or Ny*Nx column-major) doubles. */
int pxp_get_intensity(pxp_solver s, double *intensity);

typedef struct pxp_batch_s *pxp_batch;

/* A set of independent solvers advanced together on one device, admitted
 * against a device-memory budget (bytes). */
int pxp_batch_create(int device, size_t hbm_budget_bytes, pxp_batch *out);
int pxp_batch_destroy(pxp_batch b);

/* Admit a solver (created, material and initial conditions set) that is to
 * advance nsteps more steps.  PXP_ERR_NOT_READY (and no admission) when its
 * device memory would exceed the budget.  The solver stays owned by the
 * caller; it must not be stepped or destroyed while admitted. */
int pxp_batch_admit(pxp_batch b, pxp_solver s, int nsteps);

/* One round: every admitted solver with steps left advances by up to
 * max_steps steps.  2-D solvers of equal kind, size, precision and matrix
 * path share one launch (one CTA, or a cluster of CTAs, per solver, each
 * with its own step count); the groups run concurrently on streams of
 * their own, and 3-D solvers run their passes on their solvers' streams.
 * Asynchronous. */
int pxp_batch_round(pxp_batch b, int max_steps);

/* Wait for the round, then hand back (and remove from the batch) the
 * solvers that have no steps left: up to cap of them in done[], their number
 * in *count.  Their memory leaves the batch budget. */
int pxp_batch_collect(pxp_batch b, pxp_solver *done, int cap, int *count);

/* Solvers admitted and device memory charged to the budget. */
int pxp_batch_status(pxp_batch b, int *active, size_t *bytes);

/* ADI steps (Solver3D::step with the ADI solver) on a field the caller owns
 * in device memory, without allocating any device memory.  This has no
 * counterpart in the reference: it is for callers that must not allocate
 * device memory while they run -- code whose device memory is already carved
 * up by another allocator (a framework's caching allocator or a fixed pool),
 * and latency-critical loops, where cudaMalloc/cudaFree can synchronise the
 * device and stall other streams.
 *
 * dfield: Ny x Nx column-major field in the problem's precision (complex128
 * for PXP_FP64, complex64 for PXP_FP32), advanced in place by steps
 * first_step .. first_step+nsteps-1.  spheres: first-hit sphere material
 * (at most 16 may meet any one half-step plane).  stream: cudaStream_t to
 * launch on (NULL: the default stream); the call is asynchronous.
 *
 * The intermediate field between the x and y half steps lives in a fixed
 * 4 MiB array compiled into the library (every GPU that loads the library
 * holds it until the process exits): grids needing more (n*n*16 bytes in
 * FP64, n*n*8 in FP32; at most 512^2 in FP64) are rejected with
 * PXP_ERR_UNSUPPORTED and a message.  All calls on a device share that
 * array, so calls that overlap on the GPU race and must be serialised by the
 * caller.  The first call on each device looks up the array's device
 * address; make that first call before any stream capture.  The call makes
 * problem->device current for its launches and restores the caller's
 * current device before returning.  Every sampled plane is checked before
 * the first launch, so a refused call leaves the field untouched.  Errors
 * are reported through pxp_last_error(NULL, ...). */
int pxp_adi_steps_noalloc(const pxp_problem *problem, const pxp_sphere *spheres, int nspheres,
                          void *dfield, unsigned first_step, int nsteps, void *stream);

/* Failure-path self-test, no reference counterpart.  The propagation
 * kernels wait for their asynchronous copies with a bounded wait; when one
 * runs out the kernel counts it and returns instead of hanging, and the next
 * pxp_synchronize (or result copy) of every handle on that device reports
 * PXP_ERR_CUDA.  This launches, on the handle's stream, a one-thread kernel
 * whose wait (limit_ns of GPU time, at most 10 s) can never be satisfied,
 * so that a test can check that path without a fault; the handle's later
 * calls then report the error, and handles created afterwards are not
 * affected. */
int pxp_selftest_bounded_wait(pxp_solver s, unsigned long long limit_ns);

/* Last error message of the handle (NULL handle: last global error). */
int pxp_last_error(pxp_solver s, char *buf, size_t len);

/* Static text for a status code. */
const char *pxp_status_string(int status);

/* Build information: kernel architecture and version string. */
const char *pxp_build_info(void);

#ifdef __cplusplus
}
#endif
#endif /* PAXPRO_B200_H */
