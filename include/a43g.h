/*
 * a43g -- B200 (sm_100a) Green-function action and tfQMR solver with a plain C ABI.
 *
 * The operator is AngstromCube's block-sparse Green-function action Y = (H - E S) X over
 * 4x4x4-point cubes.  X and Y hold nnzb blocks of 64x64 complex numbers in the reference's
 * R1C2 layout  real_t[nnzb][2][64][64]  ([block][re,im][target point][source column],
 * source columns fastest), so a block vector produced by the reference's action_t can be
 * handed to a43g_action_multiply unchanged.
 *
 * Every entry point returns an a43g status (0 = success) and never exits the process;
 * a43g_last_error() gives the message of the last failure on the calling thread.
 * Device pointers are plain CUDA device addresses; streams are cudaStream_t passed as void*.
 */
#ifndef A43G_H
#define A43G_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    A43G_OK = 0,
    A43G_ERR_ARGUMENT = 1,   /* invalid argument or inconsistent sizes */
    A43G_ERR_CUDA = 2,       /* a CUDA runtime call failed */
    A43G_ERR_STATE = 3,      /* missing prerequisite (e.g. no energy set) */
    A43G_ERR_MEMORY = 4,     /* device allocation failed */
    A43G_ERR_UNSUPPORTED = 5 /* feature not available for this plan */
};

enum { A43G_F64 = 0, A43G_F32 = 1 };            /* real_t of the R1C2 block vectors */

typedef struct a43g_plan a43g_plan_t;

/* Cell, boundary conditions, sources, truncation and atoms, i.e. the inputs of
 * green_function::construct_Green_function (src/green_function.cxx:357-365) plus the
 * control keys it reads (green_function.truncation.radius, green_function.sources.x/y/z,
 * green_kinetic.range, green_function.projection.radius). */
typedef struct {
    uint32_t ng[3];           /* grid points per direction, multiples of 4 */
    int32_t  bc[3];           /* 0 isolated, 1 periodic, 2 vacuum, 3 repeat */
    double   hg[3];           /* grid spacings in Bohr */
    double   r_trunc;         /* truncation radius in Bohr */
    double   sources[3];      /* source cubes per direction (box centred in the cell), <0: all */
    int32_t  nFD;             /* finite-difference range: 4 (8th order) or 8 (16th order) */
    double   proj_radius;     /* projector cut-off radius in units of sigma (reference default 6) */
    int32_t  natoms;
    const double *xyzZinso;   /* [natoms][8]: x,y,z relative to the cell centre, Z, id (= index), numax, sigma, unused */
} a43g_geometry_t;

/* Plan sizes, same keys as the reference's plan members */
typedef struct {
    int64_t nnzb, nRows, nCols, nAtoms, nAtomImages, ncoeff_images, ncoeffs;
    int64_t nlists[3], lists_nnz[3];
    int64_t SHOadd_nnz, SHOprj_nnz, SHOsum_nnz;
    int64_t FD_range[3];
    int64_t ncells;
} a43g_plan_sizes_t;

/* Host copies of the plan arrays (each pointer may be NULL to skip it); the layouts are
 * those of action_plan_t, kinetic_plan_t and dyadic_plan_t (include/action_plan.hxx:32-93,
 * include/kinetic_plan.hxx:163-199, include/dyadic_plan.hxx:14-47). */
typedef struct {
    uint32_t *rowstart; uint16_t *colindx; uint32_t *rowindx; int32_t *veff_index;
    uint32_t *subset; float *rowCubePos; float *colCubePos; int16_t *target_minus_source;
    double *grid_spacing_trunc; double *kinetic_prefactor;
    uint32_t *lists_start[3]; int32_t *lists[3];
    uint32_t *AtomStarts; int8_t *AtomLmax; double *AtomSigma; int64_t *global_atom_ids;
    uint32_t *AtomImageIndex; uint32_t *AtomImageStarts; double *AtomImagePos; int8_t *AtomImageLmax;
    int8_t *AtomImageShift; double *AtomImagePhase; double *grid_spacing_dyadic;
    uint32_t *SHOadd_start; uint32_t *SHOadd_col; uint32_t *SHOprj_start; uint32_t *SHOprj_col;
    uint32_t *SHOsum_start; uint32_t *SHOsum_col; double *AtomMatrices; double *phase;
} a43g_plan_export_t;

/* Solver options and per-solve statistics (tfQMR, Freund 1993, per-column scalars) */
enum {
    A43G_SOLVE_NO_RETIRE = 1,    /* FP64 solves: keep computing on finished source cubes (the reference's
                                    tfQMRgpu does); FP32 recurrences always retire them */
    A43G_SOLVE_PRECONDITION = 2  /* right preconditioning by the cube-diagonal local operator: M^-1 of
                                    the finite-difference kinetic energy inside each 4x4x4 cube plus its
                                    mean potential minus E, applied by three 4-point transforms and a
                                    scaling (no reference counterpart: the reference's action reports
                                    has_preconditioner() false); residuals and the solution are those
                                    of the original system.  Not with a43g_solve_traced; refused
                                    (A43G_ERR_ARGUMENT) where a cube model is singular, a real
                                    energy on one of its eigenvalues */
};

typedef struct {
    double   tolerance;       /* relative residual |B - A X| / |B| per column */
    int32_t  max_iterations;  /* tfQMR iterations (two operator applications each) */
    int32_t  precision;       /* A43G_F64: plain FP64 tfQMR; A43G_F32: FP32 recurrences and operator, FP64
                                 solution, convergence checked on the FP64 residual (residual replacement) */
    double   update_factor;   /* A43G_F32: a source cube replaces its residual when its largest estimate has
                                 fallen by this factor since its last replacement (0: default 0.1) */
    int32_t  update_gap;      /* A43G_F32: at most this many iterations between replacements (0: default 10) */
    int32_t  check_every;     /* iterations between convergence checks on the host */
    uint64_t seed;            /* seed of the random shadow residual */
    int32_t  echo;            /* log level: > 0 prints one line per solve, > 1 one per convergence check */
    int32_t  flags;           /* A43G_SOLVE_NO_RETIRE */
    int32_t  batch;           /* a43g_solve_batched: (energy, k-point) pairs per wave, 0: as many as fit */
    int32_t  pad;
} a43g_solve_options_t;

typedef struct {
    int32_t iterations;       /* tfQMR iterations performed (a batched pair: until its last source finished) */
    int32_t refinements;      /* residual replacements with the FP64 operator (most of any source cube) */
    int32_t converged;        /* 1 if every column reached the tolerance */
    int32_t breakdowns;       /* columns stopped by a rho or sigma breakdown */
    double  residual_max;     /* max over columns of the true relative residual (FP64) */
    double  residual_estimate;/* tfQMR residual bound at exit */
    double  operator_applications; /* action calls made */
    double  seconds;          /* device time of the solve (a batched pair: of its wave) */
    int32_t fp64_sources;     /* A43G_F32: source cubes whose FP32 recurrences stalled and that continued in FP64 */
    int32_t pad;
} a43g_solve_stats_t;

const char *a43g_last_error(void);
const char *a43g_version(void);

/* ---- plan: replaces construct_Green_function + action_plan_t (src/green_function.cxx:357-1068) */
int a43g_plan_build(const a43g_geometry_t *geometry, a43g_plan_t **plan);
/* the same plan, with the atom-image x target-row overlap test of the dyadic plan
 * (src/dyadic_plan.cxx:264-401, a serial loop in the reference) evaluated on the current CUDA
 * device; every array is identical to a43g_plan_build's */
int a43g_plan_build_device(const a43g_geometry_t *geometry, a43g_plan_t **plan);
int a43g_plan_destroy(a43g_plan_t *plan);
int a43g_plan_get_sizes(const a43g_plan_t *plan, a43g_plan_sizes_t *sizes);
int a43g_plan_export(const a43g_plan_t *plan, const a43g_plan_export_t *out);
/* replaces green_function::update_potential (src/green_function.cxx:114-211) for one rank:
 * layout 0 = full grid V[(iz*ng_y + iy)*ng_x + ix], layout 1 = cell cubes [ncells][64] */
int a43g_plan_set_potential(a43g_plan_t *plan, const double *V, int layout);
/* atom matrices per atom id, concatenated [2][nc][nc] (hmt, ovl), already multiplied by the
 * SHO prefactors as src/energy_contour.cxx:307-323 does; offsets[natoms] in doubles */
int a43g_plan_set_atom_matrices(a43g_plan_t *plan, const double *mats, const int64_t *offsets, int64_t natoms);
/* replaces green_function::update_energy_parameter (src/green_function.cxx:64-109) */
int a43g_plan_set_energy(a43g_plan_t *plan, double E_re, double E_im, double dVol);
/* replaces green_function::update_phases (src/green_function.cxx:218-251); k in units of 2 pi/cell */
int a43g_plan_set_kpoint(a43g_plan_t *plan, const double k[3]);
/* copies plan, potential and matrices to the device (done implicitly by the calls below) */
int a43g_plan_upload(a43g_plan_t *plan);

/* ---- the operator: replaces green_action::action_t<real_t,2,1,64>::multiply
 * (include/green_action.hxx:140-176).  y and x are device pointers to real_t[nnzb][2][64][64];
 * colIndex is the device array [nnzb] of block columns (as the reference passes it);
 * nnzb and nCols must match the plan; l2nX is accepted for interface compatibility.
 * flops (optional) receives the reference's flop count of one application. */
int a43g_action_multiply(a43g_plan_t *plan, void *y, const void *x, const uint16_t *colIndex,
                         uint32_t nnzb, uint32_t nCols, unsigned l2nX, void *stream, int dtype,
                         double *flops);

/* ---- the same action without any device allocation.  No counterpart in the reference (its
 * action allocates its projector scratch on every call).  For callers that must not let a
 * library allocate device memory: hosts whose memory pool owns all device memory, loops that
 * cannot afford the device-wide synchronization of cudaMalloc.
 * The projector coefficients live in one fixed 16 MiB array compiled into the library (present
 * on every GPU that loads it until the process exits); plans that need more are rejected with
 * A43G_ERR_UNSUPPORTED.  The plan must already be current on the calling device
 * (a43g_plan_upload after the last change of potential, matrices, energy or k-point), else
 * A43G_ERR_STATE.  The first call on each device looks up the array's device address; make it
 * before any stream capture.  The looked-up address is kept for the life of the process, so the
 * entry point must not be used on a device after a cudaDeviceReset of it.  All calls on a device
 * share the array: calls whose GPU work overlaps race on it and must be serialized by the caller.
 * Arguments as a43g_action_multiply. */
int a43g_action_multiply_noalloc(a43g_plan_t *plan, void *y, const void *x, const uint16_t *colIndex,
                                 uint32_t nnzb, uint32_t nCols, void *stream, int dtype, double *flops);

/* ---- one part of the operator, for profiling and for the adjoint kernels (no reference
 * counterpart; the reference applies the parts only together inside action_t::multiply):
 * part 0: y = (V - E) x + T x  (local potential and kinetic energy, include/green_potential.hxx
 *         and include/green_kinetic.hxx);  part 1: y += sum_a p_a M_a p_a^T x  (projectors,
 *         include/green_dyadic.hxx:856-922). */
int a43g_action_part(a43g_plan_t *plan, int part, void *y, const void *x, void *stream, int dtype);

/* ---- vector-Jacobian products of the action (no reference counterpart: the reference has no
 * derivatives, forces or adjoint).  For device FP64 block vectors L and G [nnzb][2][64][64]
 * the bilinear form  F = sum over blocks and columns of L^T (H - E S) G  (complex, without
 * conjugation) is differentiated with respect to
 *   dV: the local potential, host complex [ncells][64][2]  (cell-cube layout of a43g_plan_set_potential);
 *   dM: the atom matrices M_A = dVol (dH - E dS) of the plan's atoms (export AtomStarts and
 *       global_atom_ids give their order), host complex, per atom [2][nc][nc] (real plane, then
 *       imaginary plane), concatenated;
 *   dR: the atom positions, host complex [nAtoms][3][2] (x, y, z).
 * Any output may be NULL.  With G = (H - E S)^-1 B and L the adjoint Green function (the solve at
 * conj(E), conjugated, times the weights of a functional) -dF gives the gradient of that functional.
 * Synchronizes the stream. */
int a43g_vjp(a43g_plan_t *plan, const void *L, const void *G, double *dV, double *dM, double *dR, void *stream);

/* ---- autotuner (no reference counterpart): times the schedule parameters of the action for
 * this plan in the given precision on the current device (blocks per projection CTA, blocks per
 * addition CTA, local-kernel variant, CUDA-core or tensor-core FP32 projector) and keeps the
 * fastest for the plan's later calls; allocates two scratch block vectors for its duration.
 * report (optional) receives a text summary of the timings. */
int a43g_plan_autotune(a43g_plan_t *plan, int dtype, void *stream, char *report, size_t report_size);

/* synchronizes the device and reports an error a kernel of this plan recorded (for example a
 * bounded wait of the tensor-core projector that timed out); clears the record */
int a43g_plan_device_status(a43g_plan_t *plan);

/* number of CUDA kernels this library has launched in this process (instrumentation) */
uint64_t a43g_kernel_launches(void);

/* ---- tfQMR solve of (H - E S) X = B with B the unit blocks on the diagonal (plan subset);
 * replaces tfqmrgpu::solve + action_t::solve (include/green_action.hxx:181-241).
 * X: optional device pointer double[nnzb][2][64][64] receiving the FP64 solution (in both
 * precisions); rho: optional host array complex double [nCols][64][2] receiving the diagonal
 * of the diagonal blocks divided by pi, as action_t::solve exports it. */
int a43g_solve(a43g_plan_t *plan, const a43g_solve_options_t *opts, void *X, double *rho,
               a43g_solve_stats_t *stats, void *stream);

/* the same solve, recording every `every` iterations the relative error |X - X_reference| /
 * |X_reference| (Frobenius norms over all blocks) of the current solution (with FP32
 * recurrences: the FP64 solution plus the FP32 correction not yet added to it) against the
 * device FP64 block vector X_reference, for example the plain FP64 solution.  trace receives up
 * to `capacity` rows [iteration, relative error, sources still active], the last row the error
 * of the final solution (0 active sources); *count the number of rows recorded.  No reference counterpart (a diagnostic of the mixed-precision solver). */
int a43g_solve_traced(a43g_plan_t *plan, const a43g_solve_options_t *opts, void *X, double *rho,
                      a43g_solve_stats_t *stats, void *stream, const void *X_reference, int32_t every,
                      double *trace, int32_t capacity, int32_t *count);

/* ---- batched solve over (energy, k-point) pairs on one plan geometry: energies[n][2],
 * kpoints[n][3]; rho (optional) host [n][nCols][64][2]; stats[n].  No reference counterpart as
 * one call (the reference loops over its (E, k) points one solve at a time,
 * src/energy_contour.cxx:355-386): the pairs are solved in waves, each wave one block-sparse
 * system of all its pairs' source cubes with their own energies and Bloch phases, whose
 * finished source cubes stop costing work.  The plan keeps the batch's device arrays and
 * vectors for later calls (released with the plan). */
int a43g_solve_batched(a43g_plan_t *plan, const a43g_solve_options_t *opts, int32_t n,
                       const double *energies, const double *kpoints, double dVol,
                       double *rho, a43g_solve_stats_t *stats, void *stream);

/* ---- atomic density matrices: replaces green_dyadic::get_projection_coefficients
 * (include/green_dyadic.hxx:1062-1088, with SHOprj_right, :925-1060).  G: device FP64 block
 * vector [nnzb][2][64][64] (a Green function of this plan); out: host Im <p_i|G|p_j> of every plan
 * atom, [nSHO][nSHO] each, concatenated in the order of the export's global_atom_ids.  Plans with
 * periodic atom images (nAtomImages > nAtoms) are refused with A43G_ERR_UNSUPPORTED, as the
 * reference refuses them.  Synchronizes the stream. */
int a43g_projection_coefficients(a43g_plan_t *plan, const void *G, double *out, void *stream);

/* ---- the grid Hamiltonian file that a43 exports (Hmt.xml or Hmt.json): cell, boundary
 * conditions, spacing, the local potential on the full grid and the SHO atoms with their
 * Hamiltonian and overlap matrices. */
typedef struct a43g_hamiltonian a43g_hamiltonian_t;
/* replaces green_input::load_Hamiltonian (src/green_input.cxx:29-221; a name containing ".json"
 * is read as JSON, json_reading::load_Hamiltonian, include/json_reading.hxx:61-229, falling back
 * to XML) */
int a43g_hamiltonian_load(const char *filename, a43g_hamiltonian_t **h);
/* grid points, boundary conditions, spacings, number of atoms and of matrix doubles
 * (sum over atoms of 2 nSHO^2); any output may be NULL */
int a43g_hamiltonian_info(const a43g_hamiltonian_t *h, uint32_t ng[3], int32_t bc[3], double hg[3],
                          int32_t *natoms, int64_t *nmat);
/* copies out Veff [nz][ny][nx], xyzZinso [natoms][8] (x, y, z relative to the cell centre, Z,
 * global id, numax, sigma, 0), the matrices concatenated per atom [2][nSHO][nSHO] (hamiltonian,
 * overlap) and their offsets [natoms] in doubles; any output may be NULL */
int a43g_hamiltonian_get(const a43g_hamiltonian_t *h, double *Veff, double *xyzZinso, double *mats,
                         int64_t *offsets);
/* a Hamiltonian from arrays in the layouts of a43g_hamiltonian_get (to write one) */
int a43g_hamiltonian_create(const uint32_t ng[3], const int32_t bc[3], const double hg[3], const double *Veff,
                            int32_t natoms, const double *xyzZinso, const double *mats, const int64_t *offsets,
                            a43g_hamiltonian_t **h);
/* replaces grid_operators::write_to_file (include/grid_operators.hxx:460-613): format 0 XML,
 * 1 JSON; spectrum (optional) min, max, Fermi level in Hartree */
int a43g_hamiltonian_save(const a43g_hamiltonian_t *h, const char *filename, int format, const double *spectrum);
int a43g_hamiltonian_destroy(a43g_hamiltonian_t *h);

#ifdef __cplusplus
}
#endif
#endif /* A43G_H */
