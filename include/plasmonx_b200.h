/*
 * plasmonx_b200 -- C ABI of the B200 (sm_100a) per-frequency response solve.
 *
 * Drop-in boundary for the plasmonX solver layer.  The reference has no FFI;
 * its de-facto boundary is the type-bound procedure set of `target_type`
 * (src/target/target_module.f90:20-133) called from the per-frequency loops
 * of src/solvers/algorithm_module.f90:189-465, plus the free routines
 * `gmres_solver` (src/solvers/gmres_module.f90:30-31) and `complex_inversion`
 * (src/solvers/algorithm_module.f90:510).  Each entry point below names the
 * reference interface it replaces.
 *
 * Conventions (match the reference's Fortran data so that an iso_c_binding
 * interface can pass its arrays unchanged):
 *   - all pointers are HOST pointers; the library owns every device buffer and
 *     copies in and out;
 *   - complex values are interleaved (re, im) doubles (Fortran complex(dp));
 *   - matrices are column-major; "n_var x 3" means 3 contiguous columns;
 *   - unknowns are ordered as the reference orders them: charges q_1..q_N,
 *     then dipoles mu_1x, mu_1y, mu_1z, ..., mu_Nz;
 *   - lengths are bohr, frequencies atomic units;
 *   - every call returns a plx_status; nothing calls exit/stop.  The text of
 *     the last error of a context is available from plx_last_error().
 * Thread safety: one context may be used by one host thread at a time.
 */
#ifndef PLASMONX_B200_H
#define PLASMONX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct plx_ctx plx_ctx;
typedef struct plx_geom plx_geom;

typedef enum {
    PLX_OK = 0,
    PLX_ERR_ARG = 1,            /* invalid argument (null pointer, size, enum) */
    PLX_ERR_CUDA = 2,           /* CUDA runtime / library failure */
    PLX_ERR_NOMEM = 3,          /* device allocation failed */
    PLX_ERR_BUDGET = 4,         /* request exceeds the context's HBM budget */
    PLX_ERR_NOT_CONVERGED = 5,  /* GMRES ran out of Krylov dimension (the
                                   reference stops with "GMRES not converged
                                   and restart GMRES NYI.") */
    PLX_ERR_NAN = 6,            /* non-finite value met in a residual */
    PLX_ERR_SINGULAR = 7,       /* zgetrf reported info != 0 */
    PLX_ERR_UNSUPPORTED = 8     /* model / mode combination not provided */
} plx_status;

typedef enum {
    PLX_WFQ = 0,
    PLX_WFQFMU = 1,
    PLX_BEM_DPCM = 2,           /* bem variant dpcm   (src/bem/bem_module.f90) */
    PLX_BEM_IEF = 3             /* bem variant iefpcm */
} plx_model;

typedef enum {
    PLX_INVERSION = 0,          /* solve_w_inversion  (algorithm_module.f90:189) */
    PLX_GMRES_MEM = 1,          /* solve_w_iter_mem   (algorithm_module.f90:334) */
    PLX_GMRES_OTF = 2           /* solve_w_iter_on_the_fly (algorithm_module.f90:417) */
} plx_mode;

typedef enum {
    PLX_FP64 = 0,               /* plain complex FP64 GMRES, the drop-in (the
                                   reference's algorithm step by step) */
    PLX_MIXED_BF16X3 = 1,       /* FP64 iterative refinement around an inner
                                   GMRES whose T contraction runs on the tensor
                                   cores with BF16-split operands (3 products,
                                   FP32 accumulation) */
    PLX_FP64_REFINED = 2,       /* the same refinement with an FP64 inner solve:
                                   restarted, with explicit FP64 residuals */
    PLX_MIXED_BF16 = 3          /* refinement with a single BF16 product inside */
} plx_precision;

/* Geometry and model parameters, i.e. what the reference holds in `target_`
 * and `parameters` after input (src/input_output/input_module.f90:156-258,
 * src/wfq/wfq_module.f90:96-127).  Per-type arrays have n_types entries;
 * fermi_d/fermi_s/r0 are n_types x n_types column-major ((i,j) at i + j*n_types);
 * r0 is the nearest-neighbour distance of the type pair (target_module.f90:472). */
typedef struct {
    int32_t model;              /* plx_model */
    int32_t n_atoms;
    int32_t n_types;
    int32_t rhs_potential;      /* 0: V = -E0 r ("field"), 1: V = -E0 |r - r_min| */
    const double *coord;        /* 3 x n_atoms, bohr */
    const int32_t *atom_type;   /* n_atoms, 0-based */
    const int32_t *neighbours;  /* n_types x n_atoms counts (target_module.f90:417) */
    const int32_t *n_neighbours;/* n_atoms */
    const double *eta;          /* chemical hardness (T_qq diagonal) */
    const double *r_q;          /* Gaussian charge width */
    const double *r_mu;         /* Gaussian dipole width (wFQFMu) */
    const double *tau;          /* Drude relaxation time, after sigma0/tau scaling */
    const double *density;      /* n = sigma0 / tau before scaling */
    const double *a_ij;         /* effective area A_ij */
    const double *fermi_d;      /* Fermi damping d, type pair */
    const double *fermi_s;      /* Fermi damping s, type pair */
    const double *r0;           /* nearest-neighbour distance, type pair (bohr) */
    double e0;                  /* field intensity (a.u.) */
} plx_geometry_desc;

/* Boundary-element surface (bem_type after read_gmsh_file and create_tesserae,
 * src/bem/bem_module.f90:224-491).  The triangles are given by their three
 * corners, [n_tess][3 vertices][x, y, z] in bohr, in the order of the mesh's
 * element block; the normal of a tessera is normal_factor * (v1-v0) x (v2-v0). */
typedef struct {
    int32_t variant;            /* PLX_BEM_DPCM or PLX_BEM_IEF */
    int32_t n_tess;
    int32_t accurate;           /* Green function: 0 approximate (diagonal
                                   1.0694 sqrt(4 pi a) / (2 R)), 1 accurate
                                   (accurate_green_function.f90) */
    const double *triangles;
    double normal_factor;       /* +1 or -1 (`bem normal scalar factor`) */
    double sphere_radius;       /* R of the approximate diagonal (bohr) */
    double eps_solvent;         /* `bem epsilon solvent` */
    double e0;                  /* field intensity (a.u.) */
} plx_bem_desc;

/* One solve request over the frequencies set by plx_set_frequencies. */
typedef struct {
    int32_t mode;               /* plx_mode */
    int32_t precision;          /* plx_precision */
    int32_t pol_mask;           /* bit0 x, bit1 y, bit2 z (reference 'all' = 7) */
    int32_t max_krylov;         /* GMRES dimension m (reference `gmres dimension`) */
    double tol;                 /* absolute residual tolerance, already multiplied
                                   by sqrt(n_var) as input_module.f90:250-251 does */
    int32_t freq_block;         /* frequencies solved together; 0 = automatic */
    int32_t record_trace;       /* 1: fill trace_out with the logged residuals */
    /* refinement (precision != PLX_FP64): inner Krylov dimension, inner
     * relative tolerance, maximum outer steps; 0 selects the defaults
     * (64, 1e-4, 60) */
    int32_t inner_krylov;
    double inner_tol;
    int32_t max_outer;
} plx_solve_desc;

/* ---- context --------------------------------------------------------------- */

/* Creates a context on CUDA device `device`.  hbm_budget_bytes = 0 means the
 * free device memory at creation.  Returns NULL only on allocation failure of
 * the host object; device errors are reported by later calls. */
plx_ctx *plx_ctx_create(int32_t device, uint64_t hbm_budget_bytes);
void plx_ctx_destroy(plx_ctx *ctx);
const char *plx_last_error(const plx_ctx *ctx);
/* Device bytes currently held by the context (geometries + solver state). */
uint64_t plx_ctx_bytes_in_use(const plx_ctx *ctx);
/* Kernels the library has launched on this context since its creation (its own
 * kernels; cuBLAS / cuSOLVER launches are not counted). */
int64_t plx_ctx_launches(const plx_ctx *ctx);

/* ---- geometry -------------------------------------------------------------- */

/* Uploads coordinates and parameters and builds, once per geometry, the
 * frequency-independent data on the device: the sparse Drude/Fermi
 * conductance K (construct_K_minus_P_matrix, matrix_module.f90:393-426) as a
 * CSR matrix, and -- when store_t != 0 -- the dense interaction matrix T
 * (construct_static_t_qq/qmu/muq/mumu, matrix_module.f90:58-345) needed by the
 * on-memory and inversion modes.  `*out` receives the geometry handle. */
plx_status plx_geometry_create(plx_ctx *ctx, const plx_geometry_desc *desc,
                               int32_t store_t, plx_geom **out);
void plx_geometry_destroy(plx_geom *geom);
/* BEM counterpart of plx_geometry_create: builds the Green-function derivative
 * D (construct_constant_matrix_bem, bem_module.f90:678-782) once; with
 * PLX_BEM_IEF the direct solve also builds S A^-1 and D S A^-1 on first use.
 * plx_set_frequencies then takes eps(w) (complex, one per frequency) in alpha_w.
 * The reference has no on-the-fly BEM product; PLX_GMRES_OTF is refused. */
plx_status plx_bem_create(plx_ctx *ctx, const plx_bem_desc *desc, plx_geom **out);
/* Induced field and plasmon density at points: the analysis step of the
 * reference (calculate_induced_field_at_point_{wfq,wfqfmu} and
 * calculate_density_at_point_{wfq,wfqfmu}, src/wfq/wfq_module.f90:590-650,
 * src/wfq/wfqfmu_module.f90:975-1040).  x: one solution (complex, n_var,
 * reference ordering) for polarisation i_pol (0 x, 1 y, 2 z), whose external
 * field E0 is included in the field; points: 3 x n_points, bohr,
 * column-major; field_out: 3 x n_points complex, density_out: n_points
 * complex (either may be NULL).  Atomistic models only. */
plx_status plx_field_at_points(plx_geom *geom, int32_t i_pol, const double *x, int32_t n_points,
                               const double *points, double *field_out, double *density_out);
/* BEM field at points for the analysis step (calculate_induced_field_at_point_bem,
 * src/bem/bem_module.f90:1152-1222): the tesserae as point charges q (complex
 * n_tess, the area-weighted charges a run's .freq file holds) at their centres
 * (3 x n_tess, bohr); a point whose distance to the centres' mean exceeds its
 * nearest tessera's by more than 0.5 Angstrom sees E0 along i_pol plus the
 * charges' field, any other point zero.  points: 3 x n_points, bohr;
 * field_out: 3 x n_points complex.  Needs no geometry (the analysis of a run's
 * archive has the centres and charges only). */
plx_status plx_bem_field_at_points(plx_ctx *ctx, int32_t n_tess, const double *centres, const double *q, double e0,
                                   int32_t i_pol, int32_t n_points, const double *points, double *field_out);
/* get_neighbours (src/target/target_module.f90:417-464) on the device: per atom
 * the number of atoms within the nearest-neighbour distance r0 of the pair
 * (counting the atom itself) and the per-type counts the wFQFMu dipole diagonal
 * divides by it.  coord_ang: 3 x n_atoms in ANGSTROM -- the reference tests
 * sqrt(dx^2 + dy^2 + dz^2) * ToBohr <= r0 on the input coordinates, and the
 * same expression is evaluated here without fused operations; atom_type
 * 0-based; type_z the atomic number of each type; r0: n_types x n_types, bohr.
 * Out: neighbours_out n_types x n_atoms (the `neighbours` array of
 * plx_geometry_desc), n_neighbours_out n_atoms.  At most 16 atom types. */
plx_status plx_neighbour_counts(plx_ctx *ctx, int32_t n_atoms, int32_t n_types, const double *coord_ang,
                                const int32_t *atom_type, const int32_t *type_z, const double *r0,
                                int32_t *neighbours_out, int32_t *n_neighbours_out);
/* Number of unknowns n_var (N for wFQ, 4N for wFQFMu, n_tess for BEM). */
int64_t plx_geometry_n_var(const plx_geom *geom);
/* Stored non-zeros of K (both triangles). */
int64_t plx_geometry_k_nnz(const plx_geom *geom);

/* Sets the frequency grid (field%freq, field_module.f90:157-176) and, for
 * wFQFMu, the interband polarizability alpha_t(w) of every atom type
 * (parameters%alpha_w, wfqfmu_module.f90:97-166): alpha_w is complex
 * n_types x n_freq column-major.  alpha_w may be NULL for wFQ. */
plx_status plx_set_frequencies(plx_geom *geom, int32_t n_freq, const double *omega,
                               const double *alpha_w);

/* ---- reference-shaped kernels --------------------------------------------- */

/* y = A(w_i) x: product_matrix_vector followed by new_gmres_diagonal_shift
 * (target_module.f90:1340-1356, 1392-1408; wfq_module.f90:321-424;
 * wfqfmu_module.f90:584-746).  x, y: complex n_var.  on_the_fly = 0 uses the
 * stored T, 1 generates the interaction tiles in the kernel. */
plx_status plx_matvec(plx_geom *geom, int32_t i_freq, int32_t on_the_fly,
                      const double *x, double *y);

/* Dynamic right-hand sides b(w_i), complex n_var x 3
 * (construct_dynamic_field_rhs[_on_the_fly] + assign_variables_w[_on_the_fly],
 * wfq_module.f90:260-301, wfqfmu_module.f90:177-430, rhs_module.f90:43-430).
 * Columns of polarisations not in pol_mask are zero. */
plx_status plx_rhs(plx_geom *geom, int32_t i_freq, int32_t pol_mask, double *b);

/* gmres_solver (gmres_module.f90:30-228) for one column: x holds the RHS on
 * entry and the solution on exit; tol is absolute; restart is the Krylov
 * dimension.  steps_out (optional) receives the number of Arnoldi steps and
 * trace_out (optional, restart doubles) the logged residuals. */
plx_status plx_gmres_solver(plx_geom *geom, int32_t i_freq, double *x, int32_t on_the_fly,
                            double tol, int32_t max_iter, int32_t restart,
                            int32_t *steps_out, double *trace_out);

/* complex_inversion (algorithm_module.f90:510-541) on A(w_i): zgetrf + zgetrs
 * with the 3 columns of variables_w (complex n_var x 3, RHS in / solution out). */
plx_status plx_complex_inversion(plx_geom *geom, int32_t i_freq, double *variables_w);

/* ---- the spectrum solve --------------------------------------------------- */

/* Solves every frequency of the grid: the three per-frequency loops of
 * algorithm_module.f90:189-465 with calculate_dynamic_polar and
 * calculate_cross_section (target_module.f90:1989-2054) fused in.
 *   x_out      optional, complex n_var x 3 x n_freq (variables_w per frequency);
 *              columns that were not solved hold the right-hand side, as in
 *              the reference
 *   polar_out  optional, complex 3 x 3 x n_freq (polar_w, column b = field b)
 *   results_out optional, n_freq x 20 row-major (target_%results(i,1:20))
 *   status_out optional, n_freq plx_status values
 *   steps_out  optional, 3 x n_freq Arnoldi step counts (0 if not solved)
 *   trace_out  optional, max_krylov x 3 x n_freq logged residuals (record_trace)
 * Returns the first non-OK per-frequency status, or PLX_OK. */
plx_status plx_solve(plx_geom *geom, const plx_solve_desc *desc, double *x_out,
                     double *polar_out, double *results_out, int32_t *status_out,
                     int32_t *steps_out, double *trace_out);

/* S = T X for `count` real columns (X, S: count x n_var, each column
 * contiguous), the frequency-independent contraction inside
 * product_q_block_x / product_mu_block_x (matrix_module.f90:727-1001).
 * how: 0 stored T in FP64, 1 tiles generated on the fly in FP64, 2 tensor
 * cores with BF16-split operands (3 products), 3 tensor cores, one BF16
 * product. */
plx_status plx_contract(plx_geom *geom, int32_t count, const double *X, double *S, int32_t how);

/* Allocation-free S = T X (FP64, stored T) for callers that cannot allocate
 * device memory -- their buffers come from another runtime's allocator, a
 * preallocated serving pool, or a timed loop that must not synchronise on
 * allocation calls.  No counterpart in the reference: it is the few-column
 * case of plx_contract (how = 0) with DEVICE pointers d_X, d_S (count x n_var,
 * each column contiguous) owned by the caller, and it allocates nothing.
 * Its scratch is a fixed file-scope device array of 2^21 doubles (16 MiB per
 * GPU that loads the library, held until exit); 1 <= count <= 16 and the
 * split-K partials (k-chunks x count x n_var) must fit in it, otherwise the
 * call returns PLX_ERR_ARG.  The first call on a device looks up the array's
 * device address.  All calls share the array: calls whose kernels overlap on the GPU race.  The
 * kernels run on the context's own stream, which is not ordered after the
 * caller's streams: d_X must be completely written on the device before the
 * call (synchronise the stream that wrote it).  The call synchronises the
 * context's stream and returns when S is written. */
plx_status plx_contract_noalloc(plx_geom *geom, int32_t count, const double *d_X, double *d_S);

/* ---- continuous batching ------------------------------------------------- */

/* A refinement solve (precision PLX_MIXED_BF16X3, PLX_MIXED_BF16 or
 * PLX_FP64_REFINED; mode PLX_GMRES_MEM or PLX_GMRES_OTF) whose columns come and
 * go while others are in flight: the per-frequency loops of
 * algorithm_module.f90:334-465 turned into a serving loop.  A request (a grid
 * of frequencies and polarisations with its own absolute tolerance) added with
 * plx_batch_add joins the batch at the next plx_batch_step, which runs ONE outer
 * refinement step (inner GMRES cycles on the tensor cores, then the FP64
 * residual) for every active column of every request; plx_batch_poll reports a
 * request whose columns have all finished and plx_batch_take returns its
 * results (as plx_solve does for its grid) and frees its columns.  While a
 * batch is open it owns the geometry's frequency table (plx_set_frequencies is
 * refused); close the batch before destroying the geometry.  No counterpart in
 * the reference, whose GMRES calls are serialised (algorithm_module.f90:382-385). */
typedef struct plx_batch plx_batch;
/* desc: mode, precision, inner_krylov, inner_tol, max_outer (tol and the other
 * fields are not used; each request brings its own tolerance). */
plx_status plx_batch_open(plx_geom *geom, const plx_solve_desc *desc, plx_batch **out);
/* A request: tag (distinct, >= 0), n_freq frequencies (a.u.), alpha_w as in
 * plx_set_frequencies (n_types x n_freq complex; eps(w) for BEM; NULL for
 * wFQ), polarisations pol_mask, absolute residual tolerance tol. */
plx_status plx_batch_add(plx_batch *b, int64_t tag, int32_t n_freq, const double *omega, const double *alpha_w,
                         int32_t pol_mask, double tol);
/* One outer step of every active column; n_active (optional) receives the
 * number of columns still being solved afterwards.  plx_last_solve_ms of the
 * geometry then holds the step's device time. */
plx_status plx_batch_step(plx_batch *b, int32_t *n_active);
/* One outer step of several batches (one per geometry, all on one context):
 * every inner Arnoldi step of all of them is ONE grouped tensor-core launch
 * over their operands, in place of the reference's one frequency per thread
 * (algorithm_module.f90:224-265, 365-405). */
plx_status plx_batch_step_group(plx_batch *const *batches, int32_t count, int32_t *n_active);
/* The tag of the earliest request whose columns have all finished, or -1. */
plx_status plx_batch_poll(plx_batch *b, int64_t *tag);
/* Results of a finished request (each output optional): polar_out complex
 * 3 x 3 x n_freq, results_out n_freq x 20, status_out n_freq, steps_out
 * 3 x n_freq inner Arnoldi steps; frees its columns.  Returns the first
 * non-OK status of its frequencies, or PLX_OK. */
plx_status plx_batch_take(plx_batch *b, int64_t tag, double *polar_out, double *results_out, int32_t *status_out,
                          int32_t *steps_out);
/* Columns still being solved. */
int32_t plx_batch_active(const plx_batch *b);
void plx_batch_close(plx_batch *b);

/* ---- static FQ / FQFMu ---------------------------------------------------- */

/* The static force fields whose types the w-models extend
 * (src/forcefield/fq_module.f90, src/forcefield/fqfmu_module.f90): charges
 * (and, for FQFMu, dipoles) under electronegativity equalisation with one
 * charge constraint per molecule, for the ground state or a static field. */
typedef enum {
    PLX_STATIC_FQ = 0,          /* n_var = n_atoms + n_mol */
    PLX_STATIC_FQFMU = 1        /* n_var = 4 n_atoms + n_mol: charges, constraints, dipoles */
} plx_static_forcefield;

typedef enum {                  /* T_qq kernel (construct_static_t_qq, matrix_module.f90:58-115) */
    PLX_KERNEL_COULOMB = 0,     /* 1/r, eta on the diagonal */
    PLX_KERNEL_OHNO = 1,        /* eta_ij / sqrt(1 + eta_ij^2 r^2), eta_ij the mean hardness */
    PLX_KERNEL_GAUSSIAN = 2     /* erf(r / sqrt(r_qi^2 + r_qj^2)) / r, eta on the diagonal */
} plx_charge_kernel;

typedef enum {
    PLX_GROUND_STATE = 0,       /* solve_ground_state (algorithm_module.f90:91-115): rhs -chi */
    PLX_STATIC_FIELD = 1        /* solve_static_field (algorithm_module.f90:120-145): 3 rhs */
} plx_static_what;

/* Geometry and parameters of a static problem (target_ after input).  Molecules
 * are runs of consecutive atoms (create_n_atoms_per_molecule,
 * src/input_output/input_module.f90:1007-1030); the constraint rows follow the
 * reference's indexing (add_lagrangian_blocks, matrix_module.f90:351-382), exact
 * for molecules of equal size; a geometry whose indexed rows would run past the
 * atoms is refused with PLX_ERR_ARG. */
typedef struct {
    int32_t forcefield;         /* plx_static_forcefield */
    int32_t kernel;             /* plx_charge_kernel */
    int32_t n_atoms;
    int32_t n_types;
    int32_t n_mol;
    int32_t rhs_potential;      /* static field: 0 V = -E0 r ("field"), 1 V = -E0 |r - r_min| */
    const double *coord;        /* 3 x n_atoms, bohr */
    const int32_t *atom_type;   /* n_atoms, 0-based */
    const int32_t *atoms_per_molecule;  /* n_mol */
    const double *chi;          /* electronegativity, per type */
    const double *eta;          /* chemical hardness, per type */
    const double *alpha;        /* polarizability (FQFMu), per type; may be NULL for FQ */
    const double *r_q;          /* Gaussian charge width (Gaussian kernel, FQFMu) */
    const double *r_mu;         /* Gaussian dipole width (FQFMu) */
    double e0;                  /* field intensity (a.u.) */
    int32_t factorization;      /* 0 automatic: the charge constraints eliminated on a
                                   null-space basis and the rest factored by a
                                   double-precision Cholesky, LU of the full system where
                                   that does not apply; 1 LU of the full system (the
                                   reference's form); 2 as 0 with the Cholesky factor in
                                   single precision and double-precision iterative
                                   refinement (LAPACK dsposv's algorithm); 3 as 0 with
                                   the reduced system factored by the library's own
                                   blocked Cholesky kernels instead of cuSOLVER's */
} plx_static_desc;

/* n_var of a static problem, or -1 for an invalid description. */
int64_t plx_static_n_var(const plx_static_desc *desc);

/* Builds the static matrix and right-hand side on the device and solves them
 * (construct_static_matrix, construct_ground_state_rhs /
 * construct_static_field_rhs and real_inversion, algorithm_module.f90:91-145,
 * :469-504).  Outputs (each may be NULL):
 *   variables  n_var x n_rhs column-major, n_rhs = 1 (ground state) or 3
 *              (static field x, y, z): target_%variables
 *   energy     ground state: -1/2 x.b (calculate_energy_fq, fq_module.f90:358-374)
 *   polar      static field, FQ: the 3 x 3 static polarizability, column-major
 *              (calculate_static_polar_fq, fq_module.f90:379-595).  FQFMu
 *              returns PLX_ERR_UNSUPPORTED, as the reference stops there. */
plx_status plx_static_solve(plx_ctx *ctx, const plx_static_desc *desc, int32_t what, double *variables,
                            double *energy, double *polar);

/* rotate_principal_axis (src/target/target_module.f90:684-835), host only:
 * moves the centre of mass (standard atomic masses by atomic number) to the
 * origin and rotates coord (3 x n_atoms, in place) onto the eigenvectors of the
 * inertia tensor, in ascending order of the eigenvalues.  Each eigenvector's
 * sign (left to the implementation by LAPACK) makes its last nonzero component
 * positive.  eigenvalues (3) and axes (3 x 3 column-major, the eigenvectors)
 * may be NULL.  An atomic number without a mass returns PLX_ERR_ARG. */
plx_status plx_principal_axes(int32_t n_atoms, const int32_t *atomic_number, double *coord, double *eigenvalues,
                              double *axes);

/* Device time (ms, CUDA events on the library's stream) of the last plx_solve,
 * and the number of kernels it launched. */
double plx_last_solve_ms(const plx_geom *geom);
int64_t plx_last_solve_launches(const plx_geom *geom);

/* ---- measurement -------------------------------------------------------- */

/* When enabled, the library brackets the sections of the iterative solvers
 * with CUDA events on its stream and accumulates their device time per
 * category: 0 tensor-core T contraction, 1 FP64 T contraction, 2 Arnoldi
 * orthogonalisation, 3 conductance and diagonal rows of the operator,
 * 4 least squares and solution updates, 5 static matrix and right-hand-side
 * build (plx_static_solve), 6 static dense LU factorisations and solves,
 * 7 field and density at points (plx_field_at_points, plx_bem_field_at_points:
 * the kernel alone), 8 neighbour counts (plx_neighbour_counts: the kernel
 * alone).  For the contractions it also accumulates, per launch, the
 * algorithmic flops (2 n_var^2 x real columns) and bytes (the stored T once at
 * its storage precision, the input and output columns); for 5 the bytes
 * written, for 6 the LU flops (2/3 n^3 + 2 n^2 n_rhs); for 7 and 8 the bytes
 * the kernel must read and write once (points, atoms or tesserae, results).
 * Enabling resets the counters. */
plx_status plx_profile_enable(plx_ctx *ctx, int32_t on);
/* Reads one category: accumulated time (ms), sections, flops and bytes. */
plx_status plx_profile_read(plx_ctx *ctx, int32_t category, double *ms, int64_t *launches, double *flops,
                            double *bytes);

/* ---- failure handling ------------------------------------------------------ */

/* Number of polls after which a pipeline wait inside the tensor-core kernels
 * (a copy or a matrix product that does not arrive) gives up; 0 restores the
 * default of 2^22 polls (seconds).  A kernel whose wait runs out lets every
 * copy and product it has started finish, frees its tensor memory, returns,
 * and the call reports PLX_ERR_CUDA ("... timed out waiting on its
 * pipeline"); the context stays usable.  No counterpart in the reference (its
 * CPU code has no such waits); tests shorten it to exercise that path. */
plx_status plx_set_wait_limit(plx_ctx *ctx, uint32_t polls);

#ifdef __cplusplus
}
#endif
#endif /* PLASMONX_B200_H */
