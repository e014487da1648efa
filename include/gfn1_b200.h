/* C ABI of the B200 GFN1-xTB single-point engine (non-periodic SCC energy plus
 * analytic gradient).  Plain pointers and sizes only; no CUDA or torch types.
 *
 * Units: bohr and Hartree (the reference's Rust API units).  Matrices and
 * per-atom vectors are row-major, atoms in input order.
 *
 * Status codes: 0 = OK; 1..8 mirror the reference's Gfn1Error variants
 * (gfn1-rs src/error.rs:8-17); 9..12 are device-side conditions.
 */
#ifndef GFN1_B200_H
#define GFN1_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  GFN1_OK = 0,
  GFN1_E_IO = 1,                /* Gfn1Error::Io */
  GFN1_E_PARSE = 2,             /* Gfn1Error::Parse */
  GFN1_E_INVALID_INPUT = 3,     /* Gfn1Error::InvalidInput (also: overlap not positive definite) */
  GFN1_E_MISSING_ELEMENT = 4,   /* Gfn1Error::MissingElement */
  GFN1_E_MISSING_GLOBAL = 5,    /* Gfn1Error::MissingGlobal */
  GFN1_E_LINEAR_ALGEBRA = 6,    /* Gfn1Error::LinearAlgebra */
  GFN1_E_SINGULAR_CELL = 7,     /* Gfn1Error::SingularCell (periodic input is rejected) */
  GFN1_E_SCC_NOT_CONVERGED = 8, /* Gfn1Error::SccNotConverged */
  GFN1_E_DEVICE = 9,            /* CUDA error */
  GFN1_E_TIMEOUT = 10,          /* host-side wait exceeded */
  GFN1_E_NAN = 11,              /* non-finite input or result */
  GFN1_E_UNSUPPORTED = 12       /* element outside the device path (f shells, missing data) */
};

typedef struct gfn1_engine gfn1_engine;
typedef struct gfn1_batch gfn1_batch;
typedef struct gfn1_guess gfn1_guess;

/* Plain-path subset of ElectronicOptions (gfn1-rs src/electronic.rs:157-453,
 * defaults :395-452) plus the gradient switch of AnalyticGradientOptions
 * (src/gradient.rs:21-41). */
typedef struct gfn1_options {
  int32_t max_scc;               /* 250 */
  double energy_tolerance;       /* 1e-6 Eh */
  double charge_tolerance;       /* 2e-5 e */
  double mixing;                 /* 0.4 */
  int32_t scc_broyden;           /* 1 */
  int32_t scc_broyden_size;      /* 250 */
  double electronic_temperature; /* 300 K */
  int32_t enable_dispersion;     /* 1 */
  int32_t compute_gradient;      /* 1 */
  int32_t spin_multiplicity;     /* 0 = None; n >= 1: ElectronicOptions::spin_multiplicity
                                    (src/electronic.rs:159), spin-constrained occupations
                                    in restricted orbitals (src/electronic.rs:3930-4045) */
  double level_shift;            /* 0 Eh: ElectronicOptions::level_shift (src/electronic.rs:1413-1416,
                                    2125-2137), molecules of every size */
} gfn1_options;

/* Per-batch outputs; any pointer may be NULL.  For gfn1_batch_download the
 * pointers are host memory, for gfn1_batch_outputs_device they receive device
 * pointers owned by the batch. */
typedef struct gfn1_outputs {
  double* energy;         /* [nmol]   total_free (src/python.rs:2926) */
  double* terms;          /* [nmol*15] EnergyTerms::named_values order (src/electronic.rs:681-699) */
  double* gradient;       /* [natoms*3] dE/dR (src/gradient.rs:44-54) */
  double* shell_charges;  /* [nshells] Mulliken shell charges */
  double* atomic_charges; /* [natoms] */
  double* dipole;         /* [nmol*3] Mulliken dipole (src/field.rs:89-95) */
  double* fermi_level;    /* [nmol] */
  int32_t* iterations;    /* [nmol] */
  int32_t* status;        /* [nmol] per-molecule status code */
  int32_t* rung;          /* [nmol] rung of the fallback ladder (src/electronic.rs:1390-1447) whose SCC
                             converged: 0 = the requested scheme, 1 and 2 = linear mixing with a level
                             shift, 3 = T_el raised to max(T_el, 3000 K); -1 where status is not 0 */
} gfn1_outputs;

/* Fills the ElectronicOptions defaults. */
void gfn1_default_options(gfn1_options* opt);

/* Replaces Gfn1Parameters::resolve (gfn1-rs src/params.rs:206-227) plus the
 * engine state: param_spec is NULL/"builtin" (the bundled GFN1-xTB tables) or a
 * path to a tables file written by gen_tables.py.  device = CUDA ordinal. */
int gfn1_engine_create(const char* param_spec, int device, gfn1_engine** out);
void gfn1_engine_destroy(gfn1_engine* eng);

/* Thread-local message of the last failing call on this engine (never NULL). */
const char* gfn1_last_error(const gfn1_engine* eng);

/* Number of AOs and shells of a molecule; mirrors BasisSet::build
 * (src/basis.rs:121-233).  Returns GFN1_E_UNSUPPORTED for elements outside the
 * device path. */
int gfn1_basis_size(const gfn1_engine* eng, int nat, const uint8_t* z, int32_t* nao, int32_t* nshells);

/* One molecule, host buffers.  Replaces run_electronic (src/electronic.rs:800-804)
 * when opt->compute_gradient == 0 and analytic_gradient (src/gradient.rs:56-60)
 * otherwise.  `out` arrays are sized for this one molecule. */
int gfn1_run(gfn1_engine* eng, int nat, const uint8_t* z, const double* xyz_bohr, double charge,
             const double* init_shell_q, const gfn1_options* opt, const gfn1_outputs* out);

/* Batched energy + gradient of independent molecules, host buffers in and out
 * (host<->device copies inside).  atom_offsets has nmol+1 entries; charge and
 * init_shell_q (initial SCC shell charges, the hook of
 * ElectronicOptions::scc_initial_shell_charges, src/electronic.rs:386-392) may
 * be NULL.  Returns GFN1_OK when every molecule succeeded, otherwise the largest
 * per-molecule status (see out->status). */
int gfn1_batch_energy_gradient(gfn1_engine* eng, int nmol, const int32_t* atom_offsets, const uint8_t* z,
                               const double* xyz_bohr, const double* charge, const double* init_shell_q,
                               const gfn1_options* opt, const gfn1_outputs* out);

/* Matrices and orbitals of molecule m of the last gfn1_run /
 * gfn1_batch_energy_gradient call on this engine, the optional members of
 * ElectronicResult (src/electronic.rs:600-612): S = integrals.overlap, H0 = h0,
 * P = density, W = energy_weighted_density (N x N, row-major, AO order of
 * BasisSet::build) and orbital_energies / occupations (N).  P, W, the
 * eigenvalues and occupations are those of the last diagonalisation.  The
 * eigensolver solves only for the eigenvalues the occupations need (the
 * lowest ceil(nel/2)+8, the whole spectrum when the Fermi distribution
 * reaches further, and the highest); the others are NaN.  Any pointer may be
 * NULL. */
int gfn1_last_molecule_matrices(gfn1_engine* eng, int m, double* S, double* H0, double* P, double* W, double* eps,
                                double* occ);

/* Fock matrix, shell potential and coordination numbers of molecule m of the
 * last gfn1_run / gfn1_batch_energy_gradient call, the remaining optional
 * members of ElectronicResult (src/electronic.rs:600-620):
 *   F (N x N, row-major) = fock: H0 - 1/2 S_mu,nu (v_mu + v_nu) with v the AO
 *     potential of the input charges of the last diagonalisation
 *     (fock_from_shell_potential, src/electronic.rs:3133-3158).  On a rung of
 *     the fallback ladder with a level shift the reference's member also holds
 *     the shift projector b (S - 1/2 S P_prev S); F here does not;
 *   shell_potential (nshells) = shell_scc_potential: the potential of the
 *     final output shell charges (src/electronic.rs:1980, 2031);
 *   cn (natoms) = coordination_numbers (src/hamiltonian.rs:41, 87).
 * Any pointer may be NULL. */
int gfn1_last_molecule_fock(gfn1_engine* eng, int m, double* F, double* shell_potential, double* cn);

/* Resident-batch interface: the topology (atom counts, elements, charges) is
 * uploaded once; coordinates can then be replaced and the batch re-run with
 * inputs already on the device (molecular dynamics, benchmarking).
 * gfn1_batch_create validates the input and sizes the device workspace. */
int gfn1_batch_create(gfn1_engine* eng, int nmol, const int32_t* atom_offsets, const uint8_t* z,
                      const double* charge, const gfn1_options* opt, gfn1_batch** out);
void gfn1_batch_destroy(gfn1_batch* b);
/* Copies natoms*3 coordinates (bohr); `on_device` = 1 when xyz is a device pointer. */
int gfn1_batch_set_positions(gfn1_batch* b, const double* xyz, int on_device);
/* Initial shell charges (nshells values) or NULL for the zero guess. */
int gfn1_batch_set_initial_charges(gfn1_batch* b, const double* q, int on_device);
/* Enqueues setup, SCC and gradient kernels on `stream` (a cudaStream_t passed as
 * a void pointer; NULL = the engine's stream).  Asynchronous. */
int gfn1_batch_launch(gfn1_batch* b, void* stream);
/* Enqueues one stage: 0 = setup (CN, S, H0, Coulomb matrix, repulsion, D3),
 * 1 = persistent SCC, 2 = gradient; -1 = all three (same as gfn1_batch_launch).
 * Lets a caller time each kernel with events on its own stream. */
int gfn1_batch_launch_stage(gfn1_batch* b, int stage, void* stream);
/* Per-stage SCC clock totals (GFN1_PROFILE=1 at batch creation), n <= 13:
 * prologue (H0' and the SCC state), Fock, tridiagonalisation, eigenvalues,
 * occupations, inverse iteration, back-transformation, populations, energy,
 * mixing, final, Cholesky, L^-1. */
int gfn1_batch_stage_cycles(const gfn1_batch* b, uint64_t* cycles, int n);
/* Bytes of the input blob (one host->device copy per call) and of the output
 * blob (one device->host copy per call). */
int gfn1_batch_io_bytes(const gfn1_batch* b, int64_t* h2d, int64_t* d2h);
/* Plan of the large-molecule path (molecules above 256 AOs) in the last
 * gfn1_batch_energy_gradient / gfn1_run call on this engine: the Householder
 * reduction's panel width, its minimum rows per CTA, the CTAs per molecule,
 * the reduction time the autotuner measured for that plan (ms) and whether the
 * autotuner chose it (1) or GFN1_WIDE_PANEL fixed it (0).  All zero when that
 * call had no large molecule.  No counterpart in the reference (faer chooses
 * its own blocking inside self_adjoint_eigen, src/linalg.rs:176). */
int gfn1_last_wide_plan(gfn1_engine* eng, int32_t* panel, int32_t* min_rows, int32_t* ctas_per_molecule,
                        double* reduction_ms, int32_t* tuned);
/* Synchronises and copies results to host buffers. */
int gfn1_batch_download(gfn1_batch* b, const gfn1_outputs* out);
/* As gfn1_last_molecule_matrices for molecule m of a resident batch after its
 * last launch (waits for the device first). */
int gfn1_batch_molecule_matrices(gfn1_batch* b, int m, double* S, double* H0, double* P, double* W, double* eps,
                                 double* occ);
/* As gfn1_last_molecule_fock for molecule m of a resident batch after its last
 * launch (waits for the device first). */
int gfn1_batch_molecule_fock(gfn1_batch* b, int m, double* F, double* shell_potential, double* cn);
/* Device pointers of the batch-owned result arrays (valid until destroy);
 * there `rung` is meaningful where `status` is 0. */
int gfn1_batch_outputs_device(gfn1_batch* b, gfn1_outputs* out);
/* Sizes of the batch: natoms, nshells, total AOs; launches = kernels per run. */
int gfn1_batch_info(const gfn1_batch* b, int64_t* natoms, int64_t* nshells, int64_t* naos, int32_t* launches);

/* One molecule without allocating anything (no reference counterpart: the Rust
 * library has no device memory).  For callers that cannot call cudaMalloc or
 * cudaHostAlloc at the point of use -- code running under a memory manager that
 * owns all device memory, real-time loops that forbid allocation, or a step
 * that must not change the process's memory footprint.  All device scratch is a
 * fixed 4.25 MiB library array that every GPU loading the library holds until
 * exit; host staging uses the stack.  Limits: at most 64 atoms, 128 AOs,
 * 128 shells and 250 Broyden history vectors (min(scc_broyden_size, max_scc));
 * larger inputs return GFN1_E_INVALID_INPUT with a message naming the limit.
 * Only rung 0 of the fallback ladder runs here: a molecule that needs the
 * later rungs returns GFN1_E_SCC_NOT_CONVERGED.  Like gfn1_run, the SCC starts
 * from init_shell_q when given, else from the engine's learned guess when one
 * is set (gfn1_engine_set_guess), else from zero charges.  The caller's
 * current device is the same on return.
 * The first call on a device looks up the array's device address (once per
 * device, that device current); make that first call before any stream
 * capture.  Every call reuses the same array, so calls that overlap on the GPU
 * (two host threads, or asynchronous streams) race: serialise them.  Inputs
 * and `out` are host memory; `stream` is a cudaStream_t or NULL for the
 * engine's stream.  Synchronous. */
int gfn1_run_noalloc(gfn1_engine* eng, int nat, const uint8_t* z, const double* xyz_bohr, double charge,
                     const double* init_shell_q, const gfn1_options* opt, const gfn1_outputs* out, void* stream);

/* ---- Geometry optimisation on the device: the reference's
 * optimize_geometry (gfn1-rs src/optimizer.rs:78-320: L-BFGS with history,
 * Armijo backtracking, per-atom step cap, convergence on the largest gradient
 * component or the step norm) for every molecule of a resident batch at once.
 * Options mirror GeometryOptimizationOptions (src/optimizer.rs:17-50). */
typedef struct gfn1_opt_options {
  int32_t max_iterations;     /* 250 */
  double gradient_tolerance;  /* 1e-4 Eh/bohr (largest component) */
  double step_tolerance;      /* 1e-7 bohr */
  int32_t history;            /* 12 (at most 12) */
  double initial_step;        /* 1.0 */
  double max_atom_step;       /* 0.30 bohr */
  int32_t max_rounds;         /* bound on engine passes, 100000 */
} gfn1_opt_options;

void gfn1_default_opt_options(gfn1_opt_options* o);
/* Optimises every molecule of a resident batch from its current positions
 * (gfn1_batch_set_positions; the batch must compute gradients).  Each round
 * evaluates all pending trial geometries in one engine pass on the engine's
 * stream; the L-BFGS state stays on the device and every trial's SCC starts
 * from the converged charges of the molecule's current geometry.  Outputs
 * (host, any may be NULL): final coordinates [natoms*3] (also left in the
 * batch's positions), energies and largest gradient components [nmol]
 * (NaN where status is not 0), accepted steps, converged flags and statuses
 * [nmol] (GFN1_E_INVALID_INPUT where the line search found no downhill step,
 * as the reference's error), and the number of engine passes.  Synchronous. */
int gfn1_batch_optimize(gfn1_batch* b, const gfn1_opt_options* opt, double* xyz_out, double* energy,
                        double* max_gradient, int32_t* iterations, int32_t* converged, int32_t* status,
                        int32_t* rounds);

/* ---- Learned SCC initial guess.  No counterpart in the reference, whose SCC
 * starts from zero shell charges or a caller-supplied vector (the Rust
 * `init_shell_q` hook, gfn1-rs src/electronic.rs:1231-1239); the guess fills
 * that vector on the device.  Per H/C/N/O atom: 64 radial + 32 angular
 * descriptors (cutoff 6 bohr) and the element one-hot feed three SiLU layers
 * of 128 and a linear layer to the atom's two shell charges; each molecule's
 * charges are shifted to sum to its total charge.  Molecules with other
 * elements get the zero guess.  Inference runs with BF16 weights and
 * activations (FP32 accumulation); the converged SCC always decides the result.
 *
 * Parameters (float32, gfn1_guess_param_count() values): feature mean[96],
 * feature scale[96], W1[100x128], b1[128], W2[128x128], b2[128],
 * W3[128x128], b3[128], W4[128x2], b4[2], weights row-major [in][out]. */
int64_t gfn1_guess_param_count(void);
int gfn1_guess_create(gfn1_engine* eng, const float* params, int64_t nparams, gfn1_guess** out);
void gfn1_guess_destroy(gfn1_guess* g);
/* Default guess of batches prepared from now on (NULL restores the zero guess).
 * The guess must outlive its use by the engine. */
int gfn1_engine_set_guess(gfn1_engine* eng, gfn1_guess* g);
/* Guess of a resident batch; used by launches while no initial charges are set. */
int gfn1_batch_set_guess(gfn1_batch* b, gfn1_guess* g);
/* Device-pointer entry points (stream = cudaStream_t or NULL):
 * features x[natoms x 100] (raw descriptors and one-hot when mean/scale are
 * NULL), inference y[natoms x 2] = MLP(x), and the whole prediction into
 * init_q[nshells] in the engine's shell layout (x, y are caller scratch). */
int gfn1_guess_features_device(int nmol, const int32_t* atom_off, const int32_t* z, const double* xyz,
                               const float* mean, const float* scale, float* x, void* stream);
int gfn1_guess_infer_device(gfn1_guess* g, int64_t natoms, const float* x, float* y, void* stream);
int gfn1_guess_predict_device(gfn1_guess* g, int nmol, const int32_t* atom_off, const int32_t* shell_off,
                              const int32_t* z, const double* xyz, const double* charge, float* x_scratch,
                              float* y_scratch, double* init_q, void* stream);

/* ---- Training primitives of the guess network (FP32, device pointers,
 * asynchronous on `stream`).  No reference counterpart.
 * gfn1_mlp_gemm: C[MxN] = op(A)[MxK] op(B)[KxN], op(A)(m,k) = ta ? A[k*lda+m] :
 * A[m*lda+k], op(B)(k,n) = tb ? B[n*ldb+k] : B[k*ldb+n], with epilogue
 *   0: partial sums of K-split z into C + z*M*ldc (ksplit >= 1; see
 *      gfn1_mlp_gemm_splits for the number of slices written),
 *   1: Z = acc + bias[n], C = SiLU(Z),   2: C = acc + bias[n],
 *   3: C = acc * SiLU'(zprev[m*ldz+n]).
 * Supported (ta, tb, epi): (0,0,1) (0,0,2) (0,1,3) (0,1,0) (1,0,0) (0,0,0). */
int gfn1_mlp_gemm(int ta, int tb, int epi, int M, int N, int K, const float* A, int lda, const float* B, int ldb,
                  const float* bias, const float* zprev, int ldz, float* C, float* Z, int ldc, int ksplit,
                  void* stream);
int gfn1_mlp_gemm_splits(int K, int ksplit);
/* out[i] = sum_z part[z*stride + i], z = 0..nz-1 in order. */
int gfn1_mlp_reduce(int nz, int64_t stride, const float* part, float* out, int64_t n, void* stream);
/* part[c*N + n] = sum of Y[m*ldy + n] over rows m of chunk c (ceil(M/mchunk) chunks). */
int gfn1_mlp_colsum(int M, int N, const float* Y, int ldy, int mchunk, float* part, void* stream);
/* Per molecule (2 shells per atom): q = y + (charge - sum y)/nshells; with a
 * label, loss_mol[m] = sum (q - label)^2 * inv_nsh and gy = d loss / d y. */
int gfn1_mlp_project_loss(int nmol, const int32_t* atom_off, const float* y, const double* charge,
                          const float* label, double inv_nsh, float* gy, float* q, double* loss_mol, void* stream);
/* Adam step: m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2,
 * p -= lr (m c1) / (sqrt(v c2) + eps), c1 = 1/(1-b1^t), c2 = 1/(1-b2^t). */
int gfn1_mlp_adam(int64_t n, float* p, const float* g, float* m, float* v, float lr, float beta1, float beta2,
                  float eps, float c1, float c2, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GFN1_B200_H */
