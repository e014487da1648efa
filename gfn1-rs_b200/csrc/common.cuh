// Shared definitions of the B200 GFN1-xTB engine: element tables, the batch
// descriptor the kernels read, status codes and small device helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gfn1 {

// Status codes (same numbering as include/gfn1_b200.h).  1..8 mirror the
// reference's Gfn1Error variants (src/error.rs:8-17).
enum Status : int {
  kOk = 0,
  kErrIo = 1,
  kErrParse = 2,
  kErrInvalidInput = 3,
  kErrMissingElement = 4,
  kErrMissingGlobal = 5,
  kErrLinearAlgebra = 6,
  kErrSingularCell = 7,
  kErrSccNotConverged = 8,
  kErrDevice = 9,
  kErrTimeout = 10,
  kErrNan = 11,
  kErrUnsupported = 12,
  kOptSkipped = 13,  // internal: a molecule the geometry optimiser has finished (the engine kernels skip it)
};

constexpr int kMaxZ = 86;
constexpr int kNZ = kMaxZ + 1;
constexpr int kMaxShAtom = 3;  // shells per atom on the device path
constexpr int kMaxPrim = 8;    // H 2s after orthogonalisation to 1s has 7
constexpr int kMaxRef = 5;     // D3 references per element for Z <= 86
constexpr int kTerms = 15;     // EnergyTerms::named_values (src/electronic.rs:681-699)
// Gradient kernel: threads per CTA (one CTA per molecule) and the CTAs per SM
// its register budget is sized for.
constexpr int kGradThreads = 128;
constexpr int kGradMinBlocks = 4;
// The s/p instantiation of the gradient kernel runs five CTAs per SM (96
// registers; measured on the 4096-molecule batch: 3 CTAs 7.70 ms, 4: 7.00 ms,
// 5: 6.63 ms, the spills staying in L1)
constexpr int kGradMinBlocksSp = 5;

// Per-element data, indexed by Z.  nsh == 0 marks an element the device path
// does not support (f shells, more than three shells).  Values are already converted to the model
// units (Hartree, bohr) with the reference's conventions.
struct ElemTable {
  int nsh, nao;
  int l[kMaxShAtom], nprim[kMaxShAtom], valence[kMaxShAtom], ao_first[kMaxShAtom];
  double alpha[kMaxShAtom][kMaxPrim], coef[kMaxShAtom][kMaxPrim];
  double hdiag[kMaxShAtom];   // level (Eh)
  double kcn[kMaxShAtom];     // CN shift of the self energy (Eh)
  double poly[kMaxShAtom];    // shell polynomial coefficient (x0.01)
  double refocc[kMaxShAtom];  // reference occupation of the shell
  double hard[kMaxShAtom];    // shell hardness
  double gam3, repa, repb, en, rad, rcov, r4r2;
  double xb;                  // halogen-bond strength 0.1 CXB (0 without an entry)
  int d3_nref;
  double d3_cnref[kMaxRef];
};

// Model-wide constants copied from the parameter file.
struct Globals {
  double ks, kp, kd, ksp, kdiff, enscale, kexp, kexplight;
  double a1, a2, s6, s8;
  double xbdamp, xbrad;  // halogen-bond damping and radius scaling
};

// SCC options (plain-path subset of ElectronicOptions, src/electronic.rs:157-453).
struct SccOptions {
  int max_scc;
  int broyden;       // 1 = Broyden, 0 = linear damping
  int broyden_size;  // memory
  int enable_dispersion;
  int spin_mult;     // 0: no spin multiplicity; n >= 1: spin-constrained occupations
  double energy_tol, charge_tol, mixing, etemp;
  double level_shift;  // requested virtual level shift (Eh), 0 = none
};

// Parameters of one launch of the persistent SCC kernel (one size class).
struct SccLaunch {
  int q_begin, q_end;   // range of Batch::order processed by this launch
  int* counter;         // work counter, zeroed before the launch
  double* ws;           // per-CTA global workspace, ws_stride doubles each
  long long ws_stride;
  int maxn, maxnsh, maxnat, cap;  // maxima of the class (workspace layout)
  int smem_bytes;       // dynamic shared memory of the launch
};

// Everything a kernel needs about a batch of molecules.  All pointers are
// device pointers; offsets index the flat per-batch arrays.
struct Batch {
  int nmol;
  int max_nat;
  const int* atom_off;      // [nmol+1]
  const int* shell_off;     // [nmol+1]
  const int* ao_off;        // [nmol+1]
  const long long* mat_off; // [nmol+1] offsets (doubles) of the N x N matrices
  const long long* gam_off; // [nmol+1] offsets of the nsh x nsh Coulomb matrices
  const long long* pair_off;// [nmol+1] offsets of the nat(nat-1)/2 atom-pair scratch
  const int* order;         // [nmol] processing order (most expensive first)
  const int* z;             // [natoms]
  const double* xyz;        // [natoms*3] bohr
  const double* charge;     // [nmol]
  const double* init_q;     // [nshells] or null: initial shell charges
  // per-molecule N x N matrices (offset mat_off[m])
  double *S, *H0, *P, *W;
  // per-CTA workspace of the persistent SCC kernel, ws_stride doubles per CTA
  double* ws;
  long long ws_stride;
  int ws_maxn, ws_maxnsh, ws_cap;
  double* gam;              // Coulomb matrices (offset gam_off[m])
  double* pairbuf;          // gradient pair scratch (8 per atom pair)
  // per-atom / per-shell state
  double *cn, *cn_disp_dedcn; // [natoms]
  double *shell_q, *shell_pot, *atom_q; // [nshells], [nshells], [natoms]
  double* shell_pot_in;     // [nshells] potential of the last diagonalised Fock matrix, or null
  double* se;               // [nshells] self energies
  // outputs
  double* terms;            // [nmol*kTerms]
  double* grad;             // [natoms*3]
  double* grad_classic;     // [natoms*3] repulsion + dispersion gradient
  double* dipole;           // [nmol*3]
  double* fermi;            // [nmol]
  int* iterations;          // [nmol]
  int* status;              // [nmol]
  int* rung;                // [nmol] fallback-ladder rung whose SCC converged (-1: none), or null
  double* orb_eps;          // [naos] orbital energies of the last diagonalisation (offset ao_off[m]), or null
  double* orb_occ;          // [naos] their occupations, or null
  int* queue;               // work counters: [0], [1] size classes, [2] fallback ladder, [3] failed count
  int* failed;              // [nmol] molecules whose first SCC attempt did not converge, or null
  unsigned long long* stage_cycles;  // [kStages] per-stage clock totals, or null
};

// Threads of the persistent SCC kernel resident per SM: 128-thread CTAs run
// kSccThreadsPerSm / 128 to an SM (the register budget per thread follows).
#ifndef GFN1_SCC_THREADS_PER_SM
#define GFN1_SCC_THREADS_PER_SM 512
#endif
constexpr int kSccThreadsPerSm = GFN1_SCC_THREADS_PER_SM;

// SCC stages timed when Batch::stage_cycles is set (the device counterpart of
// the reference's GFN1_PROFILE scopes, src/electronic.rs:1448, :2089-2157).
enum Stage : int {
  kStPrologue = 0,  // H0' and the SCC state (Cholesky and L^-1: kStChol, kStLinv)
  kStFock,          // shell potential + F'
  kStTridiag,       // Householder reduction
  kStEigval,        // bisection
  kStFermi,         // occupations
  kStInvIter,       // inverse iteration
  kStBackTr,        // back-transformation
  kStPop,           // C, D, Mulliken populations
  kStEnergy,        // output charges, energies, convergence test
  kStMix,           // Broyden / damped mixing
  kStFinal,         // P, W and results
  kStChol,          // Cholesky S = L L^T
  kStLinv,          // L^-1
  kStages
};

__host__ __device__ inline int tri_index(int a, int b, int nat) {
  // index of the unordered pair a < b among nat(nat-1)/2
  return a * nat - a * (a + 1) / 2 + (b - a - 1);
}

#ifdef __CUDACC__
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// Block-wide sum; every thread gets the result.  `red` needs blockDim/32 doubles.
__device__ __forceinline__ double block_sum(double v, double* red) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < nw; ++i) s += red[i];
  return s;
}
__device__ __forceinline__ double block_max(double v, double* red) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = red[0];
  for (int i = 1; i < nw; ++i) s = fmax(s, red[i]);
  return s;
}
#endif

}  // namespace gfn1
