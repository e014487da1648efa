// Device state of the batched geometry optimiser (optimize.cu), shared with
// the host driver in capi.cu.
#pragma once

#include "common.cuh"

namespace gfn1 {

constexpr int kOptNT = 128;
constexpr int kOptHist = 12;  // GeometryOptimizationOptions::history default (the host sets H <= kOptHist)

// States of a molecule.
enum OptPhase : int { kOptNeedStep = 0, kOptTrial = 1, kOptDone = 2 };

struct OptMol {
  double energy, alpha, dd, maxg, step_norm;
  double rho[kOptHist];
  int phase, tries, iterations, count, head, converged, error;
  int pad;
};

struct OptParams {
  int max_iterations, history;
  double gradient_tolerance, step_tolerance, initial_step, max_atom_step;
};

// Device arrays of a batch optimisation (natoms*3 coordinates per vector).
struct OptArrays {
  OptMol* mol;       // [nmol]
  double* x;         // [3 natoms] current geometries
  double* g;         // [3 natoms] current gradients
  double* d;         // [3 natoms] search directions
  double* S;         // [H][3 natoms] history of steps s
  double* Y;         // [H][3 natoms] history of gradient changes y
  double* q;         // [nshells] converged shell charges of the current geometries
  double* x_in;      // [3 natoms] batch coordinates (trial geometries are written here)
  double* q_in;      // [nshells] batch initial shell charges
  int* skip;         // [nmol] 1: the engine skips the molecule this round
  int* active;       // [1] molecules still optimising (counted by the round kernel)
  long long n3;      // 3 natoms
};

size_t opt_mol_bytes();
cudaError_t launch_opt_round(const Batch& B, const OptArrays& A, const OptParams& P, int nmol, int init,
                             cudaStream_t st);
cudaError_t launch_opt_skip(int nmol, const int* skip, int* status, cudaStream_t st);
cudaError_t launch_opt_final(const Batch& B, const OptArrays& A, int nmol, cudaStream_t st);

}  // namespace gfn1
