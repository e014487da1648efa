// Learned SCC initial guess: atom-centred descriptors and a small MLP that
// predicts the two shell charges of each H/C/N/O atom.  The reference has no
// counterpart; its SCC starts from zero shell charges or a caller-supplied
// vector (src/electronic.rs:1231-1239).  Kernels live in guess.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gfn1 {

constexpr int kGuessDesc = 96;   // 64 radial + 32 angular descriptors
constexpr int kGuessIn = 100;    // descriptors + element one-hot (H, C, N, O)
constexpr int kGuessHid = 128;   // three SiLU layers
constexpr int kGuessOut = 2;     // shell charges per atom
constexpr double kGuessCutoff = 6.0;  // bohr
// Packed parameter vector: mean[96], std[96], W1[100x128], b1, W2[128x128], b2,
// W3[128x128], b3, W4[128x2], b4 (weights row-major [in][out]).
constexpr long long kGuessParams = 2LL * kGuessDesc + (long long)kGuessIn * kGuessHid + kGuessHid +
                                   2LL * ((long long)kGuessHid * kGuessHid + kGuessHid) +
                                   (long long)kGuessHid * kGuessOut + kGuessOut;

// Device copy of a trained model: FP32 master parameters plus BF16 copies of
// the weight matrices used by the inference kernel.
struct GuessModel {
  float* params;     // [kGuessParams] device
  uint16_t* wbf16;   // W1 | W2 | W3 | W4 as bfloat16 bit patterns
};

// x[natoms][100]: normalised descriptors and one-hot, or the raw descriptors
// when mean/std are null.  Rows of atoms outside H/C/N/O are zero.
cudaError_t launch_guess_features(int nmol, const int* atom_off, const int* z, const double* xyz, const float* mean,
                                  const float* stdv, float* x, cudaStream_t st);
// y[natoms][2] = MLP(x) with BF16 weights and activations, FP32 accumulation.
cudaError_t launch_guess_infer(const GuessModel& g, long long natoms, const float* x, float* y, cudaStream_t st);
// init_q[shell_off[m] + 2 (a - a0) + s] = y shifted to the molecule's charge;
// zeros for molecules with atoms outside H/C/N/O.
cudaError_t launch_guess_project(int nmol, const int* atom_off, const int* shell_off, const int* z, const float* y,
                                 const double* charge, double* init_q, cudaStream_t st);
cudaError_t guess_model_upload(const float* host_params, GuessModel& g);
void guess_model_free(GuessModel& g);
size_t guess_infer_smem_bytes();

}  // namespace gfn1
