// Batched geometry optimisation on the device: gfn1-rs `optimize_geometry`
// (src/optimizer.rs:78-320) for every molecule of a resident batch at once.
//
// Per round the host launches the engine (setup, SCC, gradient) on the trial
// geometries, then opt_round_kernel, which for each molecule (one CTA):
//   * takes the trial's energy and gradient, applies the Armijo test
//     E_trial <= E + 1e-4 alpha g.d (src/optimizer.rs:238-244); on success it
//     pushes (s, y) into the L-BFGS history when y.s > 1e-12
//     (src/optimizer.rs:172-186), moves to the trial, and tests convergence
//     (largest gradient component <= gradient_tolerance or step norm <=
//     step_tolerance, src/optimizer.rs:197-198); otherwise it halves alpha, at
//     most 24 trials (src/optimizer.rs:221-257);
//   * for a molecule that needs a new step: the two-loop L-BFGS direction with
//     gamma = y.s / y.y (src/optimizer.rs:259-290), steepest descent when that
//     direction is not downhill or not finite, the per-atom step cap
//     (src/optimizer.rs:292-305) and alpha = initial_step;
//   * writes the next trial geometry into the batch's coordinates and the
//     converged shell charges of the current geometry into its initial
//     charges (the SCC of every trial starts from them), or marks the molecule
//     finished so that the engine kernels skip it.
// The only host round trip per round is the count of molecules still
// optimising.  Everything else (history, geometries, gradients, charges) stays
// in device memory between rounds.
#include <cuda_runtime.h>
#include <float.h>

#include "common.cuh"
#include "optimize.cuh"

namespace gfn1 {

__device__ __forceinline__ double opt_block_sum(double v, double* red) { return block_sum(v, red); }

// Two-loop recursion over the ring buffer (oldest first at head).
__device__ void lbfgs_direction_dev(const OptArrays& A, const OptMol& mm, int o3, int n, int H, double* q,
                                    const double* g, double* red, double* alph) {
  const int tid = threadIdx.x;
  for (int i = tid; i < n; i += kOptNT) q[i] = g[i];
  __syncthreads();
  const int cnt = mm.count;
  if (cnt == 0) {
    for (int i = tid; i < n; i += kOptNT) q[i] = -q[i];
    __syncthreads();
    return;
  }
  auto slot = [&](int k) { return (mm.head + k) % H; };  // k = 0 oldest .. cnt-1 newest
  for (int k = cnt - 1; k >= 0; --k) {
    const double* s = A.S + (long long)slot(k) * A.n3 + o3;
    const double* y = A.Y + (long long)slot(k) * A.n3 + o3;
    double p = 0.0;
    for (int i = tid; i < n; i += kOptNT) p += s[i] * q[i];
    const double a = mm.rho[slot(k)] * opt_block_sum(p, red);
    if (tid == 0) alph[k] = a;
    for (int i = tid; i < n; i += kOptNT) q[i] -= a * y[i];
    __syncthreads();
  }
  {
    const double* s = A.S + (long long)slot(cnt - 1) * A.n3 + o3;
    const double* y = A.Y + (long long)slot(cnt - 1) * A.n3 + o3;
    double pyy = 0.0, pys = 0.0;
    for (int i = tid; i < n; i += kOptNT) {
      pyy += y[i] * y[i];
      pys += y[i] * s[i];
    }
    const double yy = opt_block_sum(pyy, red);
    const double ys = opt_block_sum(pys, red);
    const double gamma = yy > 1e-18 ? ys / yy : 1.0;
    for (int i = tid; i < n; i += kOptNT) q[i] *= gamma;
    __syncthreads();
  }
  for (int k = 0; k < cnt; ++k) {
    const double* s = A.S + (long long)slot(k) * A.n3 + o3;
    const double* y = A.Y + (long long)slot(k) * A.n3 + o3;
    double p = 0.0;
    for (int i = tid; i < n; i += kOptNT) p += y[i] * q[i];
    const double beta = mm.rho[slot(k)] * opt_block_sum(p, red);
    const double c = alph[k] - beta;
    for (int i = tid; i < n; i += kOptNT) q[i] += c * s[i];
    __syncthreads();
  }
  for (int i = tid; i < n; i += kOptNT) q[i] = -q[i];
  __syncthreads();
}

// init = 1: the batch holds the evaluation of the starting geometries.
__global__ void __launch_bounds__(kOptNT) opt_round_kernel(Batch B, OptArrays A, OptParams P, int init) {
  __shared__ double red[kOptNT / 32];
  __shared__ double alph[kOptHist];
  __shared__ int flag;
  const int m = blockIdx.x, tid = threadIdx.x;
  OptMol& mm = A.mol[m];
  const int a0 = B.atom_off[m], nat = B.atom_off[m + 1] - a0;
  const int sh0 = B.shell_off[m], nsh = B.shell_off[m + 1] - sh0;
  const int o3 = 3 * a0, n = 3 * nat;
  const int H = P.history;
  double* x = A.x + o3;
  double* g = A.g + o3;
  double* d = A.d + o3;
  const double* gt = B.grad + o3;
  double* xt = A.x_in + o3;
  if (init) {
    if (tid == 0) {
      mm.phase = kOptDone;
      mm.tries = mm.iterations = mm.count = mm.head = mm.converged = 0;
      mm.error = B.status[m];
    }
    __syncthreads();
    if (B.status[m] == kOk) {
      double mx = 0.0;
      for (int i = tid; i < n; i += kOptNT) {
        x[i] = xt[i];
        g[i] = gt[i];
        mx = fmax(mx, fabs(gt[i]));
      }
      for (int s = tid; s < nsh; s += kOptNT) A.q[sh0 + s] = B.shell_q[sh0 + s];
      mx = block_max(mx, red);
      if (tid == 0) {
        mm.energy = B.terms[(long long)m * kTerms];
        mm.maxg = mx;
        mm.step_norm = 0.0;
        mm.converged = mx <= P.gradient_tolerance;
        mm.phase = mm.converged ? kOptDone : kOptNeedStep;
      }
    }
    __syncthreads();
  } else if (mm.phase == kOptTrial) {
    // ---- the trial's evaluation: Armijo test
    if (tid == 0) {
      const double et = B.terms[(long long)m * kTerms];
      flag = (B.status[m] == kOk && et <= mm.energy + 1.0e-4 * mm.alpha * mm.dd) ? 1 : 0;
    }
    __syncthreads();
    if (flag) {
      double pys = 0.0, pss = 0.0, mx = 0.0;
      int bad = 0;
      for (int i = tid; i < n; i += kOptNT) {
        const double s = xt[i] - x[i], y = gt[i] - g[i];
        pys += y * s;
        pss += s * s;
        mx = fmax(mx, fabs(gt[i]));
        if (!isfinite(s) || !isfinite(y)) bad = 1;
      }
      const double ys = block_sum(pys, red);
      const double ss = block_sum(pss, red);
      mx = block_max(mx, red);
      bad = block_max((double)bad, red) > 0.0;
      const int H0 = mm.count, hd = mm.head;
      const bool push = ys > 1.0e-12 && !bad;
      const int slot = H0 < H ? (hd + H0) % H : hd;  // full: overwrite the oldest
      if (push) {
        double* S = A.S + (long long)slot * A.n3 + o3;
        double* Y = A.Y + (long long)slot * A.n3 + o3;
        for (int i = tid; i < n; i += kOptNT) {
          S[i] = xt[i] - x[i];
          Y[i] = gt[i] - g[i];
        }
      }
      __syncthreads();
      for (int i = tid; i < n; i += kOptNT) {
        x[i] = xt[i];
        g[i] = gt[i];
      }
      for (int s = tid; s < nsh; s += kOptNT) A.q[sh0 + s] = B.shell_q[sh0 + s];
      if (tid == 0) {
        if (push) {
          mm.rho[slot] = 1.0 / ys;
          if (H0 < H) mm.count = H0 + 1;
          else mm.head = (hd + 1) % H;
        }
        mm.energy = B.terms[(long long)m * kTerms];
        mm.maxg = mx;
        mm.step_norm = sqrt(ss);
        mm.converged = mx <= P.gradient_tolerance || mm.step_norm <= P.step_tolerance;
        mm.phase = mm.converged ? kOptDone : kOptNeedStep;
      }
      __syncthreads();
    } else if (tid == 0) {
      mm.alpha *= 0.5;
      mm.tries += 1;
      if (mm.tries >= 24) {
        mm.phase = kOptDone;
        mm.error = B.status[m] != kOk ? B.status[m] : kErrInvalidInput;  // no downhill step
      }
    }
    __syncthreads();
  }
  // ---- a new step
  if (mm.phase == kOptNeedStep) {
    if (mm.iterations >= P.max_iterations) {
      if (tid == 0) mm.phase = kOptDone;
      __syncthreads();
    } else {
      lbfgs_direction_dev(A, mm, o3, n, H, d, g, red, alph);
      double pdg = 0.0;
      int bad = 0;
      for (int i = tid; i < n; i += kOptNT) {
        pdg += d[i] * g[i];
        if (!isfinite(d[i])) bad = 1;
      }
      const double dg = block_sum(pdg, red);
      bad = block_max((double)bad, red) > 0.0;
      if (dg >= 0.0 || bad) {
        for (int i = tid; i < n; i += kOptNT) d[i] = -g[i];
        __syncthreads();
      }
      double amax = 0.0;  // per-atom step cap
      for (int a = tid; a < nat; a += kOptNT)
        amax = fmax(amax, sqrt(d[3 * a] * d[3 * a] + d[3 * a + 1] * d[3 * a + 1] + d[3 * a + 2] * d[3 * a + 2]));
      amax = block_max(amax, red);
      if (P.max_atom_step > 0.0 && amax > P.max_atom_step) {
        const double sc = P.max_atom_step / amax;
        for (int i = tid; i < n; i += kOptNT) d[i] *= sc;
        __syncthreads();
      }
      double pdd = 0.0;
      for (int i = tid; i < n; i += kOptNT) pdd += g[i] * d[i];
      const double dd = block_sum(pdd, red);
      if (tid == 0) {
        mm.iterations += 1;
        mm.dd = dd;
        mm.alpha = fmax(P.initial_step, 1.0e-8);
        mm.tries = 0;
        mm.phase = kOptTrial;
      }
      __syncthreads();
    }
  }
  // ---- the next trial, or skip
  if (mm.phase == kOptTrial) {
    const double al = mm.alpha;
    for (int i = tid; i < n; i += kOptNT) xt[i] = x[i] + al * d[i];
    for (int s = tid; s < nsh; s += kOptNT) A.q_in[sh0 + s] = A.q[sh0 + s];
    if (tid == 0) {
      A.skip[m] = 0;
      atomicAdd(A.active, 1);
    }
  } else if (tid == 0) {
    A.skip[m] = 1;
  }
}

// Molecules marked in `skip` get a status the engine kernels skip.
__global__ void opt_apply_skip_kernel(int nmol, const int* skip, int* status) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < nmol && skip[m] && status[m] == kOk) status[m] = kOptSkipped;
}

// Final geometries into the batch coordinates (for the caller's last look).
__global__ void opt_final_kernel(Batch B, OptArrays A, int nmol) {
  const long long n3 = A.n3;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
    A.x_in[i] = A.x[i];
}

size_t opt_mol_bytes() { return sizeof(OptMol); }

cudaError_t launch_opt_round(const Batch& B, const OptArrays& A, const OptParams& P, int nmol, int init,
                             cudaStream_t st) {
  opt_round_kernel<<<nmol, kOptNT, 0, st>>>(B, A, P, init);
  return cudaGetLastError();
}

cudaError_t launch_opt_skip(int nmol, const int* skip, int* status, cudaStream_t st) {
  opt_apply_skip_kernel<<<(nmol + 255) / 256, 256, 0, st>>>(nmol, skip, status);
  return cudaGetLastError();
}

cudaError_t launch_opt_final(const Batch& B, const OptArrays& A, int nmol, cudaStream_t st) {
  opt_final_kernel<<<256, 256, 0, st>>>(B, A, nmol);
  return cudaGetLastError();
}

}  // namespace gfn1
