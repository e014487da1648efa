// Analytic nuclear gradient of the converged SCC (gfn1-rs src/gradient.rs:122-531,
// stock terms only).  One CTA per molecule.
//
// Phase 1, one thread per unordered atom pair (a < b):
//   * inside the 30 bohr integral cutoff, for every shell pair and AO pair the
//     overlap derivative dS/dR is contracted with
//       coeff = P (2 h_ij - v_mu - v_nu) - 2 W
//     plus the H0 polynomial term 2 P h_ij S dlnPi/dR and the dE/dCN accumulation
//     (src/gradient.rs:358-455);
//   * the Coulomb term q_i q_j d gamma_ij / dR over the shells of the two atoms
//     (src/gradient.rs:493-516, no cutoff).
//   Each pair writes its contributions to a scratch slot.
// Phase 2, one thread per atom: fixed-order sum over the atom's pairs plus the
//   diagonal CN term dsedcn * P_mu,mu (src/gradient.rs:464-469).
// Phase 3, one thread per atom: the CN chain (dE/dCN_i + dE/dCN_j) dCN/dr
//   (src/gradient.rs:470-490), then repulsion + dispersion from the setup kernel.
// Fixed-order reductions make the gradient bitwise reproducible.
#include "common.cuh"
#include "model.cuh"
#include "overlap.cuh"

namespace gfn1 {

// Overlap-derivative contraction of one shell pair (mu shell of angular
// momentum LB on atom b, nu shell LA on atom a), src/gradient.rs:358-455:
// gmu += dS/dR_b [P (2 h - v_mu - v_nu) - 2 W] + R 2 P h S dlnPi/dR, plus the
// dE/dCN accumulation of both atoms.  xs = {h, v_mu + v_nu, dlnPi/dR factor,
// -kcn_mu hscale Pi, -kcn_nu hscale Pi}.
template <int LB, int LA>
__device__ __forceinline__ void grad_shell_pair(const ElemTable& eb, int kb, const double* xb, const ElemTable& ea,
                                                int ka, const double* xa, const double* P, const double* W, int N,
                                                int mu0, int nu0, const double (&xs)[5], const double (&rv)[3],
                                                double (&gmu)[3], double& dcmu, double& dcnu) {
  double Sb[2 * LB + 1][2 * LA + 1], dA[2 * LB + 1][2 * LA + 1][3];
  overlap_block_any<LB, LA, true>(eb.nprim[kb], eb.alpha[kb], eb.coef[kb], xb, ea.nprim[ka], ea.alpha[ka],
                                  ea.coef[ka], xa, 3, Sb, dA);
  const double hij = xs[0], vsum = xs[1], dlog = xs[2];
#pragma unroll
  for (int x = 0; x < 2 * LB + 1; ++x)
#pragma unroll
    for (int y = 0; y < 2 * LA + 1; ++y) {
      const long long idx = (long long)(mu0 + x) * N + (nu0 + y);
      const double pp = P[idx], ww = W[idx];
      const double coeff = pp * (2.0 * hij - vsum) - 2.0 * ww;
      const double pg = dlog * (2.0 * pp * hij * Sb[x][y]);
#pragma unroll
      for (int c = 0; c < 3; ++c) gmu[c] += dA[x][y][c] * coeff + rv[c] * pg;
      dcmu += xs[3] * pp * Sb[x][y];
      dcnu += xs[4] * pp * Sb[x][y];
    }
}

// Molecule blockIdx.x of `mols` (or of the batch when null).  phases: bit 0
// the atom-pair terms (with gridDim.y > 1 every CTA of a molecule takes every
// gridDim.y-th block of its atom pairs), bit 1 the per-atom sums and the
// coordination-number chain (one CTA per molecule, after all pairs).  MaxL:
// the highest shell angular momentum of the batch; the s/p instantiation
// (MaxL = 1) leaves out the d-shell blocks and their registers.
template <int MaxL>
__global__ void __launch_bounds__(kGradThreads, MaxL < 2 ? kGradMinBlocksSp : kGradMinBlocks) grad_kernel(Batch B, Model M, const int* mols,
                                                                           int phases) {
  extern __shared__ double gsm[];
  const int m = mols ? mols[blockIdx.x] : blockIdx.x;
  if (B.status[m] != kOk) return;
  const int split = blockIdx.y, nsplit = gridDim.y;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int a0 = B.atom_off[m], nat = B.atom_off[m + 1] - a0;
  const int sh0 = B.shell_off[m];
  const int N = B.ao_off[m + 1] - B.ao_off[m];
  const int maxn = B.max_nat;
  double* xyz = gsm;              // 3*maxn
  double* dedcn = xyz + 3 * maxn; // maxn
  double* gel = dedcn + maxn;     // 3*maxn
  int* zs = (int*)(gel + 3 * maxn);
  int* atom_sh = zs + maxn;       // maxn+1
  int* atom_ao = atom_sh + maxn + 1;
  const double* P = B.P + B.mat_off[m];  // density of the converged SCC
  const double* W = B.W + B.mat_off[m];  // energy-weighted density
  double* pb = B.pairbuf + 8 * B.pair_off[m];

  for (int i = tid; i < nat; i += nt) {
    zs[i] = B.z[a0 + i];
    for (int x = 0; x < 3; ++x) xyz[3 * i + x] = B.xyz[3 * (a0 + i) + x];
  }
  __syncthreads();
  if (tid == 0) {
    int s = 0, o = 0;
    for (int a = 0; a < nat; ++a) {
      atom_sh[a] = s;
      atom_ao[a] = o;
      s += M.elem[zs[a]].nsh;
      o += M.elem[zs[a]].nao;
    }
    atom_sh[nat] = s;
    atom_ao[nat] = o;
  }
  __syncthreads();

  // ---- phase 1: atom pairs
  const int npair = (phases & 1) ? nat * (nat - 1) / 2 : 0;
  for (int p = tid + split * nt; p < npair; p += nt * nsplit) {
    // invert the pair index: a is the smaller atom
    int a = 0, rem = p;
    while (rem >= nat - 1 - a) {
      rem -= nat - 1 - a;
      ++a;
    }
    const int b = a + 1 + rem;
    const int za = zs[a], zb = zs[b];
    const ElemTable& ea = M.elem[za];
    const ElemTable& eb = M.elem[zb];
    const double rv[3] = {xyz[3 * b] - xyz[3 * a], xyz[3 * b + 1] - xyz[3 * a + 1], xyz[3 * b + 2] - xyz[3 * a + 2]};
    const double r2 = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
    double gmu[3] = {0, 0, 0};  // derivative with respect to atom b (mu on b, nu on a)
    double dcmu = 0.0, dcnu = 0.0;
    if (r2 <= 900.0 && r2 > 1e-24 && r2 > 1e-12) {
      const double r = sqrt(r2);
      const double rr = sqrt(r / (ea.rad + eb.rad));
      for (int kb = 0; kb < eb.nsh; ++kb) {
        const int smu = atom_sh[b] + kb;
        const double semu = B.se[sh0 + smu];
        const double vmu = B.shell_pot[sh0 + smu];
        for (int ka = 0; ka < ea.nsh; ++ka) {
          const int snu = atom_sh[a] + ka;
          const double senu = B.se[sh0 + snu];
          const double vnu = B.shell_pot[sh0 + snu];
          const double fi = 1.0 + eb.poly[kb] * rr, fj = 1.0 + ea.poly[ka] * rr;
          const double poly = fi * fj;
          const double hs = hscale(M, zb, kb, za, ka) * poly;
          const double hij = 0.5 * (semu + senu) * hs;
          double dlog = 0.0;  // src/gradient.rs:1157-1175 (scalar factor of rvec)
          if (fabs(poly) > 1e-18) dlog = (fi * ea.poly[ka] + fj * eb.poly[kb]) * 0.5 * rr / r2 / poly;
          const int mu0 = atom_ao[b] + eb.ao_first[kb], nu0 = atom_ao[a] + ea.ao_first[ka];
          const double xs[5] = {hij, vmu + vnu, dlog, -eb.kcn[kb] * hs, -ea.kcn[ka] * hs};
          if constexpr (MaxL < 2) {
            switch (eb.l[kb] * 2 + ea.l[ka]) {
              case 0: grad_shell_pair<0, 0>(eb, kb, &xyz[3 * b], ea, ka, &xyz[3 * a], P, W, N, mu0, nu0, xs, rv, gmu, dcmu, dcnu); break;
              case 1: grad_shell_pair<0, 1>(eb, kb, &xyz[3 * b], ea, ka, &xyz[3 * a], P, W, N, mu0, nu0, xs, rv, gmu, dcmu, dcnu); break;
              case 2: grad_shell_pair<1, 0>(eb, kb, &xyz[3 * b], ea, ka, &xyz[3 * a], P, W, N, mu0, nu0, xs, rv, gmu, dcmu, dcnu); break;
              default: grad_shell_pair<1, 1>(eb, kb, &xyz[3 * b], ea, ka, &xyz[3 * a], P, W, N, mu0, nu0, xs, rv, gmu, dcmu, dcnu); break;
            }
          } else
          switch (eb.l[kb] * 3 + ea.l[ka]) {
            case 0: grad_shell_pair<0, 0>(eb, kb, &xyz[3 * b], ea, ka, &xyz[3 * a], P, W, N, mu0, nu0, xs, rv, gmu, dcmu, dcnu); break;
            case 1: grad_shell_pair<0, 1>(eb, kb, &xyz[3 * b], ea, ka, &xyz[3 * a], P, W, N, mu0, nu0, xs, rv, gmu, dcmu, dcnu); break;
            case 2: grad_shell_pair<0, 2>(eb, kb, &xyz[3 * b], ea, ka, &xyz[3 * a], P, W, N, mu0, nu0, xs, rv, gmu, dcmu, dcnu); break;
            case 3: grad_shell_pair<1, 0>(eb, kb, &xyz[3 * b], ea, ka, &xyz[3 * a], P, W, N, mu0, nu0, xs, rv, gmu, dcmu, dcnu); break;
            case 4: grad_shell_pair<1, 1>(eb, kb, &xyz[3 * b], ea, ka, &xyz[3 * a], P, W, N, mu0, nu0, xs, rv, gmu, dcmu, dcnu); break;
            case 5: grad_shell_pair<1, 2>(eb, kb, &xyz[3 * b], ea, ka, &xyz[3 * a], P, W, N, mu0, nu0, xs, rv, gmu, dcmu, dcnu); break;
            case 6: grad_shell_pair<2, 0>(eb, kb, &xyz[3 * b], ea, ka, &xyz[3 * a], P, W, N, mu0, nu0, xs, rv, gmu, dcmu, dcnu); break;
            case 7: grad_shell_pair<2, 1>(eb, kb, &xyz[3 * b], ea, ka, &xyz[3 * a], P, W, N, mu0, nu0, xs, rv, gmu, dcmu, dcnu); break;
            default: grad_shell_pair<2, 2>(eb, kb, &xyz[3 * b], ea, ka, &xyz[3 * a], P, W, N, mu0, nu0, xs, rv, gmu, dcmu, dcnu); break;
          }
        }
      }
    }
    if (r2 > 1e-24) {  // Coulomb: shells of b (larger index) with shells of a
      const double r = sqrt(r2);
      if (r > 1e-12) {
        for (int kb = 0; kb < eb.nsh; ++kb) {
          const double qi = B.shell_q[sh0 + atom_sh[b] + kb];
          for (int ka = 0; ka < ea.nsh; ++ka) {
            const double qj = B.shell_q[sh0 + atom_sh[a] + ka];
            const double g = harmonic_avg(eb.hard[kb], ea.hard[ka]);
            const double den = r2 + 1.0 / (g * g);
            const double pref = -1.0 / (den * sqrt(den)) * qi * qj;
            for (int c = 0; c < 3; ++c) gmu[c] += rv[c] * pref;
          }
        }
      }
    }
    double* slot = pb + 8LL * p;  // every term is a function of R_b - R_a: the atom a force is -gmu
    slot[0] = -gmu[0];
    slot[1] = -gmu[1];
    slot[2] = -gmu[2];
    slot[3] = gmu[0];
    slot[4] = gmu[1];
    slot[5] = gmu[2];
    slot[6] = dcnu;
    slot[7] = dcmu;
  }
  if (!(phases & 2) || split != 0) return;
  __syncthreads();

  // ---- phase 2: per-atom sums in a fixed pair order
  for (int i = tid; i < nat; i += nt) {
    double g0 = 0, g1 = 0, g2 = 0, dc = 0;
    for (int j = 0; j < nat; ++j) {
      if (j == i) continue;
      const int lo = min(i, j), hi = max(i, j);
      const double* slot = pb + 8LL * tri_index(lo, hi, nat);
      const int o = (i == lo) ? 0 : 3;
      g0 += slot[o];
      g1 += slot[o + 1];
      g2 += slot[o + 2];
      dc += slot[(i == lo) ? 6 : 7];
    }
    const ElemTable& e = M.elem[zs[i]];
    for (int k = 0; k < e.nsh; ++k) {
      const int mu0 = atom_ao[i] + e.ao_first[k];
      for (int q = 0; q < 2 * e.l[k] + 1; ++q)
        dc += -e.kcn[k] * P[(long long)(mu0 + q) * N + (mu0 + q)];
    }
    gel[3 * i] = g0;
    gel[3 * i + 1] = g1;
    gel[3 * i + 2] = g2;
    dedcn[i] = dc;
  }
  __syncthreads();

  // ---- phase 3: CN chain (cutoff 30 bohr) and the classical terms
  for (int i = tid; i < nat; i += nt) {
    const double ri = M.elem[zs[i]].rcov;
    double g[3] = {gel[3 * i], gel[3 * i + 1], gel[3 * i + 2]};
    for (int j = 0; j < nat; ++j) {
      if (j == i) continue;
      const double d[3] = {xyz[3 * i] - xyz[3 * j], xyz[3 * i + 1] - xyz[3 * j + 1], xyz[3 * i + 2] - xyz[3 * j + 2]};
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (r2 <= 1e-24 || r2 > 900.0) continue;
      const double r = sqrt(r2);
      if (r <= 1e-12) continue;
      double v, dv;
      exp_count(r, ri + M.elem[zs[j]].rcov, v, dv);
      const double pref = (dedcn[i] + dedcn[j]) * dv / r;
      for (int c = 0; c < 3; ++c) g[c] += d[c] * pref;
    }
    for (int c = 0; c < 3; ++c) B.grad[3 * (a0 + i) + c] = g[c] + B.grad_classic[3 * (a0 + i) + c];
  }
}

// Launches the gradient kernel for a batch whose highest shell angular
// momentum is max_l (the s/p instantiation below 2).
cudaError_t launch_grad(int max_l, dim3 grid, size_t smem, cudaStream_t st, const Batch& B, const Model& M,
                        const int* mols, int phases) {
  auto* k = max_l >= 2 ? grad_kernel<2> : grad_kernel<1>;
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k<<<grid, kGradThreads, smem, st>>>(B, M, mols, phases);
  return cudaGetLastError();
}

}  // namespace gfn1
