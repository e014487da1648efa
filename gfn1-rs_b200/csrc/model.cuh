// GFN1-xTB model functions shared by the device kernels: H0 shell-pair scaling,
// the distance polynomial, the coordination-number counting function and the
// Klopman-Ohno kernel.
#pragma once

#include "common.cuh"

namespace gfn1 {

struct Model {
  const ElemTable* elem;        // [kNZ]
  const double* pair_scaling;   // [kNZ*kNZ]
  const double* c6ref;          // [kNZ*kNZ*kMaxRef*kMaxRef], c6ref[(zi*kNZ+zj)*25 + ri*5 + rj]
  Globals g;
};

// k_shell / kshell_pair (src/params.rs:369-376, src/hamiltonian.rs:157-165)
__device__ __forceinline__ double k_shell(const Globals& g, int l) { return l == 0 ? g.ks : (l == 1 ? g.kp : g.kd); }
__device__ __forceinline__ double kshell_pair(const Globals& g, int li, int lj) {
  if ((li == 0 && lj == 1) || (li == 1 && lj == 0)) return g.ksp;
  return 0.5 * (k_shell(g, li) + k_shell(g, lj));
}

// hscale (src/hamiltonian.rs:140-155)
__device__ __forceinline__ double hscale(const Model& M, int za, int ka, int zb, int kb) {
  const ElemTable& ea = M.elem[za];
  const ElemTable& eb = M.elem[zb];
  const int va = ea.valence[ka], vb = eb.valence[kb];
  const int la = ea.l[ka], lb = eb.l[kb];
  if (va && vb) {
    const double den = (ea.en - eb.en) * (ea.en - eb.en);
    return M.pair_scaling[za * kNZ + zb] * kshell_pair(M.g, la, lb) * (1.0 + M.g.enscale * 0.01 * den);
  } else if (va) {
    return 0.5 * (kshell_pair(M.g, la, la) + M.g.kdiff);
  } else if (vb) {
    return 0.5 * (kshell_pair(M.g, lb, lb) + M.g.kdiff);
  }
  return M.g.kdiff;
}

// Exponential counting function and its radial derivative
// (src/coordination.rs:96-106), k = 16.
__device__ __forceinline__ void exp_count(double r, double rc, double& value, double& dvalue) {
  const double kcn = 16.0;
  const double raw = -kcn * (rc / r - 1.0);
  const double arg = fmin(80.0, fmax(-80.0, raw));
  const double e = exp(arg);
  value = 1.0 / (1.0 + e);
  dvalue = (raw < -80.0 || raw > 80.0) ? 0.0 : -kcn * rc * e / (r * r * (1.0 + e) * (1.0 + e));
}

// Klopman-Ohno effective kernel with exponent 2 (src/coulomb.rs:239-248)
__device__ __forceinline__ double harmonic_avg(double a, double b) { return 2.0 / (1.0 / a + 1.0 / b); }

}  // namespace gfn1
