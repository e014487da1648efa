// Contracted STO-nG overlap blocks and their centre derivatives for s, p and d
// shells, evaluated primitive pair by primitive pair in registers.
//
// Follows the integrals of gfn1-rs src/integrals.rs: the contracted overlap
// `contracted_pair` (:290-360, index 0 of the ten moments) and its bra/ket
// derivatives `contracted_pair_with_derivatives` (:481-537, :782-868), including
// the primitive-pair screening bound `primitive_pair_bound` (:30-45) with its
// 1e-13 threshold (:17).  The 1D Gaussian moments are generated by the
// Obara-Saika recurrence E(i+1,j) = PA E(i,j) + (i E(i-1,j) + j E(i,j-1)) / 2p,
// which equals the reference's binomial expansion (`moment_1d_no_kab`, :895-920).
#pragma once

#include "common.cuh"

namespace gfn1 {

constexpr double kPi = 3.14159265358979323846;
constexpr double kPrimScreen = 1.0e-13;

// Cartesian component of AO k of a shell with angular momentum l (s: (0,0,0);
// p: x, y, z in that order, src/basis.rs:390-405).
__device__ __forceinline__ void ao_powers(int l, int k, int& px, int& py, int& pz) {
  px = (l == 1 && k == 0);
  py = (l == 1 && k == 1);
  pz = (l == 1 && k == 2);
}

// 1D moments E[i][j], i,j <= 2 (normalised so E[0][0] = 1) along one axis.
__device__ __forceinline__ void moments1d(double pa, double pb, double inv2p, double E[3][3]) {
  E[0][0] = 1.0;
  E[1][0] = pa;
  E[0][1] = pb;
  E[1][1] = pa * pb + inv2p;
  E[2][0] = pa * pa + inv2p;
  E[0][2] = pb * pb + inv2p;
  E[2][1] = pa * E[1][1] + inv2p * (E[0][1] + E[1][0]);
  E[1][2] = pb * E[1][1] + inv2p * (E[1][0] + E[0][1]);
  E[2][2] = pa * E[1][2] + inv2p * (E[0][2] + 2.0 * E[1][1]);
}

__device__ __forceinline__ double ipow(double x, int n) {
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

// Overlap block S[ka][kb] between shell (la, prims a) at A and shell (lb, prims b)
// at B; nao = 2l+1 for l <= 1.  `order_extra` is the screening order offset
// (+2 for the integral build, +3 for the gradient, src/integrals.rs:313-316, :498-501).
// When `want_deriv`, dA[ka][kb][3] receives dS/dA (bra centre); dB, when not
// null, the ket-centre derivative (equal to -dA for a two-centre overlap).
//
// Screening: the reference evaluates bound = |c_a c_b| kab (pi/p)^3/2
// (1 + r + p^-1/2)^order with kab = exp(-x), x = ab r^2 / p, and drops the pair
// when bound < 1e-13.  For x > 64 the exp-free part is checked first: if it is
// below 1e-13 e^64 the full bound is below 1e-13 too, so the same pairs are
// dropped without evaluating the exponential.
constexpr double kSkipExpArg = 64.0;
constexpr double kSkipPrefBound = 6.235149080811617e14;  // 1e-13 * e^64

template <bool WantDeriv>
__device__ void overlap_block(int la, int na, const double* alpha_a, const double* coef_a, const double* A, int lb,
                              int nb, const double* alpha_b, const double* coef_b, const double* B, int order_extra,
                              double S[3][3], double dA[3][3][3], double dB[3][3][3]) {
  const int nao_a = 2 * la + 1, nao_b = 2 * lb + 1;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      S[i][j] = 0.0;
      if (WantDeriv)
        for (int k = 0; k < 3; ++k) {
          dA[i][j][k] = 0.0;
          if (dB) dB[i][j][k] = 0.0;
        }
    }
  const double d[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
  const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  const double r = sqrt(r2);
  const int order = la + lb + order_extra;
  for (int ia = 0; ia < na; ++ia) {
    const double al = alpha_a[ia];
    for (int ib = 0; ib < nb; ++ib) {
      const double be = alpha_b[ib];
      const double p = al + be;
      const double ip = 1.0 / p;
      const double xarg = al * be * ip * r2;
      const double gpre = (kPi * ip) * sqrt(kPi * ip);
      const double pref = coef_a[ia] * coef_b[ib];
      // src/integrals.rs:30-45 (component scale is 1 for s and p AOs)
      const double pbound = fabs(pref) * gpre * ipow(1.0 + r + sqrt(ip), order);
      if (xarg > kSkipExpArg && pbound < kSkipPrefBound) continue;
      const double kab = exp(-xarg);
      if (pbound * kab < kPrimScreen) continue;
      const double c = pref * kab * gpre;
      const double inv2p = 0.5 * ip;
      double E[3][3][3];
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        const double P = (al * A[x] + be * B[x]) * ip;
        moments1d(P - A[x], P - B[x], inv2p, E[x]);
      }
      for (int ka = 0; ka < nao_a; ++ka) {
        int a[3];
        ao_powers(la, ka, a[0], a[1], a[2]);
        for (int kb = 0; kb < nao_b; ++kb) {
          int b[3];
          ao_powers(lb, kb, b[0], b[1], b[2]);
          const double ex = E[0][a[0]][b[0]], ey = E[1][a[1]][b[1]], ez = E[2][a[2]][b[2]];
          S[ka][kb] += c * ex * ey * ez;
          if (WantDeriv) {
            const double e1[3] = {ex, ey, ez};
#pragma unroll
            for (int x = 0; x < 3; ++x) {
              const double o = e1[(x + 1) % 3] * e1[(x + 2) % 3];
              const double da = 2.0 * al * E[x][a[x] + 1][b[x]] - (a[x] ? E[x][a[x] - 1][b[x]] : 0.0);
              dA[ka][kb][x] += c * da * o;
              if (dB) {
                const double db = 2.0 * be * E[x][a[x]][b[x] + 1] - (b[x] ? E[x][a[x]][b[x] - 1] : 0.0);
                dB[ka][kb][x] += c * db * o;
              }
            }
          }
        }
      }
    }
  }
}

// The same block with the angular momenta known at compile time (LA, LB in
// {0, 1}): every loop is unrolled and the block lives in registers.
template <int LA, int LB, bool WantDeriv>
__device__ __forceinline__ void overlap_block_t(int na, const double* alpha_a, const double* coef_a, const double* A,
                                                int nb, const double* alpha_b, const double* coef_b, const double* B,
                                                int order_extra, double (&S)[2 * LA + 1][2 * LB + 1],
                                                double (&dA)[2 * LA + 1][2 * LB + 1][3]) {
  constexpr int NA = 2 * LA + 1, NB = 2 * LB + 1;
#pragma unroll
  for (int i = 0; i < NA; ++i)
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      S[i][j] = 0.0;
      if (WantDeriv)
#pragma unroll
        for (int k = 0; k < 3; ++k) dA[i][j][k] = 0.0;
    }
  const double d[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
  const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  const double r = sqrt(r2);
  const int order = LA + LB + order_extra;
  for (int ia = 0; ia < na; ++ia) {
    const double al = alpha_a[ia];
    for (int ib = 0; ib < nb; ++ib) {
      const double be = alpha_b[ib];
      const double p = al + be;
      const double ip = 1.0 / p;
      const double xarg = al * be * ip * r2;
      const double gpre = (kPi * ip) * sqrt(kPi * ip);
      const double pref = coef_a[ia] * coef_b[ib];
      const double pbound = fabs(pref) * gpre * ipow(1.0 + r + sqrt(ip), order);
      if (xarg > kSkipExpArg && pbound < kSkipPrefBound) continue;
      const double kab = exp(-xarg);
      if (pbound * kab < kPrimScreen) continue;
      const double c = pref * kab * gpre;
      const double inv2p = 0.5 * ip;
      double E[3][3][3];
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        const double P = (al * A[x] + be * B[x]) * ip;
        moments1d(P - A[x], P - B[x], inv2p, E[x]);
      }
#pragma unroll
      for (int ka = 0; ka < NA; ++ka) {
        const int a[3] = {LA == 1 && ka == 0, LA == 1 && ka == 1, LA == 1 && ka == 2};
#pragma unroll
        for (int kb = 0; kb < NB; ++kb) {
          const int b[3] = {LB == 1 && kb == 0, LB == 1 && kb == 1, LB == 1 && kb == 2};
          const double ex = E[0][a[0]][b[0]], ey = E[1][a[1]][b[1]], ez = E[2][a[2]][b[2]];
          S[ka][kb] += c * ex * ey * ez;
          if (WantDeriv) {
            const double e1[3] = {ex, ey, ez};
#pragma unroll
            for (int x = 0; x < 3; ++x) {
              const double o = e1[(x + 1) % 3] * e1[(x + 2) % 3];
              const double da = 2.0 * al * E[x][a[x] + 1][b[x]] - (a[x] ? E[x][a[x] - 1][b[x]] : 0.0);
              dA[ka][kb][x] += c * da * o;
            }
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------- d shells
// Cartesian components of a shell: s (0,0,0); p x, y, z; d xx, yy, zz, xy, xz,
// yz.  The five real d AOs are the combinations of src/basis.rs:406-436 in
// their order: x^2-y^2 = sqrt3/2 (xx - yy), z^2 = (xx + yy)/2 - zz,
// xy = sqrt3 xy, xz = sqrt3 xz, yz = sqrt3 yz, over primitives normalised for
// the xx component.
constexpr double kSqrt3 = 1.7320508075688772;

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }

__host__ __device__ constexpr int cart_pow(int l, int c, int axis) {
  return l == 0 ? 0
                : (l == 1 ? (c == axis ? 1 : 0)
                          : (c < 3 ? (c == axis ? 2 : 0)
                                   : ((c == 3 && axis < 2) || (c == 4 && axis != 1) || (c == 5 && axis > 0) ? 1 : 0)));
}

// Coefficient of Cartesian component c in real AO k.
__host__ __device__ constexpr double sph_coef(int l, int k, int c) {
  return l < 2 ? (k == c ? 1.0 : 0.0)
               : (k == 0 ? (c == 0 ? 0.5 * kSqrt3 : (c == 1 ? -0.5 * kSqrt3 : 0.0))
                         : (k == 1 ? (c < 2 ? 0.5 : (c == 2 ? -1.0 : 0.0)) : (c == k + 1 ? kSqrt3 : 0.0)));
}

// Sum of |coefficients| of AO k: the component scale of the screening bound
// (src/integrals.rs:30-45).
__host__ __device__ constexpr double sph_abs_sum(int l, int k) { return l < 2 ? 1.0 : (k == 1 ? 2.0 : kSqrt3); }

// 1D moments E[i][j], i <= IA, j <= JB, by the Obara-Saika recurrences
// E(i+1,j) = PA E(i,j) + (i E(i-1,j) + j E(i,j-1)) / 2p and the same for j.
template <int IA, int JB>
__device__ __forceinline__ void moments1d_t(double pa, double pb, double inv2p, double (&E)[IA + 1][JB + 1]) {
  E[0][0] = 1.0;
#pragma unroll
  for (int i = 1; i <= IA; ++i) E[i][0] = pa * E[i - 1][0] + (i > 1 ? (i - 1) * inv2p * E[i - 2][0] : 0.0);
#pragma unroll
  for (int j = 1; j <= JB; ++j)
#pragma unroll
    for (int i = 0; i <= IA; ++i)
      E[i][j] = pb * E[i][j - 1] +
                inv2p * ((i > 0 ? i * E[i - 1][j - 1] : 0.0) + (j > 1 ? (j - 1) * E[i][j - 2] : 0.0));
}

// Overlap block (and bra-centre derivative) for shell pairs with a d shell.
// Per primitive pair the Cartesian products are formed and added to each real
// AO pair whose own screening bound, with the component scales of its two AOs,
// reaches 1e-13, so the same primitive pairs are kept as in the reference.
template <int LA, int LB, bool WantDeriv>
__device__ __forceinline__ void overlap_block_d(int na, const double* alpha_a, const double* coef_a, const double* A,
                                                int nb, const double* alpha_b, const double* coef_b, const double* B,
                                                int order_extra, double (&S)[2 * LA + 1][2 * LB + 1],
                                                double (&dA)[2 * LA + 1][2 * LB + 1][3]) {
  constexpr int NA = 2 * LA + 1, NB = 2 * LB + 1, CA = ncart(LA), CB = ncart(LB);
  constexpr int IA = LA + (WantDeriv ? 1 : 0);
  constexpr double kMaxScale = (LA == 2 ? 2.0 : 1.0) * (LB == 2 ? 2.0 : 1.0);
#pragma unroll
  for (int i = 0; i < NA; ++i)
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      S[i][j] = 0.0;
      if (WantDeriv)
#pragma unroll
        for (int k = 0; k < 3; ++k) dA[i][j][k] = 0.0;
    }
  const double d[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
  const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  const double r = sqrt(r2);
  const int order = LA + LB + order_extra;
  for (int ia = 0; ia < na; ++ia) {
    const double al = alpha_a[ia];
    for (int ib = 0; ib < nb; ++ib) {
      const double be = alpha_b[ib];
      const double p = al + be;
      const double ip = 1.0 / p;
      const double xarg = al * be * ip * r2;
      const double gpre = (kPi * ip) * sqrt(kPi * ip);
      const double pref = coef_a[ia] * coef_b[ib];
      const double pbound = fabs(pref) * gpre * ipow(1.0 + r + sqrt(ip), order);
      if (xarg > kSkipExpArg && pbound * kMaxScale < kSkipPrefBound) continue;
      const double kab = exp(-xarg);
      const double bound = pbound * kab;
      if (bound * kMaxScale < kPrimScreen) continue;
      const double c = pref * kab * gpre;
      const double inv2p = 0.5 * ip;
      double E[3][IA + 1][LB + 1];
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        const double P = (al * A[x] + be * B[x]) * ip;
        moments1d_t<IA, LB>(P - A[x], P - B[x], inv2p, E[x]);
      }
#pragma unroll
      for (int ca = 0; ca < CA; ++ca)
#pragma unroll
        for (int cb = 0; cb < CB; ++cb) {
          const int a[3] = {cart_pow(LA, ca, 0), cart_pow(LA, ca, 1), cart_pow(LA, ca, 2)};
          const int b[3] = {cart_pow(LB, cb, 0), cart_pow(LB, cb, 1), cart_pow(LB, cb, 2)};
          const double e1[3] = {E[0][a[0]][b[0]], E[1][a[1]][b[1]], E[2][a[2]][b[2]]};
          const double ov = c * e1[0] * e1[1] * e1[2];
          double dv[3] = {0.0, 0.0, 0.0};
          if constexpr (WantDeriv) {
#pragma unroll
            for (int x = 0; x < 3; ++x) {
              const double o = e1[(x + 1) % 3] * e1[(x + 2) % 3];
              const double da = 2.0 * al * E[x][a[x] + 1][b[x]] - (a[x] ? a[x] * E[x][a[x] - 1][b[x]] : 0.0);
              dv[x] = c * da * o;
            }
          }
#pragma unroll
          for (int ka = 0; ka < NA; ++ka)
#pragma unroll
            for (int kb = 0; kb < NB; ++kb) {
              const double t = sph_coef(LA, ka, ca) * sph_coef(LB, kb, cb);
              if (t == 0.0) continue;
              if (bound * (sph_abs_sum(LA, ka) * sph_abs_sum(LB, kb)) < kPrimScreen) continue;
              S[ka][kb] += t * ov;
              if (WantDeriv)
#pragma unroll
                for (int x = 0; x < 3; ++x) dA[ka][kb][x] += t * dv[x];
            }
        }
    }
  }
}

// Dispatch: s/p pairs take the register block above, pairs with a d shell the
// Cartesian-to-real one.
template <int LA, int LB, bool WantDeriv>
__device__ __forceinline__ void overlap_block_any(int na, const double* alpha_a, const double* coef_a, const double* A,
                                                  int nb, const double* alpha_b, const double* coef_b, const double* B,
                                                  int order_extra, double (&S)[2 * LA + 1][2 * LB + 1],
                                                  double (&dA)[2 * LA + 1][2 * LB + 1][3]) {
  if constexpr (LA < 2 && LB < 2)
    overlap_block_t<LA, LB, WantDeriv>(na, alpha_a, coef_a, A, nb, alpha_b, coef_b, B, order_extra, S, dA);
  else
    overlap_block_d<LA, LB, WantDeriv>(na, alpha_a, coef_a, A, nb, alpha_b, coef_b, B, order_extra, S, dA);
}

}  // namespace gfn1
