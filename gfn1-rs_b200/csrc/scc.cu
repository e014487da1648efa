// Persistent SCC kernel: each CTA pulls molecules from a work queue (most
// expensive first) and runs the complete self-consistent-charge loop of
// gfn1-rs `run_scc_with_core` (src/electronic.rs:849-2054, plain charge-vector
// branch, ladder rung 0) on the device.  The batch path launches two size
// classes concurrently (above and below 96 AOs), both with 128-thread CTAs and
// four CTAs per SM; shared memory holds the index tables and N-vectors, and the
// eigensolver's working matrix lives in the CTA's global workspace slot, cached
// by L1.  Up to 193 AOs the Householder reduction is blocked (8-column panels,
// tensor-core trailing updates); the prologue's Cholesky is left-looking over
// 8-column panels.  Wider CTAs (256/512 threads) and a working
// matrix in shared memory are used only by the allocation-free single-molecule
// entry point, which passes the room for it in the launch's shared memory.
//
// Algorithmic choices that differ from the reference but give the same results
// up to FP64 rounding:
//  * orthogonaliser: Cholesky S = L L^T instead of Lowdin S^-1/2
//    (src/linalg.rs:193-217).  The density P = C f C^T is invariant to the choice.
//    H0' = L^-1 H0 L^-T is formed once per molecule, and each iteration only adds
//    the potential term  -1/2 (M + M^T),  M = L^-1 diag(v) L  (lower triangular),
//    because  L^-1 (S o V) L^-T = L^-1 diag(v) L + (L^-1 diag(v) L)^T  for
//    V_mu,nu = v_mu + v_nu (src/electronic.rs:3133-3158).
//  * eigensolver: Householder tridiagonalisation (three barriers per column in
//    the blocked form), Sturm counts plus Laguerre steps, warm-started from
//    the previous iteration, for the eigenvalues the occupations need,
//    inverse iteration (with modified Gram-Schmidt inside eigenvalue clusters)
//    for the occupied eigenvectors only, and a blocked (compact-WY)
//    back-transformation (replaces faer's self_adjoint_eigen, src/linalg.rs:153-191).
//  * electronic energy: tr(H0 P) = sum_i f_i eps_i + sum_mu v_mu (S P)_mu,mu,
//    which holds exactly for the F that was diagonalised, so P is only formed once
//    the SCC has converged (src/electronic.rs:3182-3188, :2173-2191).
//  * Mulliken populations (S P)_mu,mu = sum_i f_i (L z_i)_mu (L^-T z_i)_mu
//    (src/electronic.rs:3160-3180).
// Fermi smearing (bisection to the bracket fixed point, :3853-3921), the
// convergence test (:1881), Broyden mixing (:3203-3309, :3759-3806) and the final
// energy assembly (:1957-2053) follow the reference step by step.
#include <float.h>

#include "common.cuh"
#include "model.cuh"

namespace gfn1 {

constexpr double kBoltzmann = 3.1668115634556e-6;  // src/constants.rs:26
constexpr int kVecSlots = 9;                          // N-length vectors kept in shared memory
constexpr int kBackNB = 16;                           // reflectors per compact-WY block

struct SccShared {
  double red[32];
  double scal[16];
  int iscal[16];
  double Tm[kBackNB][kBackNB];
  double VtV[kBackNB][kBackNB];
};

// Per-stage clock accounting by thread 0 of the CTA (no-op without a buffer).
struct StageClock {
  unsigned long long* out;
  long long t0;
  __device__ explicit StageClock(unsigned long long* o) {
    out = o;
    t0 = clock64();
  }
  __device__ __forceinline__ void mark(int stage) {
    if (!out) return;
    __syncthreads();
    if (threadIdx.x == 0) {
      const long long t = clock64();
      atomicAdd(out + stage, (unsigned long long)(t - t0));
      t0 = t;
    } else {
      t0 = clock64();
    }
  }
};

// Layout of one CTA's global workspace slot (doubles).
struct CtaWs {
  double *L, *Li, *Hp, *A, *Z, *C, *D, *iw, *W1, *W2;
  double *df, *u, *dots, *omega, *beta, *cvec, *qin, *qout, *vsh, *qlast, *dqlast, *qnext, *vout, *qat;
};
// Leading dimension of the working matrix: odd in shared memory (strided
// column accesses spread over the banks), a multiple of four doubles in global
// memory (every row starts on a 32-byte sector).
__host__ __device__ inline int work_lda(int n) { return (n & 1) ? n : n + 1; }
__host__ __device__ inline int work_lda_global(int n) { return (n + 3) & ~3; }

// Slot sizes in doubles; the slot size is a multiple of four and the working
// matrix A starts on a multiple of four (slots start 32-byte aligned).
__host__ __device__ inline long long cta_ws_size(int maxn, int maxnsh, int cap, int maxnat) {
  const long long n2 = (long long)maxn * (maxn + 1);
  const long long na = (long long)maxn * work_lda_global(maxn);
  const long long t = 11 * n2 + na + 4 + 2LL * kBackNB * maxn + 2LL * cap * maxnsh + 2LL * cap * cap + 2LL * cap +
                      8LL * maxnsh + maxnat + 64;
  return (t + 3) & ~3LL;
}
__device__ __forceinline__ CtaWs cta_ws(double* base, int maxn, int maxnsh, int cap) {
  CtaWs w;
  const long long n2 = (long long)maxn * (maxn + 1);
  w.L = base;
  w.Li = w.L + n2;
  w.Hp = w.Li + n2;
  w.A = base + ((3 * n2 + 3) & ~3LL);
  w.Z = w.A + (long long)maxn * work_lda_global(maxn);
  w.C = w.Z + n2;
  w.D = w.C + n2;
  w.iw = w.D + n2;  // 5 * n2
  w.W1 = w.iw + 5 * n2;
  w.W2 = w.W1 + (long long)kBackNB * maxn;
  w.df = w.W2 + (long long)kBackNB * maxn;
  w.u = w.df + (long long)cap * maxnsh;
  w.dots = w.u + (long long)cap * maxnsh;
  w.beta = w.dots + (long long)cap * cap;
  w.omega = w.beta + (long long)cap * cap;
  w.cvec = w.omega + cap;
  w.qin = w.cvec + cap;
  w.qout = w.qin + maxnsh;
  w.vsh = w.qout + maxnsh;
  w.qlast = w.vsh + maxnsh;
  w.dqlast = w.qlast + maxnsh;
  w.qnext = w.dqlast + maxnsh;
  w.vout = w.qnext + maxnsh;
  w.qat = w.vout + maxnsh;
  return w;
}

__host__ __device__ inline int scc_ints(int maxnsh, int maxn, int maxnat) {
  return 3 * maxnsh + maxn + maxnat + 1;
}
__host__ __device__ inline size_t scc_smem_fixed(int maxnsh, int maxn, int maxnat) {
  const size_t ib = ((size_t)4 * scc_ints(maxnsh, maxn, maxnat) + 15) & ~(size_t)15;
  return ib + sizeof(double) * kVecSlots * (size_t)maxn;
}

// Sturm count and characteristic polynomial at x for the symmetric tridiagonal
// (d, esq = e^2): returns #eigenvalues <= x and the values p, p', p'' of
// p_n(x) = det(T - x I) up to one common positive factor.  The recurrence
//   p_i = (d_i - x) p_{i-1} - e_{i-1}^2 p_{i-2}
// is LAPACK dlaebz's ratio recurrence q_i = p_i / p_{i-1} multiplied through by
// p_{i-1}, so the count (the number of negative q_i) is the same but the loop
// needs no division.  The pair (p_i, p_{i-1}) and its derivatives are rescaled
// by an exact power of two every 4 steps.  The pivot guard |q_i| < pivmin sets
// q_i = -2^-600 (LAPACK: -pivmin; the two differ only when e_i^2 < 2^-600 |d_i -
// x|, an exact split) and moves the pair to a scale where |p_i| is near 1.  The
// derivatives may overflow; they only steer the Laguerre step.
__device__ __forceinline__ double pow2_inv_scale(double m) {  // 2^-floor(log2 m), clamped to 2^+-1000
  const long long ex = ((__double_as_longlong(m) >> 52) & 0x7ff) - 1023;
  const long long sc = 1023 - (ex < -1000 ? -1000 : (ex > 1000 ? 1000 : ex));
  return __longlong_as_double(sc << 52);
}
__device__ __forceinline__ int sturm_poly(const double* d, const double* esq, int n, double x, double pivmin,
                                          double& pout, double& dpout, double& ddpout) {
  constexpr double kGuardScale = 0x1p600;
  double pm = 1.0, p = d[0] - x, dpm = 0.0, dp = -1.0, ddpm = 0.0, ddp = 0.0;
  if (fabs(p) < pivmin) {
    p = -1.0;
    pm = kGuardScale;
    dp = -kGuardScale;
  }
  int c = p <= 0.0;
  auto step = [&](double t, double e2) {
    double pn = t * p - e2 * pm;
    double dpn = t * dp - p - e2 * dpm;
    double ddpn = t * ddp - 2.0 * dp - e2 * ddpm;
    if (fabs(pn) <= pivmin * fabs(p)) {
      const double s = pow2_inv_scale(fabs(p)) * kGuardScale;
      pn = p * -pow2_inv_scale(fabs(p));
      p = pn * -kGuardScale;
      dp *= s;
      dpn *= s;
      ddp *= s;
      ddpn *= s;
    }
    c += (pn > 0.0) != (p > 0.0);
    pm = p;
    p = pn;
    dpm = dp;
    dp = dpn;
    ddpm = ddp;
    ddp = ddpn;
  };
  int i = 1;
  // groups of four steps with the loads issued first, then a rescale
  for (; i + 3 < n; i += 4) {
    const double t0 = d[i] - x, t1 = d[i + 1] - x, t2 = d[i + 2] - x, t3 = d[i + 3] - x;
    const double e0 = esq[i - 1], e1 = esq[i], e2 = esq[i + 1], e3 = esq[i + 2];
    step(t0, e0);
    step(t1, e1);
    step(t2, e2);
    step(t3, e3);
    const double sc = pow2_inv_scale(fmax(fabs(p), fabs(pm)));
    p *= sc;
    pm *= sc;
    dp *= sc;
    dpm *= sc;
    ddp *= sc;
    ddpm *= sc;
  }
  for (; i < n; ++i) step(d[i] - x, esq[i - 1]);
  pout = p;
  dpout = dp;
  ddpout = ddp;
  return c;
}

__device__ __forceinline__ double hash_unit(unsigned a, unsigned b) {
  unsigned h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u) * 0x85EBCA77u;
  h ^= h >> 15;
  h *= 0x2C1B3C6Du;
  h ^= h >> 12;
  h *= 0x297A2D39u;
  h ^= h >> 15;
  return (double)(h & 0xFFFFFF) / 16777216.0 - 0.5;
}

// Gaussian elimination with partial pivoting of the tridiagonal T - lam I.
// The five factor arrays of eigenvector column j are stored interleaved,
// w[(a * n + i) * ldw + j], so the threads of a warp access consecutive words;
// the pivots are kept as reciprocals, so the solves only multiply.
__device__ void tri_factor(const double* d, const double* e, int n, double lam, double tiny, double* w, int ldw) {
  double a = d[0] - lam;
  double c = n > 1 ? e[0] : 0.0;
  const long long s = (long long)n * ldw;
  for (int k = 0; k < n - 1; ++k) {
    const double b = e[k];
    const double an = d[k + 1] - lam;
    const double cn = (k + 1 < n - 1) ? e[k + 1] : 0.0;
    double* wk = w + (long long)k * ldw;
    if (fabs(a) >= fabs(b)) {
      double piv = a;
      if (fabs(piv) < tiny) piv = piv >= 0.0 ? tiny : -tiny;
      const double r = 1.0 / piv;
      wk[0] = r;
      wk[s] = c;
      wk[2 * s] = 0.0;
      wk[3 * s] = b * r;
      wk[4 * s] = 0.0;
      a = an - b * r * c;
      c = cn;
    } else {
      const double r = 1.0 / b;
      const double mult = a * r;
      wk[0] = r;
      wk[s] = an;
      wk[2 * s] = cn;
      wk[3 * s] = mult;
      wk[4 * s] = 1.0;
      a = c - mult * an;
      c = -mult * cn;
    }
  }
  if (fabs(a) < tiny) a = a >= 0.0 ? tiny : -tiny;
  w[(long long)(n - 1) * ldw] = 1.0 / a;
}

// Back substitution of tri_solve from the last forward-eliminated entry
// `cur`; returns |x|^2 of the solution.
__device__ double tri_back(const double* w, int n, int ldw, double* x, long long stride, double cur) {
  const long long s = (long long)n * ldw;
  double x2 = cur * w[(long long)(n - 1) * ldw];  // x[n-1]
  x[(n - 1) * stride] = x2;
  double nrm = x2 * x2;
  if (n == 1) return nrm;
  const double* w2 = w + (long long)(n - 2) * ldw;
  double x1 = (x[(n - 2) * stride] - w2[s] * x2) * w2[0];  // x[n-2]
  x[(n - 2) * stride] = x1;
  nrm += x1 * x1;
  int k = n - 3;
  for (; k >= 3; k -= 4) {
    double rh[4], u1[4], u2[4], rp[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double* wk = w + (long long)(k - q) * ldw;
      rh[q] = x[(k - q) * stride];
      u1[q] = wk[s];
      u2[q] = wk[2 * s];
      rp[q] = wk[0];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double x0 = (rh[q] - u1[q] * x1 - u2[q] * x2) * rp[q];
      x[(k - q) * stride] = x0;
      nrm += x0 * x0;
      x2 = x1;
      x1 = x0;
    }
  }
  for (; k >= 0; --k) {
    const double* wk = w + (long long)k * ldw;
    const double x0 = (x[k * stride] - wk[s] * x1 - wk[2 * s] * x2) * wk[0];
    x[k * stride] = x0;
    nrm += x0 * x0;
    x2 = x1;
    x1 = x0;
  }
  return nrm;
}

// Solves (T - lam I) x = b in place with the factors of tri_factor.  The
// running entries are carried in registers and the loads of x and of the
// factors are issued four steps ahead of their use, so the serial recurrences
// do not wait on memory at every step.  Returns |x|^2 of the solution.
__device__ double tri_solve(const double* w, int n, int ldw, double* x, long long stride) {
  const long long s = (long long)n * ldw;
  double cur = x[0];
  int k = 0;
  for (; k + 4 <= n - 1; k += 4) {
    double fl[4], mu[4], xn[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double* wk = w + (long long)(k + q) * ldw;
      fl[q] = wk[4 * s];
      mu[q] = wk[3 * s];
      xn[q] = x[(k + q + 1) * stride];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double xk = cur, xk1 = xn[q];
      if (fl[q] != 0.0) {
        xk = xn[q];
        xk1 = cur;
      }
      xk1 -= mu[q] * xk;
      x[(k + q) * stride] = xk;
      cur = xk1;
    }
  }
  for (; k < n - 1; ++k) {
    const double* wk = w + (long long)k * ldw;
    double xk = cur, xk1 = x[(k + 1) * stride];
    if (wk[4 * s] != 0.0) {
      const double t = xk;
      xk = xk1;
      xk1 = t;
    }
    xk1 -= wk[3 * s] * xk;
    x[k * stride] = xk;
    cur = xk1;
  }
  return tri_back(w, n, ldw, x, stride, cur);
}

// tri_factor for the shift lam together with the forward elimination of the
// right-hand side b_i = hash_unit(i, col) + 1e-3 (the start vector of inverse
// iteration), stored in x; returns the last eliminated entry, from which
// tri_back completes the first solve.
__device__ double tri_factor_rhs(const double* d, const double* e, int n, double lam, double tiny, double* w,
                                 int ldw, double* x, long long stride, unsigned col) {
  double a = d[0] - lam;
  double c = n > 1 ? e[0] : 0.0;
  const long long s = (long long)n * ldw;
  double cur = hash_unit(0, col) + 1e-3;
  for (int k = 0; k < n - 1; ++k) {
    const double b = e[k];
    const double an = d[k + 1] - lam;
    const double cn = (k + 1 < n - 1) ? e[k + 1] : 0.0;
    double* wk = w + (long long)k * ldw;
    double xk = cur, xk1 = hash_unit(k + 1, col) + 1e-3;
    if (fabs(a) >= fabs(b)) {
      double piv = a;
      if (fabs(piv) < tiny) piv = piv >= 0.0 ? tiny : -tiny;
      const double r = 1.0 / piv;
      wk[0] = r;
      wk[s] = c;
      wk[2 * s] = 0.0;
      wk[3 * s] = b * r;
      wk[4 * s] = 0.0;
      xk1 -= (b * r) * xk;
      a = an - b * r * c;
      c = cn;
    } else {
      const double r = 1.0 / b;
      const double mult = a * r;
      wk[0] = r;
      wk[s] = an;
      wk[2 * s] = cn;
      wk[3 * s] = mult;
      wk[4 * s] = 1.0;
      const double t = xk;
      xk = xk1;
      xk1 = t - mult * xk;
      a = c - mult * an;
      c = -mult * cn;
    }
    x[k * stride] = xk;
    cur = xk1;
  }
  if (fabs(a) < tiny) a = a >= 0.0 ? tiny : -tiny;
  w[(long long)(n - 1) * ldw] = 1.0 / a;
  return cur;
}

// ---------------------------------------------------------------- stages

// Householder reduction of the symmetric A (full storage, leading dimension lda)
// to tridiagonal (d, e); reflector k is kept in row k right of the diagonal
// with its factor in tau[k] (H_k = I - tau_k v v^T).  Two barriers per column:
// the matrix-vector product and the p.v partial sums, then the rank-2 update,
// during which warp 0 also forms the norm of the next pivot row.
// Four interleaved warp reductions (their shuffle latencies overlap).
__device__ __forceinline__ void warp_sum4(double& a, double& b, double& c, double& d) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
    d += __shfl_xor_sync(0xffffffffu, d, o);
  }
}

// D += A B for one 8x8x4 FP64 tile on the tensor cores (PTX mma.m8n8k4 .f64,
// row-major A, column-major B): lane l holds A[l/4][l%4], B[l%4][l/4] and
// D[l/4][2(l%4)], D[l/4][2(l%4)+1].
__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Householder reduction of the symmetric A (full storage, leading dimension
// lda) to tridiagonal form: d, e, reflector scalars tau, and the reflector of
// column k in row k (entries k+1..N-1).  Per column: p = beta A22 v by warps
// over rows (four rows at a time, lanes over columns), one barrier, then the
// rank-2 update A22 -= v w^T + w v^T with w = p - K v, which also yields the
// norm of the next column; a second barrier.  While the trailing size is at
// most 32 * kCols, each lane keeps v_j and w_j of its columns in registers, so
// the update reads and writes each element once.
// One column of the Householder reduction after its reflector (v0, beta,
// alpha) is known: p = beta A22 v, the rank-2 update and the norm of the next
// column, which it returns.  Cached: the trailing size fits 32 * kCols and each
// lane keeps its columns of v and w in registers.
template <int NT, bool Cached>
__device__ __forceinline__ double householder_column(double* A, int lda, int N, int k, double v0, double beta,
                                                     double alpha, double* d, double* e, double* tau, double* pvec,
                                                     SccShared& sh) {
  constexpr int NW = NT / 32;
  constexpr int kCols = 6;
  constexpr bool cached = Cached;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int m = N - k - 1;
  double* rowk = A + (long long)k * lda + (k + 1);
  double* a22 = A + (long long)(k + 1) * lda + (k + 1);
  double vreg[kCols], wreg[kCols];
#pragma unroll
  for (int c = 0; c < kCols; ++c) {
    const int j = lane + 32 * c;
    vreg[c] = (cached && j < m) ? (j == 0 ? v0 : rowk[j]) : 0.0;
  }
  // p = beta A22 v
  double pv_part = 0.0;
  for (int i0 = wid; i0 < m; i0 += 4 * NW) {
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    if (cached) {
#pragma unroll
      for (int c = 0; c < kCols; ++c) {
        const int j = lane + 32 * c;
        if (j < m) {
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const int i = i0 + r * NW;
            if (i < m) s[r] += a22[(long long)i * lda + j] * vreg[c];
          }
        }
      }
    } else {
      for (int j = lane; j < m; j += 32) {
        const double v = (j == 0) ? v0 : rowk[j];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int i = i0 + r * NW;
          if (i < m) s[r] += a22[(long long)i * lda + j] * v;
        }
      }
    }
    warp_sum4(s[0], s[1], s[2], s[3]);
    if (lane == 0) {
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int i = i0 + r * NW;
        if (i < m) {
          const double pi = beta * s[r];
          pvec[i] = pi;
          pv_part += pi * (i == 0 ? v0 : rowk[i]);
        }
      }
    }
  }
  if (lane == 0) sh.red[wid] = pv_part;
  __syncthreads();
  double pv = 0.0;
#pragma unroll
  for (int w = 0; w < NW; ++w) pv += sh.red[w];
  const double K = 0.5 * beta * pv;
  if (tid == 0) {
    d[k] = A[(long long)k * lda + k];
    e[k] = alpha;
    tau[k] = beta;
  }
#pragma unroll
  for (int c = 0; c < kCols; ++c) {
    const int j = lane + 32 * c;
    wreg[c] = (cached && j < m) ? pvec[j] - K * vreg[c] : 0.0;
  }
  // A22 -= v w^T + w v^T; warp 0 also takes the norm of the next column (row 1 of A22 from entry 1)
  double nrm = 0.0;
  for (int i = wid; i < m; i += NW) {
    double* brow = a22 + (long long)i * lda;
    const double vi = (i == 0) ? v0 : rowk[i];
    const double wi = pvec[i] - K * vi;
    if (cached) {
#pragma unroll
      for (int c = 0; c < kCols; ++c) {
        const int j = lane + 32 * c;
        if (j < m) {
          const double nb = brow[j] - (vi * wreg[c] + wi * vreg[c]);
          brow[j] = nb;
          if (i == 0 && j >= 1) nrm += nb * nb;
        }
      }
    } else {
      for (int j = lane; j < m; j += 32) {
        const double vj = (j == 0) ? v0 : rowk[j];
        const double wj = pvec[j] - K * vj;
        const double nb = brow[j] - (vi * wj + wi * vj);
        brow[j] = nb;
        if (i == 0 && j >= 1) nrm += nb * nb;
      }
    }
  }
  if (wid == 0) {
    nrm = warp_sum(nrm);
    if (lane == 0) sh.scal[3] = nrm;
  }
  __syncthreads();
  if (tid == 0) rowk[0] = v0;  // the reflector of column k is row k from entry k+1
  return sh.scal[3];
}

// The large-trailing-size column out of line, so that the hot loop of the
// usual sizes stays compact.
template <int NT>
__device__ __noinline__ double householder_column_wide(double* A, int lda, int N, int k, double v0, double beta,
                                                       double alpha, double* d, double* e, double* tau, double* pvec,
                                                       SccShared& sh) {
  return householder_column<NT, false>(A, lda, N, k, v0, beta, alpha, d, e, tau, pvec, sh);
}

template <int NT>
__device__ void tridiagonalize(double* A, int lda, int N, double* d, double* e, double* tau, double* pvec,
                               SccShared& sh) {
  constexpr int kCols = 6;
  const int tid = threadIdx.x;
  double part = 0.0;
  if (N >= 3)
    for (int j = 1 + tid; j < N; j += NT) part += A[j] * A[j];
  double xn2 = block_sum(part, sh.red);
  for (int k = 0; k < N - 2; ++k) {
    const int m = N - k - 1;
    const double* rowk = A + (long long)k * lda + (k + 1);
    const double x0 = rowk[0];
    const double tail = xn2 - x0 * x0;
    if (tail == 0.0) {  // column already reduced
      __syncthreads();
      if (tid == 0) {
        d[k] = A[(long long)k * lda + k];
        e[k] = x0;
        tau[k] = 0.0;
      }
      double p2 = 0.0;
      const double* nrow = A + (long long)(k + 1) * lda;
      for (int j = k + 2 + tid; j < N; j += NT) p2 += nrow[j] * nrow[j];
      xn2 = block_sum(p2, sh.red);
      continue;
    }
    const double xn = sqrt(xn2);
    const double alpha = x0 >= 0.0 ? -xn : xn;
    const double v0 = x0 - alpha;
    const double beta = 2.0 / (v0 * v0 + tail);
    xn2 = (m <= 32 * kCols) ? householder_column<NT, true>(A, lda, N, k, v0, beta, alpha, d, e, tau, pvec, sh)
                            : householder_column_wide<NT>(A, lda, N, k, v0, beta, alpha, d, e, tau, pvec, sh);
  }
  __syncthreads();
  if (tid == 0) {
    if (N >= 2) {
      d[N - 2] = A[(long long)(N - 2) * lda + (N - 2)];
      e[N - 2] = A[(long long)(N - 1) * lda + (N - 2)];
      tau[N - 2] = 0.0;
    }
    d[N - 1] = A[(long long)(N - 1) * lda + (N - 1)];
    e[N - 1] = 0.0;
    tau[N - 1] = 0.0;
  }
  __syncthreads();
}

// Blocked Householder reduction (panels of kPanel columns, four-warp CTAs, at
// most 32 * 6 + 1 rows): the same reflectors as tridiagonalize, but the rank-2
// updates of a panel are applied lazily to each panel column and, at the end
// of the panel, to the trailing matrix in one FP64 tensor-core pass,
// A22 -= V W^T + W V^T.  Per column: the column with the panel's earlier
// updates (x), its reflector (stored in row k as before), p = beta (A22 v -
// V (W^T v) - W (V^T v)) with A22 as of the panel start, and w = p - K v kept
// in Wp (kPanel x N, row l for the panel's column l).  V is read from the
// reflector rows of A.  xs and pvec are N-vectors of scratch.  A is the
// global working matrix (32-byte aligned, lda a multiple of four).
constexpr int kPanel = 8;
template <int NT>
__device__ void tridiagonalize_blocked(double* A, int lda, int N, double* d, double* e, double* tau, double* pvec,
                                       double* xs, double* Wp, SccShared& sh) {
  constexpr int NW = NT / 32;
  constexpr int kCols = 6;
  static_assert(NW == 4, "four warps");
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  for (int k0 = 0; k0 < N - 2; k0 += kPanel) {
    const int nbp = min(kPanel, N - 2 - k0);
    // W of the previous column at row k, which thread 0 wrote: every thread
    // forms it itself, so that the column needs no barrier after W is stored
    double w_last = 0.0;
    for (int j = 0; j < nbp; ++j) {
      const int k = k0 + j, m = N - k - 1;
      // x: row k (= column k) from the diagonal, with the panel's earlier updates
      double part = 0.0;
      for (int t = tid; t <= m; t += NT) {
        const int i = k + t;
        double x = A[(long long)k * lda + i];
#pragma unroll 4
        for (int l = 0; l < j; ++l) {
          const double* vl = A + (long long)(k0 + l) * lda;
          const double* wl = Wp + (long long)l * N;
          const double wk = (l == j - 1) ? w_last : wl[k];
          x -= vl[k] * wl[i] + wk * vl[i];
        }
        xs[t] = x;
        if (t >= 1) part += x * x;
      }
      part = warp_sum(part);
      if (lane == 0) sh.red[wid] = part;
      __syncthreads();
      const double xn2 = (sh.red[0] + sh.red[1]) + (sh.red[2] + sh.red[3]);
      const double x0 = xs[1];
      const double tail = xn2 - x0 * x0;
      if (tid == 0) d[k] = xs[0];
      if (tail == 0.0) {  // column already reduced: no reflector, W column zero
        for (int t = tid; t < m; t += NT) {
          A[(long long)k * lda + k + 1 + t] = xs[1 + t];
          Wp[(long long)j * N + k + 1 + t] = 0.0;
        }
        if (tid == 0) {
          e[k] = x0;
          tau[k] = 0.0;
        }
        w_last = 0.0;
        __syncthreads();
        continue;
      }
      const double xn = sqrt(xn2);
      const double alpha = x0 >= 0.0 ? -xn : xn;
      const double v0 = x0 - alpha;
      const double beta = 2.0 / (v0 * v0 + tail);
      double vreg[kCols];
#pragma unroll
      for (int c = 0; c < kCols; ++c) {
        const int jj = lane + 32 * c;
        vreg[c] = jj < m ? (jj == 0 ? v0 : xs[1 + jj]) : 0.0;
      }
      if (wid == 0) {  // the reflector of column k is row k from entry k+1
#pragma unroll
        for (int c = 0; c < kCols; ++c) {
          const int jj = lane + 32 * c;
          if (jj < m) A[(long long)k * lda + k + 1 + jj] = vreg[c];
        }
      }
      // raw A22 v: A22 is kept symmetric, so entry t is column t of A22
      // dotted with v, and each row of A22 read across the threads is
      // contiguous (no cross-lane sums); v from shared memory.  Each thread
      // takes two adjacent columns with 16-byte loads: the pair of absolute
      // columns (c, c + 1), c even, so that every load is aligned (A starts on
      // 32 bytes, lda is a multiple of four); a pair may reach column k (left
      // of A22) or column N (the row's padding), whose sums are dropped.  Per
      // column, two partial sums over odd and even rows, eight rows in
      // flight.
      {
        const int u0 = (k + 1) >> 1, np = ((N - 1) >> 1) - u0 + 1, ld2 = lda >> 1;
        const double2* rowk = reinterpret_cast<const double2*>(A + (long long)(k + 1) * lda) + u0;
        for (int p = tid; p < np; p += NT) {
          const double2* col = rowk + p;
          const double2 a0 = col[0];
          double s0 = a0.x * v0, s1 = 0.0, q0 = a0.y * v0, q1 = 0.0;
          int r = 1;
          for (; r + 7 < m; r += 8) {
            double2 a[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) a[u] = col[(long long)(r + u) * ld2];
#pragma unroll
            for (int u = 0; u < 8; u += 2) {
              const double xa = xs[1 + r + u], xb = xs[2 + r + u];
              s0 += a[u].x * xa;
              q0 += a[u].y * xa;
              s1 += a[u + 1].x * xb;
              q1 += a[u + 1].y * xb;
            }
          }
          for (; r < m; ++r) {
            const double2 a = col[(long long)r * ld2];
            s0 += a.x * xs[1 + r];
            q0 += a.y * xs[1 + r];
          }
          const int t = 2 * (u0 + p) - (k + 1);  // A22 index of the pair's first column
          if (t >= 0) pvec[t] = s0 + s1;
          if (t + 1 < m) pvec[t + 1] = q0 + q1;
        }
      }
      for (int l = wid; l < j; l += NW) {
        const double* vl = A + (long long)(k0 + l) * lda + (k + 1);
        const double* wl = Wp + (long long)l * N + (k + 1);
        double om = 0.0, nu = 0.0;
#pragma unroll
        for (int c = 0; c < kCols; ++c) {
          const int jj = lane + 32 * c;
          if (jj < m) {
            om += wl[jj] * vreg[c];
            nu += vl[jj] * vreg[c];
          }
        }
        om = warp_sum(om);
        nu = warp_sum(nu);
        if (lane == 0) {
          sh.VtV[0][l] = om;
          sh.VtV[1][l] = nu;
        }
      }
      __syncthreads();
      // p = beta (A22 v - V (W^T v) - W (V^T v)) and p.v
      // (at most two entries per thread: N <= 32 * kCols + 1; v kept in
      // registers, since the next column overwrites xs without a barrier)
      double pv_part = 0.0;
      double vt[2] = {0.0, 0.0};
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int t = tid + u * NT;
        if (t < m) {
          const int i = k + 1 + t;
          double p = pvec[t];
#pragma unroll 4
          for (int l = 0; l < j; ++l)
            p -= A[(long long)(k0 + l) * lda + i] * sh.VtV[0][l] + Wp[(long long)l * N + i] * sh.VtV[1][l];
          p *= beta;
          pvec[t] = p;
          vt[u] = t == 0 ? v0 : xs[1 + t];
          pv_part += p * vt[u];
        }
      }
      pv_part = warp_sum(pv_part);
      if (lane == 0) sh.red[4 + wid] = pv_part;
      __syncthreads();
      const double K = 0.5 * beta * ((sh.red[4] + sh.red[5]) + (sh.red[6] + sh.red[7]));
      // each thread stores W at the rows whose x it forms in the next column
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int t = tid + u * NT;
        if (t < m) Wp[(long long)j * N + k + 1 + t] = pvec[t] - K * vt[u];
      }
      w_last = pvec[0] - K * v0;
      if (tid == 0) {
        e[k] = alpha;
        tau[k] = beta;
      }
      if (j == nbp - 1) __syncthreads();  // the trailing update reads all of W
    }
    // trailing matrix: A22 -= V W^T + W V^T for rows and columns >= s0, as
    // 8x8 tiles starting from A, k over the panel's columns
    const int s0 = k0 + nbp, ms = N - s0;
    const int T = (ms + 7) >> 3;
    for (int tile = wid; tile < T * T; tile += NW) {
      const int I = tile / T, J = tile - I * T;
      const int i = s0 + I * 8 + g, jb = s0 + J * 8 + g, jc = s0 + J * 8 + 2 * t4;
      double c0 = (i < N && jc < N) ? A[(long long)i * lda + jc] : 0.0;
      double c1 = (i < N && jc + 1 < N) ? A[(long long)i * lda + jc + 1] : 0.0;
      for (int l0 = 0; l0 < nbp; l0 += 4) {
        const int l = l0 + t4;
        const bool lok = l < nbp;
        const double* vl = A + (long long)(k0 + (lok ? l : 0)) * lda;
        const double* wl = Wp + (long long)(lok ? l : 0) * N;
        dmma_m8n8k4(c0, c1, (lok && i < N) ? -vl[i] : 0.0, (lok && jb < N) ? wl[jb] : 0.0);
        dmma_m8n8k4(c0, c1, (lok && i < N) ? -wl[i] : 0.0, (lok && jb < N) ? vl[jb] : 0.0);
      }
      if (i < N && jc < N) A[(long long)i * lda + jc] = c0;
      if (i < N && jc + 1 < N) A[(long long)i * lda + jc + 1] = c1;
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (N >= 2) {
      d[N - 2] = A[(long long)(N - 2) * lda + (N - 2)];
      e[N - 2] = A[(long long)(N - 1) * lda + (N - 2)];
      tau[N - 2] = 0.0;
    }
    d[N - 1] = A[(long long)(N - 1) * lda + (N - 1)];
    e[N - 1] = 0.0;
    tau[N - 1] = 0.0;
  }
  __syncthreads();
}

// Eigenvalues k = 0..nneed-1 and N-1 of the tridiagonal, one thread each.
// Bisection on the Sturm count until the count at the iterate x says that
// eigenvalue k is the nearest one above (count k) or below (count k+1); from
// there Laguerre steps toward it.  For a polynomial with real roots the
// Laguerre step in a chosen direction lands between x and the adjacent root on
// that side, so the iterates approach eigenvalue k monotonically and converge
// cubically (Li & Zeng, "Laguerre's iteration in solving the symmetric
// tridiagonal eigenproblem - revisited", SIAM J. Sci. Comput. 15, 1994).
// Every evaluation also tightens the bisection bracket, and a step that leaves
// it falls back to bisection.
// Eigenvalue k of the tridiagonal (one thread).  x0: a first iterate inside
// (gl, gu), e.g. the eigenvalue of the previous SCC iteration (the search then
// usually starts next to eigenvalue k and takes Laguerre steps at once);
// otherwise the midpoint.
__device__ __forceinline__ double eigenvalue_k(const double* d, const double* esq, int N, int k, double gl, double gu,
                                              double pivmin, double atol, double x0 = 0.0, bool warm = false) {
  const double dn = (double)N;
  double lo = gl, hi = gu;
  double x = (warm && x0 > lo && x0 < hi) ? x0 : 0.5 * (lo + hi);
  for (int it = 0; it < 160; ++it) {
    double p, dp, ddp;
    const int c = sturm_poly(d, esq, N, x, pivmin, p, dp, ddp);
    if (c >= k + 1)
      hi = x;
    else
      lo = x;
    const double tol = 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + atol;
    if (hi - lo <= tol) {
      x = 0.5 * (lo + hi);
      break;
    }
    double xn = 0.5 * (lo + hi);
    if (c == k || c == k + 1) {
      // u = p/p', w = p p''/p'^2; step = N u / (1 + sigma sqrt((N-1)(N(1-w)-1)))
      // with sigma chosen so that the step moves toward eigenvalue k.
      const double u = p / dp;
      const double w = (p * ddp) / (dp * dp);
      const double sq = sqrt((dn - 1.0) * (dn * (1.0 - w) - 1.0));
      const bool up = (c == k);
      const double sigma = ((u > 0.0) == up) ? -1.0 : 1.0;
      const double step = dn * u / (1.0 + sigma * sq);
      const double xt = x - step;
      // The Newton ratio u points to the nearest eigenvalue: when it points
      // away from eigenvalue k, x sits next to the neighbour on the other
      // side, where the Laguerre step is tiny and proves nothing.
      const bool nearest = up ? (u < 0.0) : (u > 0.0);
      if (nearest && fabs(step) <= 32.0 * tol) {  // cubic convergence: the step bounds the error
        x = fmin(fmax(xt, lo), hi);
        break;
      }
      if (xt > lo && xt < hi && (nearest || fabs(step) >= 0.125 * (hi - lo))) xn = xt;
    }
    if (xn <= lo || xn >= hi) break;
    x = xn;
  }
  return x;
}

// nwarm: eps[0..nwarm) and eps[N-1] hold the previous SCC iteration's
// eigenvalues, the first iterates of their searches (0: none).
template <int NT>
__device__ void eigenvalues(const double* d, const double* esq, int N, int nneed, double gl, double gu,
                            double pivmin, double atol, double* eps, int nwarm = 0) {
  const int nlist = (nneed < N) ? nneed + 1 : N;
  for (int slot = threadIdx.x; slot < nlist; slot += NT) {
    const int k = (slot < nneed) ? slot : N - 1;
    eps[k] = eigenvalue_k(d, esq, N, k, gl, gu, pivmin, atol, eps[k], nwarm > 0 && (k < nwarm || k == N - 1));
  }
  __syncthreads();
}

// Fermi occupations by bisection to the bracket fixed point (src/electronic.rs:
// 3853-3921), one warp.  Only eps[0..nneed) and eps[N-1] are known: orbitals in
// between lie at or above eps[nneed-1]; while a trial mu keeps them beyond the
// +80 kT clamp each contributes exactly 2/(1+e^80).  When a decision would need
// them, `ambiguous` is set and the caller computes every eigenvalue.
template <int CAP>
__device__ void fermi_warp(const double* eps, int N, int nneed, double nelec, double kt, double* occ, double& mu_out,
                           double& ts_out, bool& ambiguous) {
  constexpr double cap = CAP;  // electrons per orbital: 2, or 1 in a spin channel
  const int lane = threadIdx.x & 31;
  ambiguous = false;
  double mu = 0.0, ts = 0.0;
  if (kt <= 0.0) {  // aufbau (src/electronic.rs:3830-3851); needs every orbital up to the HOMO
    double rem = fmax(nelec, 0.0);
    int homo = 0;
    for (int i = 0; i < N; ++i) {
      const double fill = fmin(rem, cap);
      if (lane == 0) occ[i] = fill;
      rem -= fill;
      if (fill > 1e-12) homo = i;
    }
    if (homo >= nneed && nneed < N) ambiguous = true;
    mu = eps[homo];
  } else if (nelec <= 0.0) {
    for (int i = lane; i < N; i += 32) occ[i] = 0.0;
    mu = eps[0];
  } else if (nelec >= cap * N) {
    for (int i = lane; i < N; i += 32) occ[i] = cap;
    mu = eps[N - 1];
  } else {
    const double c80 = cap / (1.0 + exp(80.0));
    const double cm80 = cap / (1.0 + exp(-80.0));
    const int nunc = (nneed < N) ? (N - 1 - nneed) : 0;
    const double etop = eps[nneed - 1];
    const double ikt = 1.0 / kt;
    auto fo = [&](double ei, double m) {
      const double x = (ei - m) * ikt;
      if (x >= 80.0) return c80;
      if (x <= -80.0) return cm80;
      return cap / (1.0 + exp(x));
    };
    double lo = eps[0] - 100.0 * kt - 10.0, hi = eps[N - 1] + 100.0 * kt + 10.0;
    for (int it = 0; it < 200; ++it) {
      const double mid = 0.5 * (lo + hi);
      double s = 0.0;
      for (int i = lane; i < nneed; i += 32) s += fo(eps[i], mid);
      if (lane == 0 && nneed < N) s += fo(eps[N - 1], mid);
      s = warp_sum(s);
      if (nunc > 0) {
        if ((etop - mid) / kt >= 80.0) s += nunc * c80;
        else if (s < nelec) {
          ambiguous = true;
          break;
        }
      }
      double nlo = lo, nhi = hi;
      if (s < nelec) nlo = mid;
      else nhi = mid;
      if (nlo == lo && nhi == hi) break;
      lo = nlo;
      hi = nhi;
    }
    mu = 0.5 * (lo + hi);
    if (!ambiguous && nunc > 0 && !((etop - mu) / kt >= 80.0)) ambiguous = true;
    if (!ambiguous) {
      double t = 0.0;
      for (int i = lane; i < N; i += 32) {
        const bool known = i < nneed || i == N - 1;
        const double f = known ? fo(eps[i], mu) : c80;
        occ[i] = f;
        const double nn = fmin(1.0 - 1e-16, fmax(1e-16, f / cap));
        t += cap * kt * (nn * log(nn) + (1.0 - nn) * log(1.0 - nn));
      }
      ts = warp_sum(t);
    }
  }
  mu_out = mu;
  ts_out = ts;
}

// Finite-temperature occupations (kt > 0, 0 < nelec < 2N) by the whole CTA.
// The reference bisects [eps_0 - 100 kT - 10, eps_N-1 + 100 kT + 10] on
// "electron count < nelec" until the bracket stops shrinking
// (src/electronic.rs:3853-3921); here each round places one trial mu per warp,
// NW + 1 equal subintervals, and keeps the subinterval where the count crosses
// nelec, so the bracket converges to the same crossing in log_(NW+1) rounds.
// Eigenvalues beyond eps[nneed-1] are unknown (apart from eps[N-1]); they are
// clamped at +80 kT like in fermi_warp, and a trial mu at which they would
// matter makes the result ambiguous (the caller then computes all of them).
// Shared scratch: sh.VtV rows 0 and 1.
template <int NT, int CAP>
__device__ void fermi_cta(const double* eps, int N, int nneed, double nelec, double kt, double* occ, SccShared& sh,
                          double& mu_out, double& ts_out, bool& ambiguous) {
  constexpr int NW = NT / 32;
  constexpr double cap = CAP;  // electrons per orbital: 2, or 1 in a spin channel
  static_assert(NW <= 16, "one trial point per warp");
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const double c80 = cap / (1.0 + exp(80.0));
  const double cm80 = cap / (1.0 + exp(-80.0));
  const int nunc = (nneed < N) ? (N - 1 - nneed) : 0;
  const double etop = eps[nneed - 1];
  const double ikt = 1.0 / kt;
  auto fo = [&](double ei, double m) {
    const double x = (ei - m) * ikt;
    if (x >= 80.0) return c80;
    if (x <= -80.0) return cm80;
    return cap / (1.0 + exp(x));
  };
  double lo = eps[0] - 100.0 * kt - 10.0, hi = eps[N - 1] + 100.0 * kt + 10.0;
  bool amb = false;
  for (int round = 0; round < 64; ++round) {
    const double h = (hi - lo) / (double)(NW + 1);
    const double mid = fmin(lo + (double)(wid + 1) * h, hi);
    double sm = 0.0;
    for (int i = lane; i < nneed; i += 32) sm += fo(eps[i], mid);
    if (lane == 0 && nneed < N) sm += fo(eps[N - 1], mid);
    sm = warp_sum(sm);
    double flag = 0.0;
    if (nunc > 0) {
      if ((etop - mid) / kt >= 80.0)
        sm += nunc * c80;
      else if (sm < nelec)
        flag = 1.0;
    }
    if (lane == 0) {
      sh.VtV[0][wid] = sm;
      sh.VtV[1][wid] = flag;
    }
    __syncthreads();
    int j = NW;
    for (int q = NW - 1; q >= 0; --q)
      if (sh.VtV[0][q] >= nelec) j = q;
    for (int q = 0; q < NW; ++q)
      if (sh.VtV[1][q] != 0.0) amb = true;
    const double nlo = (j == 0) ? lo : fmin(lo + (double)j * h, hi);
    const double nhi = (j == NW) ? hi : fmin(lo + (double)(j + 1) * h, hi);
    __syncthreads();
    if (amb || (nlo == lo && nhi == hi)) break;
    lo = nlo;
    hi = nhi;
  }
  const double mu = 0.5 * (lo + hi);
  if (!amb && nunc > 0 && !((etop - mu) / kt >= 80.0)) amb = true;
  double ts = 0.0;
  if (!amb) {
    double t = 0.0;
    for (int i = tid; i < N; i += NT) {
      const bool known = i < nneed || i == N - 1;
      const double f = known ? fo(eps[i], mu) : c80;
      occ[i] = f;
      const double nn = fmin(1.0 - 1e-16, fmax(1e-16, f / cap));
      t += cap * kt * (nn * log(nn) + (1.0 - nn) * log(1.0 - nn));
    }
    ts = block_sum(t, sh.red);
  }
  mu_out = mu;
  ts_out = ts;
  ambiguous = amb;
}

// A requested spin multiplicity fills the alpha and beta channels on their own,
// each orbital holding at most one electron per channel (src/electronic.rs:
// 3930-4045): occupation = alpha + beta, mu = their mean, TS = their sum.
// Every thread takes part; the results land in sh.scal[1] (mu), sh.scal[2]
// (TS) and sh.iscal[2] (ambiguous); `tmp` (N doubles) holds the beta channel.
// Kept out of line: inlined, this rarely used path changes how the compiler
// lays out the hot SCC loop (the closed-shell SCC stage measured 30% slower).
template <int NT>
__device__ __noinline__ void spin_channel_occupations(const double* eps, int N, int nneed, double nalpha,
                                                      double nbeta, double kt, double* occ, double* tmp,
                                                      SccShared& sh) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  auto channel = [&](double ne, double* o, double& fm, double& ft, bool& amb) {
    if (kt > 0.0 && ne > 0.0 && ne < (double)N) {
      fermi_cta<NT, 1>(eps, N, nneed, ne, kt, o, sh, fm, ft, amb);
    } else {
      if (wid == 0) {
        double m, t;
        bool a;
        fermi_warp<1>(eps, N, nneed, ne, kt, o, m, t, a);
        if (lane == 0) {
          sh.scal[4] = m;
          sh.scal[5] = t;
          sh.iscal[4] = a ? 1 : 0;
        }
      }
      __syncthreads();
      fm = sh.scal[4];
      ft = sh.scal[5];
      amb = sh.iscal[4] != 0;
      __syncthreads();
    }
  };
  double fa, ta, fb, tb;
  bool aa, ab;
  channel(nalpha, occ, fa, ta, aa);
  channel(nbeta, tmp, fb, tb, ab);
  for (int i = tid; i < N; i += NT) occ[i] += tmp[i];
  if (tid == 0) {
    sh.scal[1] = 0.5 * (fa + fb);
    sh.scal[2] = ta + tb;
    sh.iscal[2] = (aa || ab) ? 1 : 0;
  }
  __syncthreads();
}

// Z := Q Z for the first ncol columns, Q = H_0 ... H_{N-3}, applied in blocks of
// kBackNB reflectors as Q_b = I - V T V^T (compact WY, forward direction).
template <int NT>
__device__ void back_transform(const double* A, int lda, const double* tau, int N, double* Z, int ldz, int ncol,
                               double* W1, double* W2, SccShared& sh) {
  constexpr int NW = NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nref = N - 2;
  if (nref <= 0 || ncol <= 0) return;
  for (int kb = ((nref - 1) / kBackNB) * kBackNB; kb >= 0; kb -= kBackNB) {
    const int nb = min(kBackNB, nref - kb);
    // V^T V, one thread per pair i < j (rows >= kb + j + 1 hold both reflectors)
    for (int p = tid; p < nb * (nb - 1) / 2; p += NT) {
      int i = 0, rem = p;
      while (rem >= nb - 1 - i) {
        rem -= nb - 1 - i;
        ++i;
      }
      const int j = i + 1 + rem;
      const double* vi = A + (long long)(kb + i) * lda;
      const double* vj = A + (long long)(kb + j) * lda;
      double s0 = 0.0, s1 = 0.0;
      int r = kb + j + 1;
      for (; r + 1 < N; r += 2) {
        s0 += vi[r] * vj[r];
        s1 += vi[r + 1] * vj[r + 1];
      }
      if (r < N) s0 += vi[r] * vj[r];
      sh.VtV[i][j] = s0 + s1;
    }
    __syncthreads();
    if (wid == 0) {  // T upper triangular: T_jj = tau_j, T[0:j,j] = -tau_j T[0:j,0:j] V^T v_j
      for (int j = 0; j < nb; ++j) {
        const double tj = tau[kb + j];
        if (lane < j) {
          double s = 0.0;
          for (int l = lane; l < j; ++l) s += sh.Tm[lane][l] * sh.VtV[l][j];
          sh.Tm[lane][j] = -tj * s;
        }
        if (lane == j) sh.Tm[j][j] = tj;
        __syncwarp();
      }
    }
    // W1 = V^T Z on the FP64 tensor cores: pairs of 8x8 tiles of (reflector
    // j, column c) sharing the reflector fragment, k over the rows r;
    // reflector j has entries r > kb + j
    {
      const int g = lane >> 2, t4 = lane & 3;
      const int TC = (ncol + 7) >> 3, TJ = (nb + 7) >> 3, TC2 = (TC + 1) >> 1;
      for (int tile = wid; tile < TJ * TC2; tile += NW) {
        const int JT = tile / TC2, CT = 2 * (tile - JT * TC2);
        const int j = JT * 8 + g, cb0 = CT * 8 + g, cb1 = cb0 + 8;
        const bool jok = j < nb, ok0 = cb0 < ncol, ok1 = cb1 < ncol;
        const double* vj = A + (long long)(kb + (jok ? j : 0)) * lda;
        double d00 = 0.0, d01 = 0.0, d10 = 0.0, d11 = 0.0;
#pragma unroll 4
        for (int r0 = kb + 1; r0 < N; r0 += 4) {
          const int r = r0 + t4;
          const bool rin = r < N;
          const double* zr = Z + (long long)(rin ? r : 0) * ldz;
          const double a = (jok && rin && r > kb + j) ? vj[r] : 0.0;
          const double b0 = (rin && ok0) ? zr[cb0] : 0.0;
          const double b1 = (rin && ok1) ? zr[cb1] : 0.0;
          dmma_m8n8k4(d00, d01, a, b0);
          dmma_m8n8k4(d10, d11, a, b1);
        }
        const int cc = CT * 8 + 2 * t4;
        if (jok) {
          double* w1 = W1 + j * ncol;
          if (cc < ncol) w1[cc] = d00;
          if (cc + 1 < ncol) w1[cc + 1] = d01;
          if (cc + 8 < ncol) w1[cc + 8] = d10;
          if (cc + 9 < ncol) w1[cc + 9] = d11;
        }
      }
    }
    __syncthreads();
    for (int idx = tid; idx < nb * ncol; idx += NT) {
      const int j = idx / ncol, c = idx - j * ncol;
      double s = 0.0;
      for (int l = j; l < nb; ++l) s += sh.Tm[j][l] * W1[l * ncol + c];
      W2[j * ncol + c] = s;
    }
    __syncthreads();
    // Z -= V W2 on the FP64 tensor cores: pairs of 8x8 tiles of (row r,
    // column c) sharing the reflector fragment, starting from Z, k over the
    // reflectors j
    {
      const int g = lane >> 2, t4 = lane & 3;
      const int TC = (ncol + 7) >> 3, TR = (N - kb - 1 + 7) >> 3, TC2 = (TC + 1) >> 1;
      for (int tile = wid; tile < TR * TC2; tile += NW) {
        const int RT = tile / TC2, CT = 2 * (tile - RT * TC2);
        const int r = kb + 1 + RT * 8 + g, cb0 = CT * 8 + g, cb1 = cb0 + 8, cc = CT * 8 + 2 * t4;
        const bool rok = r < N, ok0 = cb0 < ncol, ok1 = cb1 < ncol;
        double* zr = Z + (long long)(rok ? r : 0) * ldz;
        double d00 = (rok && cc < ncol) ? zr[cc] : 0.0;
        double d01 = (rok && cc + 1 < ncol) ? zr[cc + 1] : 0.0;
        double d10 = (rok && cc + 8 < ncol) ? zr[cc + 8] : 0.0;
        double d11 = (rok && cc + 9 < ncol) ? zr[cc + 9] : 0.0;
#pragma unroll 4
        for (int j0 = 0; j0 < nb; j0 += 4) {
          const int j = j0 + t4;
          const bool jok = j < nb;
          const double a = (rok && jok && r > kb + j) ? -A[(long long)(kb + j) * lda + r] : 0.0;
          const double* w2 = W2 + (jok ? j : 0) * ncol;
          const double b0 = (jok && ok0) ? w2[cb0] : 0.0;
          const double b1 = (jok && ok1) ? w2[cb1] : 0.0;
          dmma_m8n8k4(d00, d01, a, b0);
          dmma_m8n8k4(d10, d11, a, b1);
        }
        if (rok) {
          if (cc < ncol) zr[cc] = d00;
          if (cc + 1 < ncol) zr[cc + 1] = d01;
          if (cc + 8 < ncol) zr[cc + 8] = d10;
          if (cc + 9 < ncol) zr[cc + 9] = d11;
        }
      }
    }
    __syncthreads();
  }
}

// Index tables of one molecule (one thread): shell -> atom, shell -> index
// within its atom, shell -> first AO, AO -> shell, atom -> first shell.
__device__ void build_index_tables(const Batch& B, const Model& M, int a0, int nat, int* sh_atom, int* sh_k,
                                   int* sh_ao0, int* ao_sh, int* atom_sh) {
  int s = 0, o = 0;
  for (int a = 0; a < nat; ++a) {
    const ElemTable& el = M.elem[B.z[a0 + a]];
    atom_sh[a] = s;
    for (int k = 0; k < el.nsh; ++k) {
      sh_atom[s + k] = a;
      sh_k[s + k] = k;
      sh_ao0[s + k] = o + el.ao_first[k];
      for (int q = 0; q < 2 * el.l[k] + 1; ++q) ao_sh[o + el.ao_first[k] + q] = s + k;
    }
    s += el.nsh;
    o += el.nao;
  }
  atom_sh[nat] = s;
}

// Per-molecule view shared by the SCC stages: sizes, offsets and the index
// tables (shell -> atom, shell -> shell index within its atom, shell -> first
// AO, AO -> shell, atom -> first shell), plus the molecule's Coulomb matrix.
struct MolCtx {
  int m, a0, nat, sh0, nsh, N;
  const int *sh_atom, *sh_k, *sh_ao0, *ao_sh, *atom_sh;
  const double* G;
};

// (1) Shell potential of the input charges (src/coulomb.rs:140-193):
// w.qat, w.vsh and the AO potential vao.
template <int NT>
__device__ void stage_potential(const Batch& B, const Model& M, const MolCtx& c, CtaWs& w, double* vao) {
  const int tid = threadIdx.x;
  const int a0 = c.a0, nat = c.nat, nsh = c.nsh, N = c.N;
  const int *sh_atom = c.sh_atom, *ao_sh = c.ao_sh, *atom_sh = c.atom_sh;
  const double* G = c.G;
  for (int a = tid; a < nat; a += NT) {
    double q = 0.0;
    for (int s = atom_sh[a]; s < atom_sh[a + 1]; ++s) q += w.qin[s];
    w.qat[a] = q;
  }
  __syncthreads();
  for (int i = tid; i < nsh; i += NT) {
    double v = 0.0;
    for (int j = 0; j < nsh; ++j) v += G[(long long)j * nsh + i] * w.qin[j];  // G symmetric: coalesced column
    const int a = sh_atom[i];
    const double qa = w.qat[a];
    v += qa * qa * M.elem[B.z[a0 + a]].gam3;
    w.vsh[i] = v;
  }
  __syncthreads();
  for (int i = tid; i < N; i += NT) vao[i] = w.vsh[ao_sh[i]];
  __syncthreads();
}

// (9) Output shell and atomic charges, electronic energy, second- and
// third-order energies and the charge rms (src/electronic.rs:2173-2191,
// :3160-3200); also the output potential w.vout.
template <int NT>
__device__ void stage_charges_energy(const Batch& B, const Model& M, const MolCtx& c, CtaWs& w, const double* pop,
                                     const double* occ, const double* eps, const double* vao, int nocc, SccShared& sh,
                                     double& e_el, double& e2, double& e3, double& rms) {
  const int tid = threadIdx.x;
  const int a0 = c.a0, nat = c.nat, nsh = c.nsh, N = c.N;
  const int *sh_atom = c.sh_atom, *sh_k = c.sh_k, *sh_ao0 = c.sh_ao0, *atom_sh = c.atom_sh;
  const double* G = c.G;
  for (int s = tid; s < nsh; s += NT) {
    const ElemTable& el = M.elem[B.z[a0 + sh_atom[s]]];
    const int k = sh_k[s];
    double p = 0.0;
    for (int q = 0; q < 2 * el.l[k] + 1; ++q) p += pop[sh_ao0[s] + q];
    w.qout[s] = el.refocc[k] - p;
  }
  double part = 0.0;
  for (int i = tid; i < N; i += NT) part += (i < nocc ? occ[i] * eps[i] : 0.0) + vao[i] * pop[i];
  e_el = block_sum(part, sh.red);
  for (int a = tid; a < nat; a += NT) {
    double q = 0.0;
    for (int s = atom_sh[a]; s < atom_sh[a + 1]; ++s) q += w.qout[s];
    w.qat[a] = q;
  }
  __syncthreads();
  double p2 = 0.0, p3 = 0.0, pr = 0.0;
  for (int i = tid; i < nsh; i += NT) {
    double v = 0.0;
    for (int j = 0; j < nsh; ++j) v += G[(long long)j * nsh + i] * w.qout[j];  // G symmetric: coalesced column
    p2 += w.qout[i] * v;
    const int a = sh_atom[i];
    const double qa = w.qat[a];
    const double g3 = M.elem[B.z[a0 + a]].gam3;
    w.vout[i] = v + qa * qa * g3;
    const double r = w.qout[i] - w.qin[i];
    pr += r * r;
  }
  for (int a = tid; a < nat; a += NT) {
    const double qa = w.qat[a];
    p3 += qa * qa * qa * M.elem[B.z[a0 + a]].gam3 / 3.0;
  }
  e2 = 0.5 * block_sum(p2, sh.red);
  e3 = block_sum(p3, sh.red);
  rms = nsh ? sqrt(block_sum(pr, sh.red) / nsh) : 0.0;
}

// (10) Charge mixing: modified Broyden (src/electronic.rs:3203-3309), linear
// damped step on the first iteration, a singular solve or an untrusted vector
// (:3311-3316, :3759-3761); the next input charges land in w.qin.
template <int NT>
__device__ void stage_mix(const SccOptions& opt, const MolCtx& c, CtaWs& w, int cap, int& bro_iter, SccShared& sh) {
  constexpr int NW = NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nsh = c.nsh;
  const double mixing = fmin(1.0, fmax(0.01, opt.mixing));
  const int memory = max(opt.broyden_size, 2);
  bool have_next = false;
  if (opt.broyden) {
    bro_iter += 1;
    if (bro_iter == 1) {
      for (int s = tid; s < nsh; s += NT) {
        const double r = w.qout[s] - w.qin[s];
        w.dqlast[s] = r;
        w.qlast[s] = w.qin[s];
        w.qnext[s] = w.qin[s] + mixing * r;
      }
      have_next = true;
      __syncthreads();
    } else {
      const int itn = bro_iter - 1;
      const int it1 = (itn - 1) % memory;
      const int slot = it1 % cap;
      double pn = 0.0, pd = 0.0;
      for (int s = tid; s < nsh; s += NT) {
        const double r = w.qout[s] - w.qin[s];
        pn += r * r;
        const double dfv = r - w.dqlast[s];
        pd += dfv * dfv;
      }
      const double dqn = sqrt(block_sum(pn, sh.red));
      const double dfn = sqrt(block_sum(pd, sh.red));
      const double inv = 1.0 / fmax(dfn, DBL_EPSILON);
      double* dfs = w.df + (long long)slot * nsh;
      double* us = w.u + (long long)slot * nsh;
      for (int s = tid; s < nsh; s += NT) {
        const double r = w.qout[s] - w.qin[s];
        const double dfv = (r - w.dqlast[s]) * inv;
        dfs[s] = dfv;
        us[s] = mixing * dfv + inv * (w.qin[s] - w.qlast[s]);
      }
      if (tid == 0) {
        double om = dqn > 0.01 / 100000.0 ? 0.01 / dqn : 100000.0;
        if (om < 1.0) om = 1.0;
        w.omega[slot] = om;
      }
      __syncthreads();
      const int start = itn > memory ? itn - memory + 1 : 1;
      const int mact = itn - start + 1;
      // dot products df_new . df_j for every active slot, and c_j = omega_j df_j . dq
      for (int r = wid; r < mact; r += NW) {
        const int sj = ((start + r - 1) % memory) % cap;
        const double* dj = w.df + (long long)sj * nsh;
        double s1 = 0.0, s2 = 0.0;
        for (int s = lane; s < nsh; s += 32) {
          s1 += dfs[s] * dj[s];
          s2 += dj[s] * (w.qout[s] - w.qin[s]);
        }
        s1 = warp_sum(s1);
        s2 = warp_sum(s2);
        if (lane == 0) {
          w.dots[(long long)slot * cap + sj] = s1;
          w.dots[(long long)sj * cap + slot] = s1;
          w.cvec[r] = s2;
        }
      }
      __syncthreads();
      for (int idx = tid; idx < mact * mact; idx += NT) {
        const int r = idx / mact, c = idx % mact;
        const int si = ((start + r - 1) % memory) % cap, sj = ((start + c - 1) % memory) % cap;
        double b = w.omega[si] * w.omega[sj] * w.dots[(long long)si * cap + sj];
        if (r == c) b += 0.01 * 0.01;
        w.beta[(long long)r * mact + c] = b;
      }
      for (int r = tid; r < mact; r += NT) {
        const int si = ((start + r - 1) % memory) % cap;
        w.cvec[r] *= w.omega[si];
      }
      __syncthreads();
      // Gauss-Jordan with partial pivoting (src/electronic.rs:3767-3806)
      bool ok = true;
      for (int col = 0; col < mact; ++col) {
        if (tid == 0) {
          int piv = col;
          double pabs = fabs(w.beta[(long long)col * mact + col]);
          for (int r = col + 1; r < mact; ++r) {
            const double v = fabs(w.beta[(long long)r * mact + col]);
            if (v > pabs) {
              piv = r;
              pabs = v;
            }
          }
          sh.iscal[1] = (pabs < 1e-18) ? -1 : piv;
        }
        __syncthreads();
        const int piv = sh.iscal[1];
        if (piv < 0) {
          ok = false;
          break;
        }
        if (piv != col) {
          for (int j = tid; j < mact; j += NT) {
            const double t = w.beta[(long long)piv * mact + j];
            w.beta[(long long)piv * mact + j] = w.beta[(long long)col * mact + j];
            w.beta[(long long)col * mact + j] = t;
          }
          if (tid == 0) {
            const double t = w.cvec[piv];
            w.cvec[piv] = w.cvec[col];
            w.cvec[col] = t;
          }
          __syncthreads();
        }
        const double dg = w.beta[(long long)col * mact + col];
        __syncthreads();
        for (int j = col + tid; j < mact; j += NT) w.beta[(long long)col * mact + j] /= dg;
        if (tid == 0) w.cvec[col] /= dg;
        __syncthreads();
        for (int idx = tid; idx < mact * (mact - col); idx += NT) {
          const int r = idx / (mact - col), j = col + idx % (mact - col);
          if (r == col) continue;
          const double f = w.beta[(long long)r * mact + col];
          if (f == 0.0 || j == col) continue;
          w.beta[(long long)r * mact + j] -= f * w.beta[(long long)col * mact + j];
        }
        for (int r = tid; r < mact; r += NT) {
          if (r == col) continue;
          const double f = w.beta[(long long)r * mact + col];
          if (f != 0.0) w.cvec[r] -= f * w.cvec[col];
        }
        __syncthreads();
        for (int r = tid; r < mact; r += NT)
          if (r != col) w.beta[(long long)r * mact + col] = 0.0;
        __syncthreads();
      }
      if (ok) {
        for (int s = tid; s < nsh; s += NT) {
          const double r = w.qout[s] - w.qin[s];
          double qn = w.qin[s] + mixing * r;
          for (int rr = 0; rr < mact; ++rr) {
            const int si = ((start + rr - 1) % memory) % cap;
            qn -= w.omega[si] * w.cvec[rr] * w.u[(long long)si * nsh + s];
          }
          w.qnext[s] = qn;
          w.dqlast[s] = r;
          w.qlast[s] = w.qin[s];
        }
        have_next = true;
      }
      __syncthreads();
    }
    if (have_next) {  // trusted_charge_vector (src/electronic.rs:3759-3761)
      int bad = 0;
      for (int s = tid; s < nsh; s += NT)
        if (!isfinite(w.qnext[s]) || fabs(w.qnext[s]) >= 10.0) bad = 1;
      if (block_max((double)bad, sh.red) > 0.0) have_next = false;
    }
  }
  if (!have_next)
    for (int s = tid; s < nsh; s += NT) w.qnext[s] = w.qin[s] + mixing * (w.qout[s] - w.qin[s]);
  __syncthreads();
  for (int s = tid; s < nsh; s += NT) w.qin[s] = w.qnext[s];
}

// Results of a finished SCC: energy terms, iterations, status, Fermi level,
// Mulliken dipole, shell charges and potential, atomic charges.
template <int NT>
__device__ void stage_results(const Batch& B, const MolCtx& c, CtaWs& w, int iter, bool converged, double e_el,
                              double e2, double e3, double ts, double mu) {
  const int tid = threadIdx.x;
  const int a0 = c.a0, nat = c.nat, nsh = c.nsh;
  const int m = c.m, sh0 = c.sh0;
  if (tid == 0) {
    double* t = B.terms + (long long)m * kTerms;
    const double erep = t[2], edisp = t[7], ehal = t[8];
    const double total_internal = e_el + e2 + e3 + erep + edisp + ehal;
    t[0] = total_internal + ts;
    t[1] = total_internal;
    t[3] = e_el;
    t[4] = e2;
    t[5] = e3;
    t[14] = ts;
    B.iterations[m] = iter;
    B.status[m] = converged ? kOk : kErrSccNotConverged;
    B.fermi[m] = mu;
    double dx = 0, dy = 0, dz = 0;
    for (int a = 0; a < nat; ++a) {
      dx += w.qat[a] * B.xyz[3 * (a0 + a)];
      dy += w.qat[a] * B.xyz[3 * (a0 + a) + 1];
      dz += w.qat[a] * B.xyz[3 * (a0 + a) + 2];
    }
    B.dipole[3 * m] = dx;
    B.dipole[3 * m + 1] = dy;
    B.dipole[3 * m + 2] = dz;
  }
  for (int s = tid; s < nsh; s += NT) {
    B.shell_q[sh0 + s] = w.qout[s];
    B.shell_pot[sh0 + s] = w.vout[s];
    if (B.shell_pot_in) B.shell_pot_in[sh0 + s] = w.vsh[s];
  }
  for (int a = tid; a < nat; a += NT) B.atom_q[a0 + a] = w.qat[a];
}

template <int NT, bool Robust>
__device__ void scc_molecule(const Batch& B, const Model& M, const SccOptions& opt, const SccLaunch& SL, int m,
                             SccShared& sh, int* sh_atom, int* sh_k, int* ao_sh, int* atom_sh, int* sh_ao0,
                             double* vec, double* As, long long as_cap) {
  constexpr int NW = NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int a0 = B.atom_off[m], nat = B.atom_off[m + 1] - a0;
  const int sh0 = B.shell_off[m], nsh = B.shell_off[m + 1] - sh0;
  const int N = B.ao_off[m + 1] - B.ao_off[m];
  const long long mo = B.mat_off[m];
  const double* S = B.S + mo;
  const double* H0 = B.H0 + mo;
  CtaWs w = cta_ws(SL.ws + (long long)blockIdx.x * SL.ws_stride, SL.maxn, SL.maxnsh, SL.cap);
  double* L = w.L;
  double* Li = w.Li;
  double* Hp = w.Hp;
  double* Z = w.Z;
  double* C = w.C;
  double* iw = w.iw;
  const double* G = B.gam + B.gam_off[m];
  const bool a_shared = (long long)N * work_lda(N) <= as_cap;  // shared memory when the launch gave room
  const int lda = a_shared ? work_lda(N) : work_lda_global(N);
  double* A = a_shared ? As : w.A;
  double* d = vec;
  double* e = vec + N;
  double* tau = vec + 2 * N;
  double* eps = vec + 3 * N;
  double* occ = vec + 4 * N;
  double* pop = vec + 5 * N;
  double* vao = vec + 6 * N;
  double* pvec = vec + 7 * N;
  double* esq = vec + 8 * N;
  const int cap = SL.cap;

  // ---- index tables
  if (tid == 0) {
    build_index_tables(B, M, a0, nat, sh_atom, sh_k, sh_ao0, ao_sh, atom_sh);
    sh.iscal[0] = kOk;
  }
  __syncthreads();

  StageClock clk(B.stage_cycles);
  const MolCtx mc{m, a0, nat, sh0, nsh, N, sh_atom, sh_k, sh_ao0, ao_sh, atom_sh, G};
  // ---- Cholesky S = L L^T, left-looking over panels of 8 columns: the
  // panel minus (its rows of L) x (the panel's rows of L)^T over the finished
  // columns on the FP64 tensor cores, the 8x8 diagonal block by one thread
  // (registers; its factor and reciprocal pivots staged in shared memory),
  // then the rows below by a triangular solve, one thread per row.
  for (long long i = tid; i < (long long)N * N; i += NT) L[i] = S[i];
  __syncthreads();
  {
    const int g = lane >> 2, t4 = lane & 3;
    double(*Ld)[kBackNB] = sh.Tm;  // free until the first back-transformation
    for (int c0 = 0; c0 < N; c0 += 8) {
      const int nbc = min(8, N - c0);
      if (c0 > 0) {
        const int TR = (N - c0 + 7) >> 3;
        const bool jok = g < nbc;
        const double* lj = L + (long long)(jok ? c0 + g : 0) * N;
        for (int RT = wid; RT < TR; RT += NW) {
          const int i = c0 + RT * 8 + g;
          const bool iok = i < N;
          const double* li = L + (long long)(iok ? i : 0) * N;
          double d0 = 0.0, d1 = 0.0;
#pragma unroll 4
          for (int k0 = 0; k0 < c0; k0 += 4) {
            const int k = k0 + t4;
            dmma_m8n8k4(d0, d1, iok ? li[k] : 0.0, jok ? lj[k] : 0.0);
          }
          if (iok) {
            double* out = L + (long long)i * N + c0 + 2 * t4;
            if (2 * t4 < nbc) out[0] -= d0;
            if (2 * t4 + 1 < nbc) out[1] -= d1;
          }
        }
        __syncthreads();
      }
      if (tid == 0) {
        double D[8][8];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j <= i; ++j) D[i][j] = (i < nbc) ? L[(long long)(c0 + i) * N + c0 + j] : (i == j ? 1.0 : 0.0);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          // the reference rejects overlaps with an eigenvalue <= eigen_tolerance (1e-12)
          if (j < nbc && !(D[j][j] > 1e-12)) sh.iscal[0] = kErrInvalidInput;
          const double r = sqrt(fmax(D[j][j], 1e-300));
          const double inv = 1.0 / r;
          D[j][j] = r;
          Ld[j][8] = inv;
#pragma unroll
          for (int i = j + 1; i < 8; ++i) D[i][j] *= inv;
#pragma unroll
          for (int k = j + 1; k < 8; ++k)
#pragma unroll
            for (int i = k; i < 8; ++i) D[i][k] -= D[i][j] * D[k][j];
        }
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j <= i; ++j) {
            Ld[i][j] = D[i][j];
            if (i < nbc) L[(long long)(c0 + i) * N + c0 + j] = D[i][j];
          }
      }
      __syncthreads();
      for (int i = c0 + 8 + tid; i < N; i += NT) {  // rows below: x L_dd^T = row
        double* row = L + (long long)i * N + c0;
        double x[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = row[j];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
#pragma unroll
          for (int k = 0; k < j; ++k) x[j] -= x[k] * Ld[j][k];
          x[j] *= Ld[j][8];
          row[j] = x[j];
        }
      }
      __syncthreads();
    }
  }
  if (sh.iscal[0] != kOk) {
    if (tid == 0) {
      B.status[m] = sh.iscal[0];
      B.iterations[m] = 0;
    }
    return;
  }
  for (int i = wid; i < N; i += NW)
    for (int j = i + 1 + lane; j < N; j += 32) L[(long long)i * N + j] = 0.0;
  __syncthreads();
  clk.mark(kStChol);
  // L^-1 by forward substitution L X = I, one thread per column.  The lanes
  // of a warp step through the rows together, so row i of L is a broadcast
  // and the reads of X[k][c] coalesce; a warp starts at its first column
  // (rows above it are zeros in all of its columns), four partial sums.
  for (int c0 = 0; c0 < N; c0 += NT) {
    const int c = c0 + tid;
    const int cc = min(c, N - 1);
    const int kw = min(N, c0 + (tid & ~31));  // the warp's first column
    if (c < N)
      for (int i = 0; i < kw; ++i) Li[(long long)i * N + c] = 0.0;
    for (int i = kw; i < N; ++i) {
      const double* li = L + (long long)i * N;
      double s0 = (i == c) ? 1.0 : 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
      int k = kw;
      for (; k + 3 < i; k += 4) {
        s0 -= li[k] * Li[(long long)k * N + cc];
        s1 -= li[k + 1] * Li[(long long)(k + 1) * N + cc];
        s2 -= li[k + 2] * Li[(long long)(k + 2) * N + cc];
        s3 -= li[k + 3] * Li[(long long)(k + 3) * N + cc];
      }
      for (; k < i; ++k) s0 -= li[k] * Li[(long long)k * N + cc];
      if (c < N) Li[(long long)i * N + c] = ((s0 + s1) + (s2 + s3)) / li[i];
    }
  }
  __syncthreads();
  clk.mark(kStLinv);
  // H0' = L^-1 H0 L^-T on the FP64 tensor cores: U = L^-1 H0 in 8x8 tiles
  // (row i of L^-1 ends at the diagonal), then H0' = U (L^-1)^T for the tiles
  // on and below the diagonal, each written to both triangles so that H0' is
  // exactly symmetric.  U uses the global work matrix, free until the first
  // iteration.  Each warp owns whole tiles; lanes beyond N load zeros.
  {
    double* U = w.A;
    const int T = (N + 7) >> 3;
    const int g = lane >> 2, t4 = lane & 3;
    for (int tile = wid; tile < T * T; tile += NW) {
      const int I = tile / T, J = tile - I * T;
      const int i = I * 8 + g, jb = J * 8 + g;
      const int kend = min(N, I * 8 + 8);
      double d0 = 0.0, d1 = 0.0;
#pragma unroll 4
      for (int k0 = 0; k0 < kend; k0 += 4) {
        const int k = k0 + t4;
        const double a = (i < N && k < N) ? Li[(long long)i * N + k] : 0.0;
        const double b = (k < N && jb < N) ? H0[(long long)k * N + jb] : 0.0;
        dmma_m8n8k4(d0, d1, a, b);
      }
      const int jc = J * 8 + 2 * t4;
      if (i < N && jc < N) U[(long long)i * N + jc] = d0;
      if (i < N && jc + 1 < N) U[(long long)i * N + jc + 1] = d1;
    }
    __syncthreads();
    for (int tile = wid; tile < T * (T + 1) / 2; tile += NW) {
      int I = 0;
      while ((I + 1) * (I + 2) / 2 <= tile) ++I;
      const int J = tile - I * (I + 1) / 2;
      const int i = I * 8 + g, jb = J * 8 + g;
      const int kend = min(N, J * 8 + 8);
      double d0 = 0.0, d1 = 0.0;
#pragma unroll 4
      for (int k0 = 0; k0 < kend; k0 += 4) {
        const int k = k0 + t4;
        const double a = (i < N && k < N) ? U[(long long)i * N + k] : 0.0;
        const double b = (jb < N && k < N) ? Li[(long long)jb * N + k] : 0.0;
        dmma_m8n8k4(d0, d1, a, b);
      }
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int j = J * 8 + 2 * t4 + c;
        if (i < N && j < N && (I != J || j <= i)) {
          const double v = c ? d1 : d0;
          Hp[(long long)i * N + j] = v;
          Hp[(long long)j * N + i] = v;
        }
      }
    }
    __syncthreads();
  }

  // ---- SCC state
  double nref = 0.0;
  for (int s = 0; s < nsh; ++s) nref += M.elem[B.z[a0 + sh_atom[s]]].refocc[sh_k[s]];
  const double nelec = nref - B.charge[m];
  // a requested spin multiplicity: alpha and beta electron counts (validated on the host)
  const bool spin = opt.spin_mult > 0;
  const double nalpha = spin ? 0.5 * (rint(nelec) + (opt.spin_mult - 1)) : 0.0;
  const double nbeta = spin ? 0.5 * (rint(nelec) - (opt.spin_mult - 1)) : 0.0;
  const int nneed0 = min(N, max(1, (int)ceil(spin ? nalpha : 0.5 * nelec) + 8));
  int bro_iter = 0;
  double last_e = 0.0;
  bool have_e = false;
  bool converged = false;
  int nneed_last = nneed0;  // eigenvalues 0..nneed_last-1 and N-1 of the last diagonalisation are known
  int iter = 0;
  int nocc = 0;
  double e_el = 0.0, e2 = 0.0, e3 = 0.0, ts = 0.0, mu = 0.0, rms = 0.0;
  // The reference's fallback ladder (src/electronic.rs:1390-1447): rung 0 is
  // the requested options (the main kernel); rungs 1-3 (the Robust kernel,
  // for molecules rung 0 left unconverged) restart from the initial charges
  // with linear mixing 0.2 and a level shift of max(requested, 0.2 Eh), then
  // 0.1 / max(requested, 0.1), then Broyden at T_el >= 3000 K without shift.
  // A requested level shift sends every molecule to the Robust kernel, which
  // then starts at rung 0 (the main kernel carries no level-shift code).
  const int rung_first = Robust ? (opt.level_shift != 0.0 ? 0 : 1) : 0, rung_last = Robust ? 3 : 0;
  [[maybe_unused]] int rung_used = rung_first;  // the rung whose SCC converged (reported by the ladder kernel)
  for (int rung = rung_first; rung <= rung_last && !converged; ++rung) {
  rung_used = rung;
  SccOptions ro = opt;
  double lshift = Robust ? opt.level_shift : 0.0;
  if (rung == 1 || rung == 2) {
    ro.broyden = 0;
    ro.mixing = rung == 1 ? 0.20 : 0.10;
    lshift = fmax(opt.level_shift, rung == 1 ? 0.20 : 0.10);
    ro.max_scc = max(opt.max_scc, 800);
  } else if (rung == 3) {
    ro.etemp = fmax(opt.etemp, 3000.0);
    ro.max_scc = max(opt.max_scc, 250);
    lshift = 0.0;
  }
  const double kt = fmax(ro.etemp, 0.0) * kBoltzmann;
  for (int s = tid; s < nsh; s += NT) w.qin[s] = B.init_q ? B.init_q[sh0 + s] : 0.0;
  bro_iter = 0;
  last_e = 0.0;
  have_e = false;
  bool have_prev = false;  // a previous density to shift against (rungs with a level shift)
  __syncthreads();
  clk.mark(kStPrologue);

  for (iter = 1; iter <= ro.max_scc; ++iter) {
    // (1) shell potential from the input charges
    stage_potential<NT>(B, M, mc, w, vao);
    // (2) F' = H0' - 1/2 (M + M^T) with M = L^-1 diag(v) L lower triangular,
    //     so F'_ij = H0'_ij - M_ij / 2 below the diagonal and H0'_ii - M_ii on
    //     it.  M on the FP64 tensor cores: pairs of 8x8 tiles (I, J), (I, J+1)
    //     on and below the diagonal sharing the L^-1 fragment, k from the
    //     pair's first column to its last row (the entries of L above the
    //     diagonal are stored zeros, so the second tile's extra k add nothing).
    {
      const int T = (N + 7) >> 3;
      const int g = lane >> 2, t4 = lane & 3;
      int I = 0, base = 0;  // base: pairs of the rows of tiles before I
      for (int task = wid;; task += NW) {
        while (I < T && task >= base + (I >> 1) + 1) {
          base += (I >> 1) + 1;
          ++I;
        }
        if (I >= T) break;
        const int J = 2 * (task - base);
        const bool two = J + 1 <= I;
        const int i = I * 8 + g, jb0 = J * 8 + g, jb1 = jb0 + 8;
        const bool iok = i < N;
        const double* lirow = Li + (long long)(iok ? i : 0) * N;
        const int kend = min(N, I * 8 + 8);
        double d00 = 0.0, d01 = 0.0, d10 = 0.0, d11 = 0.0;
#pragma unroll 4
        for (int k0 = J * 8; k0 < kend; k0 += 4) {
          const int k = k0 + t4;
          const bool kin = k < N;
          const double* lk = L + (long long)(kin ? k : 0) * N;
          const double vk = kin ? vao[k] : 0.0;
          const double a = (iok && kin) ? lirow[k] : 0.0;
          const double b0 = (kin && jb0 < N) ? lk[jb0] * vk : 0.0;
          dmma_m8n8k4(d00, d01, a, b0);
          if (two) {
            const double b1 = (kin && jb1 < N) ? lk[jb1] * vk : 0.0;
            dmma_m8n8k4(d10, d11, a, b1);
          }
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int j = J * 8 + 2 * t4 + (c & 1) + (c >> 1) * 8;
          if (iok && j <= i && (c < 2 || two)) {
            const double mv = c == 0 ? d00 : c == 1 ? d01 : c == 2 ? d10 : d11;
            const double f = Hp[(long long)i * N + j] - (i == j ? mv : 0.5 * mv);
            A[(long long)i * lda + j] = f;
            A[(long long)j * lda + i] = f;
          }
        }
      }
    }
    __syncthreads();
    if (Robust && lshift != 0.0 && have_prev) {
      // level shift F += lshift (S - S P_prev S / 2) (src/electronic.rs:2125-2137);
      // in the orthonormal basis F' += lshift (I - Z f Z^T / 2) with the
      // previous iteration's eigenvectors Z and occupations f
      for (long long idx = tid; idx < (long long)N * N; idx += NT) {
        const int i = (int)(idx / N), j = (int)(idx % N);
        if (j > i) continue;
        double sp = 0.0;
        for (int k = 0; k < nocc; ++k) sp += occ[k] * Z[(long long)i * N + k] * Z[(long long)j * N + k];
        const double val = lshift * ((i == j ? 1.0 : 0.0) - 0.5 * sp);
        A[(long long)i * lda + j] += val;
        if (i != j) A[(long long)j * lda + i] += val;
      }
      __syncthreads();
    }
    clk.mark(kStFock);
    // (3) Householder tridiagonalisation
    if constexpr (NT == 128) {
      if (N <= 32 * 6 + 1 && !a_shared)  // e^2 is formed after the reduction, so its slot is the reduction's scratch
        tridiagonalize_blocked<NT>(A, lda, N, d, e, tau, pvec, esq, w.W1, sh);
      else
        tridiagonalize<NT>(A, lda, N, d, e, tau, pvec, sh);
    } else {
      tridiagonalize<NT>(A, lda, N, d, e, tau, pvec, sh);
    }
    clk.mark(kStTridiag);
    // (4) eigenvalues needed by the occupations
    double gl = INFINITY, gu = -INFINITY, onenrm = 0.0, emax2 = 0.0;
    for (int i = tid; i < N; i += NT) {
      const double off = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < N - 1 ? fabs(e[i]) : 0.0);
      gl = fmin(gl, d[i] - off);
      gu = fmax(gu, d[i] + off);
      onenrm = fmax(onenrm, fabs(d[i]) + off);
      if (i < N - 1) {
        esq[i] = e[i] * e[i];
        emax2 = fmax(emax2, esq[i]);
      }
    }
    gl = -block_max(-gl, sh.red);
    gu = block_max(gu, sh.red);
    onenrm = block_max(onenrm, sh.red);
    emax2 = block_max(emax2, sh.red);
    const double pivmin = DBL_MIN * fmax(1.0, emax2);
    {
      const double span = gu - gl;
      gl -= 2.1 * DBL_EPSILON * fabs(gl) + 4.0 * DBL_EPSILON * span + pivmin;
      gu += 2.1 * DBL_EPSILON * fabs(gu) + 4.0 * DBL_EPSILON * span + pivmin;
    }
    int nneed = nneed0;
    for (int attempt = 0; attempt < 2; ++attempt) {
      // from the previous iteration's eigenvalues once this rung has one
      eigenvalues<NT>(d, esq, N, nneed, gl, gu, pivmin, 4.0 * DBL_EPSILON * onenrm, eps,
                      (iter > 1 && attempt == 0) ? nneed_last : 0);
      clk.mark(kStEigval);
      // (5) occupations (src/electronic.rs:3815-3921)
      if (spin) {
        spin_channel_occupations<NT>(eps, N, nneed, nalpha, nbeta, kt, occ, pop, sh);
      } else if (kt > 0.0 && nelec > 0.0 && nelec < 2.0 * N) {
        double fm, ft;
        bool amb;
        fermi_cta<NT, 2>(eps, N, nneed, nelec, kt, occ, sh, fm, ft, amb);
        if (tid == 0) {
          sh.scal[1] = fm;
          sh.scal[2] = ft;
          sh.iscal[2] = amb ? 1 : 0;
        }
      } else if (wid == 0) {  // aufbau and the empty / full limits
        double fm, ft;
        bool amb;
        fermi_warp<2>(eps, N, nneed, nelec, kt, occ, fm, ft, amb);
        if (lane == 0) {
          sh.scal[1] = fm;
          sh.scal[2] = ft;
          sh.iscal[2] = amb ? 1 : 0;
        }
      }
      __syncthreads();
      clk.mark(kStFermi);
      if (!sh.iscal[2] || nneed == N) break;
      nneed = N;
    }
    mu = sh.scal[1];
    ts = sh.scal[2];
    nneed_last = nneed;
    // number of orbitals whose occupation matters at FP64 resolution
    int nocc_loc = 0;
    for (int i = tid; i < N; i += NT)
      if ((i < nneed || i == N - 1) && occ[i] > 1e-30) nocc_loc = max(nocc_loc, i + 1);
    nocc = (int)block_max((double)nocc_loc, sh.red);
    // (6) inverse iteration for the occupied eigenvectors (columns of Z)
    const double ortol = 1e-5 * onenrm;
    const double tiny = DBL_EPSILON * fmax(onenrm, 1e-300);
    for (int j = tid; j < nocc; j += NT) {
      const bool start = (j == 0) || (eps[j] - eps[j - 1] > ortol);
      if (!start) continue;
      int jend = j + 1;
      while (jend < nocc && eps[jend] - eps[jend - 1] <= ortol) ++jend;
      double* ws = iw + j;  // column j of the interleaved factor arrays
      double lam_prev = -INFINITY;
      for (int jj = j; jj < jend; ++jj) {
        double lam = eps[jj];
        const double pert = 10.0 * DBL_EPSILON * fmax(fabs(lam), onenrm);
        if (jj > j && lam - lam_prev < pert) lam = lam_prev + pert;
        lam_prev = lam;
        double* x = Z + jj;  // column jj, stride N
        if (jend - j == 1) {
          // isolated: the start vector's forward elimination runs with the
          // factorisation, the two solves are not normalised in between
          // (growth below 1e40), and the second one returns |x|^2
          const double cur = tri_factor_rhs(d, e, N, lam, tiny, ws, N, x, N, (unsigned)jj);
          tri_back(ws, N, N, x, N, cur);
          const double nrm = tri_solve(ws, N, N, x, N);
          const double inv = 1.0 / sqrt(fmax(nrm, 1e-300));
#pragma unroll 8
          for (int i = 0; i < N; ++i) x[(long long)i * N] *= inv;
          continue;
        }
        tri_factor(d, e, N, lam, tiny, ws, N);
#pragma unroll 4
        for (int i = 0; i < N; ++i) x[(long long)i * N] = hash_unit(i, jj) + 1e-3;
        const int nit = 4;
        for (int it = 0; it < nit; ++it) {
          tri_solve(ws, N, N, x, N);
          for (int q = j; q < jj; ++q) {  // modified Gram-Schmidt inside the cluster
            double dot = 0.0;
            for (int i = 0; i < N; ++i) dot += Z[(long long)i * N + q] * x[(long long)i * N];
            for (int i = 0; i < N; ++i) x[(long long)i * N] -= dot * Z[(long long)i * N + q];
          }
          double nrm = 0.0;
#pragma unroll 8
          for (int i = 0; i < N; ++i) nrm += x[(long long)i * N] * x[(long long)i * N];
          const double inv = 1.0 / sqrt(fmax(nrm, 1e-300));
#pragma unroll 8
          for (int i = 0; i < N; ++i) x[(long long)i * N] *= inv;
        }
      }
    }
    __syncthreads();
    clk.mark(kStInvIter);
    // (7) back-transformation Z := Q Z
    back_transform<NT>(A, lda, tau, N, Z, N, nocc, w.W1, w.W2, sh);
    clk.mark(kStBackTr);
    // (8) C = L^-T Z, D = L Z (= S C) and the AO populations
    //     (S P)_mu,mu = sum_i f_i C_mu,i D_mu,i on the FP64 tensor cores: each
    //     warp owns 8-row blocks of mu and runs over pairs of 8-column tiles
    //     of the occupied eigenvectors (the rows of L and L^-T are shared by
    //     the pair; four independent accumulator chains where the ranges of
    //     k overlap).  Row mu of L ends and column mu of L^-1 starts at the
    //     diagonal.  D only feeds the populations and is not stored.
    {
      const int T = (N + 7) >> 3, Ti = (nocc + 7) >> 3;
      const int g = lane >> 2, t4 = lane & 3;
      for (int MU = wid; MU < T; MU += NW) {
        const int mu = MU * 8 + g;
        const bool mu_ok = mu < N;
        const double* lrow = L + (long long)(mu_ok ? mu : 0) * N;
        const int kd = min(N, MU * 8 + 8), kc = MU * 8;  // D: k < kd; C: k >= kc
        double pp = 0.0;
        for (int IV = 0; IV < Ti; IV += 2) {
          const int ib0 = IV * 8 + g, ib1 = ib0 + 8;
          const bool ok0 = ib0 < nocc, ok1 = ib1 < nocc;
          double c00 = 0.0, c01 = 0.0, c10 = 0.0, c11 = 0.0;
          double d00 = 0.0, d01 = 0.0, d10 = 0.0, d11 = 0.0;
#pragma unroll 4
          for (int k0 = 0; k0 < N; k0 += 4) {
            const int k = k0 + t4;
            const bool kin = k < N;
            const double* zk = Z + (long long)(kin ? k : 0) * N;
            const double b0 = (kin && ok0) ? zk[ib0] : 0.0;
            const double b1 = (kin && ok1) ? zk[ib1] : 0.0;
            if (k0 < kd) {
              const double a = (mu_ok && kin) ? lrow[k] : 0.0;
              dmma_m8n8k4(d00, d01, a, b0);
              dmma_m8n8k4(d10, d11, a, b1);
            }
            if (k0 >= kc) {
              const double a = (mu_ok && kin) ? Li[(long long)k * N + mu] : 0.0;
              dmma_m8n8k4(c00, c01, a, b0);
              dmma_m8n8k4(c10, c11, a, b1);
            }
          }
          const int ic = IV * 8 + 2 * t4;
          if (mu_ok) {
            if (ic < nocc) {
              C[(long long)mu * N + ic] = c00;
              pp += occ[ic] * c00 * d00;
            }
            if (ic + 1 < nocc) {
              C[(long long)mu * N + ic + 1] = c01;
              pp += occ[ic + 1] * c01 * d01;
            }
            if (ic + 8 < nocc) {
              C[(long long)mu * N + ic + 8] = c10;
              pp += occ[ic + 8] * c10 * d10;
            }
            if (ic + 9 < nocc) {
              C[(long long)mu * N + ic + 9] = c11;
              pp += occ[ic + 9] * c11 * d11;
            }
          }
        }
        pp += __shfl_xor_sync(0xffffffffu, pp, 1);
        pp += __shfl_xor_sync(0xffffffffu, pp, 2);
        if (t4 == 0 && mu < N) pop[mu] = pp;
      }
    }
    __syncthreads();
    clk.mark(kStPop);
    // (9) output charges, energies
    stage_charges_energy<NT>(B, M, mc, w, pop, occ, eps, vao, nocc, sh, e_el, e2, e3, rms);
    if (Robust && lshift != 0.0) {
      // with a shifted Fock matrix sum(f eps) is not tr(F P): E_el = tr(H0 P) = sum_k f_k z_k^T H0' z_k
      double part = 0.0;
      for (long long idx = tid; idx < (long long)N * nocc; idx += NT) {
        const int i = (int)(idx / nocc), k = (int)(idx % nocc);
        double hz = 0.0;
        for (int j = 0; j < N; ++j) hz += Hp[(long long)i * N + j] * Z[(long long)j * N + k];
        part += occ[k] * Z[(long long)i * N + k] * hz;
      }
      e_el = block_sum(part, sh.red);
    }
    const double escc = e_el + e2 + e3 + ts;
    const double err = have_e ? fabs(escc - last_e) : INFINITY;
    if (err < opt.energy_tol && rms < opt.charge_tol) {
      converged = true;
      break;
    }
    clk.mark(kStEnergy);
    // (10) charge mixing
    stage_mix<NT>(ro, mc, w, cap, bro_iter, sh);
    last_e = escc;
    have_e = true;
    have_prev = lshift != 0.0;
    __syncthreads();
    clk.mark(kStMix);
  }
  if (iter > ro.max_scc) iter = ro.max_scc;
  }  // rungs
  if (!Robust && !converged && B.failed && tid == 0) B.failed[atomicAdd(B.queue + 3, 1)] = m;
  if constexpr (Robust) {  // rung-0 molecules keep the 0 the host wrote before the launches
    if (B.rung && tid == 0) B.rung[m] = converged ? rung_used : -1;
  }

  // ---- results
  stage_results<NT>(B, mc, w, iter, converged, e_el, e2, e3, ts, mu);
  if (B.orb_eps) {  // orbital energies (NaN where the eigensolver did not need them) and occupations
    const int ao0 = B.ao_off[m];
    for (int i = tid; i < N; i += NT) {
      B.orb_eps[ao0 + i] = (i < nneed_last || i == N - 1) ? eps[i] : __longlong_as_double(0x7ff8000000000000LL);
      B.orb_occ[ao0 + i] = occ[i];
    }
  }
  // density and energy-weighted density of the last diagonalisation
  // (src/linalg.rs:243-273), kept per molecule for the gradient kernel:
  // P = C f C^T and W = C f eps C^T on the FP64 tensor cores, 8x8 tiles on
  // and below the diagonal written to both triangles
  {
    const int T = (N + 7) >> 3;
    const int g = lane >> 2, t4 = lane & 3;
    for (int tile = wid; tile < T * (T + 1) / 2; tile += NW) {
      int I = 0;
      while ((I + 1) * (I + 2) / 2 <= tile) ++I;
      const int J = tile - I * (I + 1) / 2;
      const int i = I * 8 + g, jb = J * 8 + g;
      double p0 = 0.0, p1 = 0.0, q0 = 0.0, q1 = 0.0;
#pragma unroll 4
      for (int k0 = 0; k0 < nocc; k0 += 4) {
        const int k = k0 + t4;
        const double ci = (i < N && k < nocc) ? C[(long long)i * N + k] * occ[k] : 0.0;
        const double cj = (jb < N && k < nocc) ? C[(long long)jb * N + k] : 0.0;
        dmma_m8n8k4(p0, p1, ci, cj);
        dmma_m8n8k4(q0, q1, k < nocc ? ci * eps[k] : 0.0, cj);
      }
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int j = J * 8 + 2 * t4 + c;
        if (i < N && j <= i) {
          const double pv = c ? p1 : p0, qv = c ? q1 : q0;
          B.P[mo + (long long)i * N + j] = pv;
          B.P[mo + (long long)j * N + i] = pv;
          B.W[mo + (long long)i * N + j] = qv;
          B.W[mo + (long long)j * N + i] = qv;
        }
      }
    }
  }
  __syncthreads();
  clk.mark(kStFinal);
}

// Persistent SCC kernel.  Robust = false: molecules q_begin..q_end of the
// processing order (rung 0 of the fallback ladder); Robust = true: the
// molecules the rung-0 launches left unconverged (rungs 1-3).
template <int NT, bool Robust>
__global__ void __launch_bounds__(NT, (kSccThreadsPerSm / NT) > 0 ? kSccThreadsPerSm / NT : 1)
    scc_kernel(Batch B, Model M, SccOptions opt, SccLaunch SL) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ SccShared sh;
  __shared__ int next;
  int* sh_atom = (int*)smraw;
  int* sh_k = sh_atom + SL.maxnsh;
  int* sh_ao0 = sh_k + SL.maxnsh;
  int* ao_sh = sh_ao0 + SL.maxnsh;
  int* atom_sh = ao_sh + SL.maxn;  // maxnat + 1
  const size_t ib = ((size_t)4 * scc_ints(SL.maxnsh, SL.maxn, SL.maxnat) + 15) & ~(size_t)15;
  double* vec = (double*)(smraw + ib);
  double* As = vec + (size_t)kVecSlots * SL.maxn;
  const long long as_cap = ((long long)SL.smem_bytes - (long long)scc_smem_fixed(SL.maxnsh, SL.maxn, SL.maxnat)) / 8;
  const int nfailed = Robust ? B.queue[3] : 0;  // written by the rung-0 launches before this one
  for (;;) {
    if (threadIdx.x == 0) next = Robust ? atomicAdd(B.queue + 2, 1) : SL.q_begin + atomicAdd(SL.counter, 1);
    __syncthreads();
    const int idx = next;
    __syncthreads();
    int m;
    if (Robust) {
      if (idx >= nfailed) break;
      m = B.failed[idx];
    } else {
      if (idx >= SL.q_end) break;
      m = B.order[idx];
      if (B.status[m] != kOk) continue;  // rejected during setup
    }
    scc_molecule<NT, Robust>(B, M, opt, SL, m, sh, sh_atom, sh_k, ao_sh, atom_sh, sh_ao0, vec, As, as_cap);
  }
}

// ============================================================ large molecules
// Molecules too large for one SM run on many SMs: the kernels of wide.cuh
// (included at the end of this file) share the stage functions above.

__host__ __device__ inline size_t dense_table_bytes(int maxnsh, int maxn, int maxnat) {
  return ((size_t)4 * scc_ints(maxnsh, maxn, maxnat) + 15) & ~(size_t)15;
}

struct DenseTables {
  int *sh_atom, *sh_k, *sh_ao0, *ao_sh, *atom_sh;
};
__device__ DenseTables dense_tables(unsigned char* raw, int maxnsh, int maxn) {
  DenseTables t;
  t.sh_atom = (int*)raw;
  t.sh_k = t.sh_atom + maxnsh;
  t.sh_ao0 = t.sh_k + maxnsh;
  t.ao_sh = t.sh_ao0 + maxnsh;
  t.atom_sh = t.ao_sh + maxn;
  return t;
}

long long scc_workspace_doubles(int maxn, int maxnsh, int cap, int maxnat) {
  return cta_ws_size(maxn, maxnsh, cap, maxnat);
}

// Dynamic shared memory for a class: index tables, vectors and, when
// `matrix_n` > 0, room for a matrix_n x work_lda(matrix_n) working matrix.
size_t scc_smem_bytes(int maxnsh, int maxn, int maxnat, int matrix_n) {
  const size_t fixed = scc_smem_fixed(maxnsh, maxn, maxnat);
  return matrix_n > 0 ? fixed + sizeof(double) * (size_t)matrix_n * work_lda(matrix_n) : fixed;
}

// Largest dynamic shared memory a CTA of the class may request: the SM's
// 228 KB shared by its kSccThreadsPerSm / nt CTAs (1 KB of which each CTA reserves), less
// the kernel's static shared memory.
size_t scc_max_dynamic_smem(int nt) {
  cudaFuncAttributes a;
  const cudaError_t e = nt == 512   ? cudaFuncGetAttributes(&a, scc_kernel<512, false>)
                        : nt == 256 ? cudaFuncGetAttributes(&a, scc_kernel<256, false>)
                                    : cudaFuncGetAttributes(&a, scc_kernel<128, false>);
  const size_t stat = e == cudaSuccess ? a.sharedSizeBytes : 8192;
  const int ctas = std::max(1, kSccThreadsPerSm / nt);
  const size_t per_cta = 233472 / ctas - 1024;  // the SM's 228 KB shared by its CTAs
  return per_cta - stat - 256;
}

template <int NT, bool Robust>
static cudaError_t launch_scc_nt(int grid, size_t smem, cudaStream_t st, const Batch& B, const Model& M,
                                 const SccOptions& opt, const SccLaunch& SL) {
  cudaError_t e = cudaFuncSetAttribute(scc_kernel<NT, Robust>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  scc_kernel<NT, Robust><<<grid, NT, smem, st>>>(B, M, opt, SL);
  return cudaGetLastError();
}

// Host launcher of one size class (nt = 512, 256 or 128 threads per CTA;
// 512 / nt CTAs share an SM).
cudaError_t launch_scc(int nt, int grid, size_t smem, cudaStream_t st, const Batch& B, const Model& M,
                       const SccOptions& opt, const SccLaunch& SL) {
  if (nt == 512) return launch_scc_nt<512, false>(grid, smem, st, B, M, opt, SL);
  if (nt == 256) return launch_scc_nt<256, false>(grid, smem, st, B, M, opt, SL);
  if (nt == 128) return launch_scc_nt<128, false>(grid, smem, st, B, M, opt, SL);
  return cudaErrorInvalidValue;
}

// Host launcher of the fallback-ladder kernel (rungs 1-3 for the molecules
// listed in B.failed; returns at once when the list is empty).
cudaError_t launch_scc_robust(int nt, int grid, size_t smem, cudaStream_t st, const Batch& B, const Model& M,
                              const SccOptions& opt, const SccLaunch& SL) {
  if (nt == 512) return launch_scc_nt<512, true>(grid, smem, st, B, M, opt, SL);
  if (nt == 256) return launch_scc_nt<256, true>(grid, smem, st, B, M, opt, SL);
  if (nt == 128) return launch_scc_nt<128, true>(grid, smem, st, B, M, opt, SL);
  return cudaErrorInvalidValue;
}

}  // namespace gfn1

#include "wide.cuh"
