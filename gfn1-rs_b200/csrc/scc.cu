// Persistent SCC kernel: each CTA pulls molecules from a work queue (most
// expensive first) and runs the complete self-consistent-charge loop of
// gfn1-rs `run_scc_with_core` (src/electronic.rs:849-2054, plain charge-vector
// branch, ladder rung 0) on the device.
//
// Algorithmic choices that differ from the reference but give the same results
// up to FP64 rounding:
//  * orthogonaliser: Cholesky S = L L^T instead of Lowdin S^-1/2
//    (src/linalg.rs:193-217).  The density P = C f C^T is invariant to the choice.
//    H0' = L^-1 H0 L^-T is formed once per molecule, and each iteration only adds
//    the potential term  -1/2 (M + M^T),  M = L^-1 diag(v) L  (lower triangular),
//    because  L^-1 (S o V) L^-T = L^-1 diag(v) L + (L^-1 diag(v) L)^T  for
//    V_mu,nu = v_mu + v_nu (src/electronic.rs:3133-3158).
//  * eigensolver: Householder tridiagonalisation, Sturm-sequence bisection for the
//    eigenvalues and inverse iteration (with modified Gram-Schmidt inside
//    eigenvalue clusters) for the occupied eigenvectors only, followed by the
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
constexpr int kVecSlots = 12;                         // N-length scratch vectors per CTA

struct SccShared {
  double red[32];
  double scal[16];
  int iscal[16];
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

// Layout of one CTA's workspace slot (doubles).  maxn / maxnsh / cap / maxnat
// are the batch maxima; matrices use the molecule's own N as leading dimension.
struct CtaWs {
  double *L, *Li, *Hp, *A, *Z, *C, *D, *iw, *vec;
  double *df, *u, *dots, *omega, *beta, *cvec, *qin, *qout, *vsh, *qlast, *dqlast, *qnext, *vout, *qat;
};
__host__ __device__ inline long long cta_ws_size(int maxn, int maxnsh, int cap, int maxnat) {
  const long long n2 = (long long)maxn * maxn;
  return 12 * n2 + (long long)kVecSlots * maxn + 2LL * cap * maxnsh + 2LL * cap * cap + 2LL * cap +
         8LL * maxnsh + maxnat + 64;
}
__device__ __forceinline__ CtaWs cta_ws(double* base, int maxn, int maxnsh, int cap) {
  CtaWs w;
  const long long n2 = (long long)maxn * maxn;
  w.L = base;
  w.Li = w.L + n2;
  w.Hp = w.Li + n2;
  w.A = w.Hp + n2;
  w.Z = w.A + n2;
  w.C = w.Z + n2;
  w.D = w.C + n2;
  w.iw = w.D + n2;  // 5 * n2
  w.vec = w.iw + 5 * n2;
  w.df = w.vec + (long long)kVecSlots * maxn;
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

// Sturm count: number of eigenvalues of the symmetric tridiagonal (d, e2 = e^2)
// that are <= x (LAPACK dlaebz convention with the pivmin guard).
__device__ __forceinline__ int sturm_count(const double* d, const double* e2, int n, double x, double pivmin) {
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  int c = q <= 0.0;
  for (int i = 1; i < n; ++i) {
    q = d[i] - x - e2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    c += q <= 0.0;
  }
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

// Solve (T - lam I) y = x by Gaussian elimination with partial pivoting on the
// tridiagonal matrix; the factors are built on the fly (n steps) in `w`
// (5 arrays of n).  Tiny pivots are replaced by +-tiny.
__device__ void tri_factor(const double* d, const double* e, int n, double lam, double tiny, double* w) {
  double* u0 = w;
  double* u1 = w + n;
  double* u2 = w + 2 * n;
  double* ml = w + 3 * n;
  double* pv = w + 4 * n;
  double a = d[0] - lam;            // current pivot-row diagonal
  double c = n > 1 ? e[0] : 0.0;    // current pivot-row superdiagonal
  for (int k = 0; k < n - 1; ++k) {
    const double b = e[k];               // subdiagonal of row k+1
    const double an = d[k + 1] - lam;    // diagonal of row k+1
    const double cn = (k + 1 < n - 1) ? e[k + 1] : 0.0;  // superdiagonal of row k+1
    if (fabs(a) >= fabs(b)) {
      double piv = a;
      if (fabs(piv) < tiny) piv = piv >= 0.0 ? tiny : -tiny;
      const double mult = b / piv;
      u0[k] = piv;
      u1[k] = c;
      u2[k] = 0.0;
      ml[k] = mult;
      pv[k] = 0.0;
      a = an - mult * c;
      c = cn;
    } else {
      const double mult = a / b;
      u0[k] = b;
      u1[k] = an;
      u2[k] = cn;
      ml[k] = mult;
      pv[k] = 1.0;
      a = c - mult * an;
      c = -mult * cn;
    }
  }
  if (fabs(a) < tiny) a = a >= 0.0 ? tiny : -tiny;
  u0[n - 1] = a;
}

__device__ void tri_solve(const double* w, int n, double* x, long long stride) {
  const double* u0 = w;
  const double* u1 = w + n;
  const double* u2 = w + 2 * n;
  const double* ml = w + 3 * n;
  const double* pv = w + 4 * n;
  for (int k = 0; k < n - 1; ++k) {
    double xk = x[k * stride], xk1 = x[(k + 1) * stride];
    if (pv[k] != 0.0) {
      const double t = xk;
      xk = xk1;
      xk1 = t;
    }
    xk1 -= ml[k] * xk;
    x[k * stride] = xk;
    x[(k + 1) * stride] = xk1;
  }
  x[(n - 1) * stride] /= u0[n - 1];
  if (n > 1) x[(n - 2) * stride] = (x[(n - 2) * stride] - u1[n - 2] * x[(n - 1) * stride]) / u0[n - 2];
  for (int k = n - 3; k >= 0; --k)
    x[k * stride] = (x[k * stride] - u1[k] * x[(k + 1) * stride] - u2[k] * x[(k + 2) * stride]) / u0[k];
}

__device__ void scc_molecule(const Batch& B, const Model& M, const SccOptions& opt, int m, SccShared& sh,
                             int* sh_atom, int* sh_k, int* ao_sh, int* atom_sh, int* sh_ao0) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
  const int a0 = B.atom_off[m], nat = B.atom_off[m + 1] - a0;
  const int sh0 = B.shell_off[m], nsh = B.shell_off[m + 1] - sh0;
  const int ao0 = B.ao_off[m], N = B.ao_off[m + 1] - ao0;
  const long long mo = B.mat_off[m];
  const double* S = B.S + mo;
  const double* H0 = B.H0 + mo;
  CtaWs w = cta_ws(B.ws + (long long)blockIdx.x * B.ws_stride, B.ws_maxn, B.ws_maxnsh, B.ws_cap);
  double* L = w.L;
  double* Li = w.Li;
  double* Hp = w.Hp;
  double* A = w.A;
  double* Z = w.Z;
  double* C = w.C;
  double* D = w.D;
  double* iw = w.iw;
  const double* G = B.gam + B.gam_off[m];
  double* vec = w.vec;
  double* d = vec;
  double* e = vec + N;
  double* tau = vec + 2 * N;
  double* eps = vec + 3 * N;
  double* occ = vec + 4 * N;
  double* pop = vec + 5 * N;
  double* vao = vec + 6 * N;
  double* hv = vec + 7 * N;
  double* pvec = vec + 8 * N;
  double* esq = vec + 9 * N;
  const int cap = B.ws_cap;

  // ---- index tables
  if (tid == 0) {
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
    sh.iscal[0] = kOk;
  }
  __syncthreads();

  StageClock clk(B.stage_cycles);
  // ---- Cholesky S = L L^T (right-looking, in place on L)
  for (long long i = tid; i < (long long)N * N; i += nt) L[i] = S[i];
  __syncthreads();
  for (int k = 0; k < N; ++k) {
    if (tid == 0) {
      const double a = L[(long long)k * N + k];
      // the reference rejects overlaps with an eigenvalue <= eigen_tolerance (1e-12)
      if (!(a > 1e-12)) sh.iscal[0] = kErrInvalidInput;
      const double r = sqrt(fmax(a, 1e-300));
      L[(long long)k * N + k] = r;
      sh.scal[0] = r;
    }
    __syncthreads();
    const double lkk = sh.scal[0];
    for (int i = k + 1 + tid; i < N; i += nt) L[(long long)i * N + k] /= lkk;
    __syncthreads();
    for (int i = k + 1 + wid; i < N; i += nw) {
      const double lik = L[(long long)i * N + k];
      for (int j = k + 1 + lane; j <= i; j += 32) L[(long long)i * N + j] -= lik * L[(long long)j * N + k];
    }
    __syncthreads();
  }
  if (sh.iscal[0] != kOk) {
    if (tid == 0) {
      B.status[m] = sh.iscal[0];
      B.iterations[m] = 0;
    }
    return;
  }
  for (int i = wid; i < N; i += nw)
    for (int j = i + 1 + lane; j < N; j += 32) L[(long long)i * N + j] = 0.0;
  __syncthreads();
  // L^-1, one thread per column
  for (int j = tid; j < N; j += nt) {
    for (int i = 0; i < j; ++i) Li[(long long)i * N + j] = 0.0;
    Li[(long long)j * N + j] = 1.0 / L[(long long)j * N + j];
    for (int i = j + 1; i < N; ++i) {
      double s = 0.0;
      for (int k = j; k < i; ++k) s += L[(long long)i * N + k] * Li[(long long)k * N + j];
      Li[(long long)i * N + j] = -s / L[(long long)i * N + i];
    }
  }
  __syncthreads();
  // H0' = L^-1 H0 L^-T: T = H0 L^-T into A, then H0' = L^-1 T
  for (int i = wid; i < N; i += nw)
    for (int j = lane; j < N; j += 32) {
      double s = 0.0;
      for (int k = 0; k <= j; ++k) s += H0[(long long)i * N + k] * Li[(long long)j * N + k];
      A[(long long)i * N + j] = s;
    }
  __syncthreads();
  for (int i = wid; i < N; i += nw)
    for (int j = lane; j <= i; j += 32) {
      double s = 0.0;
      for (int k = 0; k <= i; ++k) s += Li[(long long)i * N + k] * A[(long long)k * N + j];
      Hp[(long long)i * N + j] = s;
    }
  __syncthreads();
  for (int i = wid; i < N; i += nw)
    for (int j = i + 1 + lane; j < N; j += 32) Hp[(long long)i * N + j] = Hp[(long long)j * N + i];

  clk.mark(kStPrologue);
  // ---- SCC state
  double nref = 0.0;
  for (int s = 0; s < nsh; ++s) nref += M.elem[B.z[a0 + sh_atom[s]]].refocc[sh_k[s]];
  const double nelec = nref - B.charge[m];
  const double kt = fmax(opt.etemp, 0.0) * kBoltzmann;
  for (int s = tid; s < nsh; s += nt) w.qin[s] = B.init_q ? B.init_q[sh0 + s] : 0.0;
  const double mixing = fmin(1.0, fmax(0.01, opt.mixing));
  const int memory = max(opt.broyden_size, 2);
  int bro_iter = 0;
  double last_e = 0.0;
  bool have_e = false;
  bool converged = false;
  int iter = 0;
  double e_el = 0.0, e2 = 0.0, e3 = 0.0, ts = 0.0, mu = 0.0, rms = 0.0;
  __syncthreads();

  for (iter = 1; iter <= opt.max_scc; ++iter) {
    // (1) shell potential from the input charges (src/coulomb.rs:140-193)
    for (int a = tid; a < nat; a += nt) {
      double q = 0.0;
      for (int s = atom_sh[a]; s < atom_sh[a + 1]; ++s) q += w.qin[s];
      w.qat[a] = q;
    }
    __syncthreads();
    for (int i = tid; i < nsh; i += nt) {
      double v = 0.0;
      for (int j = 0; j < nsh; ++j) v += G[(long long)i * nsh + j] * w.qin[j];
      const int a = sh_atom[i];
      const double qa = w.qat[a];
      v += qa * qa * M.elem[B.z[a0 + a]].gam3;
      w.vsh[i] = v;
    }
    __syncthreads();
    for (int i = tid; i < N; i += nt) vao[i] = w.vsh[ao_sh[i]];
    __syncthreads();
    // (2) F' = H0' - 1/2 (M + M^T), M = L^-1 diag(v) L, full symmetric storage in A
    for (int i = wid; i < N; i += nw)
      for (int j = lane; j <= i; j += 32) {
        double s = 0.0;
        for (int k = j; k <= i; ++k) s += Li[(long long)i * N + k] * vao[k] * L[(long long)k * N + j];
        const double f = Hp[(long long)i * N + j] - (i == j ? s : 0.5 * s);
        A[(long long)i * N + j] = f;
        A[(long long)j * N + i] = f;
      }
    __syncthreads();
    clk.mark(kStFock);
    // (3) Householder tridiagonalisation; v_k kept in row k right of the diagonal
    for (int k = 0; k < N - 2; ++k) {
      const int mlen = N - k - 1;
      double* rowk = A + (long long)k * N + (k + 1);
      double part = 0.0;
      for (int i = tid; i < mlen; i += nt) part += rowk[i] * rowk[i];
      const double xn2 = block_sum(part, sh.red);
      const double x0 = rowk[0];
      const double tail = xn2 - x0 * x0;
      if (tail == 0.0) {
        if (tid == 0) {
          d[k] = A[(long long)k * N + k];
          e[k] = x0;
          tau[k] = 0.0;
        }
        __syncthreads();
        continue;
      }
      const double xn = sqrt(xn2);
      const double alpha = x0 >= 0.0 ? -xn : xn;
      const double v0 = x0 - alpha;
      const double beta = 2.0 / (v0 * v0 + tail);
      for (int i = tid; i < mlen; i += nt) hv[i] = (i == 0) ? v0 : rowk[i];
      __syncthreads();
      if (tid == 0) {
        d[k] = A[(long long)k * N + k];
        e[k] = alpha;
        tau[k] = beta;
        rowk[0] = v0;
      }
      // p = beta * B v
      double pv_part = 0.0;
      for (int i = wid; i < mlen; i += nw) {
        const double* brow = A + (long long)(k + 1 + i) * N + (k + 1);
        double s = 0.0;
        for (int j = lane; j < mlen; j += 32) s += brow[j] * hv[j];
        s = warp_sum(s) * beta;
        if (lane == 0) {
          pvec[i] = s;
          pv_part += s * hv[i];
        }
      }
      const double pv = block_sum(pv_part, sh.red);
      const double K = 0.5 * beta * pv;
      for (int i = wid; i < mlen; i += nw) {
        double* brow = A + (long long)(k + 1 + i) * N + (k + 1);
        const double vi = hv[i], wi = pvec[i] - K * vi;
        for (int j = lane; j < mlen; j += 32) {
          const double vj = hv[j], wj = pvec[j] - K * vj;
          brow[j] -= vi * wj + wi * vj;
        }
      }
      __syncthreads();
    }
    if (tid == 0) {
      if (N >= 2) {
        d[N - 2] = A[(long long)(N - 2) * N + (N - 2)];
        e[N - 2] = A[(long long)(N - 1) * N + (N - 2)];
        tau[N - 2] = 0.0;
      }
      d[N - 1] = A[(long long)(N - 1) * N + (N - 1)];
      e[N - 1] = 0.0;
      tau[N - 1] = 0.0;
    }
    __syncthreads();
    clk.mark(kStTridiag);
    // (4) eigenvalues by bisection
    double gl = INFINITY, gu = -INFINITY, onenrm = 0.0, emax2 = 0.0;
    for (int i = tid; i < N; i += nt) {
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
    for (int k = tid; k < N; k += nt) {
      double lo = gl, hi = gu;
      for (int it = 0; it < 128; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break;
        if (sturm_count(d, esq, N, mid, pivmin) >= k + 1) hi = mid;
        else lo = mid;
      }
      eps[k] = 0.5 * (lo + hi);
    }
    __syncthreads();
    clk.mark(kStEigval);
    // (5) occupations (src/electronic.rs:3815-3921), warp 0
    if (wid == 0) {
      double f_mu = 0.0, f_ts = 0.0;
      if (kt <= 0.0) {
        double rem = fmax(nelec, 0.0);
        int homo = 0;
        for (int i = 0; i < N; ++i) {
          const double fill = fmin(rem, 2.0);
          if (lane == 0) occ[i] = fill;
          rem -= fill;
          if (fill > 1e-12) homo = i;
        }
        f_mu = eps[homo];
      } else if (nelec <= 0.0) {
        for (int i = lane; i < N; i += 32) occ[i] = 0.0;
        f_mu = eps[0];
      } else if (nelec >= 2.0 * N) {
        for (int i = lane; i < N; i += 32) occ[i] = 2.0;
        f_mu = eps[N - 1];
      } else {
        double lo = eps[0] - 100.0 * kt - 10.0, hi = eps[N - 1] + 100.0 * kt + 10.0;
        for (int it = 0; it < 200; ++it) {
          const double mid = 0.5 * (lo + hi);
          double s = 0.0;
          for (int i = lane; i < N; i += 32) s += 2.0 / (1.0 + exp(fmin(80.0, fmax(-80.0, (eps[i] - mid) / kt))));
          s = warp_sum(s);
          double nlo = lo, nhi = hi;
          if (s < nelec) nlo = mid;
          else nhi = mid;
          if (nlo == lo && nhi == hi) break;
          lo = nlo;
          hi = nhi;
        }
        f_mu = 0.5 * (lo + hi);
        double t = 0.0;
        for (int i = lane; i < N; i += 32) {
          const double f = 2.0 / (1.0 + exp(fmin(80.0, fmax(-80.0, (eps[i] - f_mu) / kt))));
          occ[i] = f;
          const double nn = fmin(1.0 - 1e-16, fmax(1e-16, 0.5 * f));
          t += 2.0 * kt * (nn * log(nn) + (1.0 - nn) * log(1.0 - nn));
        }
        f_ts = warp_sum(t);
      }
      if (lane == 0) {
        sh.scal[1] = f_mu;
        sh.scal[2] = f_ts;
      }
    }
    __syncthreads();
    mu = sh.scal[1];
    ts = sh.scal[2];
    // number of orbitals whose occupation matters at FP64 resolution
    int nocc_loc = 0;
    for (int i = tid; i < N; i += nt)
      if (occ[i] > 1e-30) nocc_loc = max(nocc_loc, i + 1);
    const int nocc = (int)block_max((double)nocc_loc, sh.red);
    clk.mark(kStFermi);
    // (6) inverse iteration for the occupied eigenvectors (columns of Z)
    const double ortol = 1e-5 * onenrm;
    const double tiny = DBL_EPSILON * fmax(onenrm, 1e-300);
    for (int j = tid; j < nocc; j += nt) {
      const bool start = (j == 0) || (eps[j] - eps[j - 1] > ortol);
      if (!start) continue;
      int jend = j + 1;
      while (jend < nocc && eps[jend] - eps[jend - 1] <= ortol) ++jend;
      double* ws = iw + (long long)5 * N * j;
      double lam_prev = -INFINITY;
      for (int jj = j; jj < jend; ++jj) {
        double lam = eps[jj];
        const double pert = 10.0 * DBL_EPSILON * fmax(fabs(lam), onenrm);
        if (jj > j && lam - lam_prev < pert) lam = lam_prev + pert;
        lam_prev = lam;
        tri_factor(d, e, N, lam, tiny, ws);
        double* x = Z + jj;  // column jj, stride N
        for (int i = 0; i < N; ++i) x[(long long)i * N] = hash_unit(i, jj) + 1e-3;
        const int nit = (jend - j > 1) ? 5 : 3;
        for (int it = 0; it < nit; ++it) {
          tri_solve(ws, N, x, N);
          for (int q = j; q < jj; ++q) {  // modified Gram-Schmidt inside the cluster
            double dot = 0.0;
            for (int i = 0; i < N; ++i) dot += Z[(long long)i * N + q] * x[(long long)i * N];
            for (int i = 0; i < N; ++i) x[(long long)i * N] -= dot * Z[(long long)i * N + q];
          }
          double nrm = 0.0;
          for (int i = 0; i < N; ++i) nrm += x[(long long)i * N] * x[(long long)i * N];
          const double inv = 1.0 / sqrt(fmax(nrm, 1e-300));
          for (int i = 0; i < N; ++i) x[(long long)i * N] *= inv;
        }
      }
    }
    __syncthreads();
    clk.mark(kStInvIter);
    // (7) back-transformation Z := Q Z, one thread per eigenvector column
    for (int j = tid; j < nocc; j += nt) {
      for (int k = N - 3; k >= 0; --k) {
        const double tk = tau[k];
        if (tk == 0.0) continue;
        const double* v = A + (long long)k * N + (k + 1);
        double s = 0.0;
        for (int i = 0; i < N - k - 1; ++i) s += v[i] * Z[(long long)(k + 1 + i) * N + j];
        s *= tk;
        for (int i = 0; i < N - k - 1; ++i) Z[(long long)(k + 1 + i) * N + j] -= s * v[i];
      }
    }
    __syncthreads();
    clk.mark(kStBackTr);
    // (8) C = L^-T Z, D = L Z and the AO populations (S P)_mu,mu
    for (int mu_ = wid; mu_ < N; mu_ += nw) {
      double popp = 0.0;
      for (int i = lane; i < nocc; i += 32) {
        double c = 0.0, dd = 0.0;
        for (int k = mu_; k < N; ++k) c += Li[(long long)k * N + mu_] * Z[(long long)k * N + i];
        for (int k = 0; k <= mu_; ++k) dd += L[(long long)mu_ * N + k] * Z[(long long)k * N + i];
        C[(long long)mu_ * N + i] = c;
        D[(long long)mu_ * N + i] = dd;
        popp += occ[i] * c * dd;
      }
      popp = warp_sum(popp);
      if (lane == 0) pop[mu_] = popp;
    }
    __syncthreads();
    clk.mark(kStPop);
    // (9) output charges, energies (src/electronic.rs:2173-2191)
    for (int s = tid; s < nsh; s += nt) {
      const ElemTable& el = M.elem[B.z[a0 + sh_atom[s]]];
      const int k = sh_k[s];
      double p = 0.0;
      for (int q = 0; q < 2 * el.l[k] + 1; ++q) p += pop[sh_ao0[s] + q];
      w.qout[s] = el.refocc[k] - p;
    }
    double part = 0.0;
    for (int i = tid; i < N; i += nt) part += occ[i] * eps[i] + vao[i] * pop[i];
    e_el = block_sum(part, sh.red);
    for (int a = tid; a < nat; a += nt) {
      double q = 0.0;
      for (int s = atom_sh[a]; s < atom_sh[a + 1]; ++s) q += w.qout[s];
      w.qat[a] = q;
    }
    __syncthreads();
    double p2 = 0.0, p3 = 0.0, pr = 0.0;
    for (int i = tid; i < nsh; i += nt) {
      double v = 0.0;
      for (int j = 0; j < nsh; ++j) v += G[(long long)i * nsh + j] * w.qout[j];
      p2 += w.qout[i] * v;
      const int a = sh_atom[i];
      const double qa = w.qat[a];
      const double g3 = M.elem[B.z[a0 + a]].gam3;
      w.vout[i] = v + qa * qa * g3;
      const double r = w.qout[i] - w.qin[i];
      pr += r * r;
    }
    for (int a = tid; a < nat; a += nt) {
      const double qa = w.qat[a];
      p3 += qa * qa * qa * M.elem[B.z[a0 + a]].gam3 / 3.0;
    }
    e2 = 0.5 * block_sum(p2, sh.red);
    e3 = block_sum(p3, sh.red);
    rms = nsh ? sqrt(block_sum(pr, sh.red) / nsh) : 0.0;
    const double escc = e_el + e2 + e3 + ts;
    const double err = have_e ? fabs(escc - last_e) : INFINITY;
    if (err < opt.energy_tol && rms < opt.charge_tol) {
      converged = true;
      break;
    }
    clk.mark(kStEnergy);
    // (10) charge mixing
    bool have_next = false;
    if (opt.broyden) {
      bro_iter += 1;
      if (bro_iter == 1) {
        for (int s = tid; s < nsh; s += nt) {
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
        for (int s = tid; s < nsh; s += nt) {
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
        for (int s = tid; s < nsh; s += nt) {
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
        for (int r = wid; r < mact; r += nw) {
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
        for (int idx = tid; idx < mact * mact; idx += nt) {
          const int r = idx / mact, c = idx % mact;
          const int si = ((start + r - 1) % memory) % cap, sj = ((start + c - 1) % memory) % cap;
          double b = w.omega[si] * w.omega[sj] * w.dots[(long long)si * cap + sj];
          if (r == c) b += 0.01 * 0.01;
          w.beta[(long long)r * mact + c] = b;
        }
        for (int r = tid; r < mact; r += nt) {
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
            for (int j = tid; j < mact; j += nt) {
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
          for (int j = col + tid; j < mact; j += nt) w.beta[(long long)col * mact + j] /= dg;
          if (tid == 0) w.cvec[col] /= dg;
          __syncthreads();
          for (int idx = tid; idx < mact * (mact - col); idx += nt) {
            const int r = idx / (mact - col), j = col + idx % (mact - col);
            if (r == col) continue;
            const double f = w.beta[(long long)r * mact + col];
            if (f == 0.0 || j == col) continue;
            w.beta[(long long)r * mact + j] -= f * w.beta[(long long)col * mact + j];
          }
          for (int r = tid; r < mact; r += nt) {
            if (r == col) continue;
            const double f = w.beta[(long long)r * mact + col];
            if (f != 0.0) w.cvec[r] -= f * w.cvec[col];
          }
          __syncthreads();
          for (int r = tid; r < mact; r += nt)
            if (r != col) w.beta[(long long)r * mact + col] = 0.0;
          __syncthreads();
        }
        if (ok) {
          for (int s = tid; s < nsh; s += nt) {
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
        for (int s = tid; s < nsh; s += nt)
          if (!isfinite(w.qnext[s]) || fabs(w.qnext[s]) >= 10.0) bad = 1;
        if (block_max((double)bad, sh.red) > 0.0) have_next = false;
      }
    }
    if (!have_next)
      for (int s = tid; s < nsh; s += nt) w.qnext[s] = w.qin[s] + mixing * (w.qout[s] - w.qin[s]);
    __syncthreads();
    for (int s = tid; s < nsh; s += nt) w.qin[s] = w.qnext[s];
    last_e = escc;
    have_e = true;
    __syncthreads();
    clk.mark(kStMix);
  }
  if (iter > opt.max_scc) iter = opt.max_scc;

  // ---- results
  if (tid == 0) {
    double* t = B.terms + (long long)m * kTerms;
    const double erep = t[2], edisp = t[7];
    const double total_internal = e_el + e2 + e3 + erep + edisp;
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
  for (int s = tid; s < nsh; s += nt) {
    B.shell_q[sh0 + s] = w.qout[s];
    B.shell_pot[sh0 + s] = w.vout[s];
  }
  for (int a = tid; a < nat; a += nt) B.atom_q[a0 + a] = w.qat[a];
  // density and energy-weighted density of the last diagonalisation
  // (src/linalg.rs:243-273), kept per molecule for the gradient kernel
  int nocc = 0;
  for (int i = 0; i < N; ++i)
    if (occ[i] > 1e-30) nocc = i + 1;
  for (int i = wid; i < N; i += nw)
    for (int j = lane; j <= i; j += 32) {
      double p = 0.0, q = 0.0;
      for (int k = 0; k < nocc; ++k) {
        const double cc = C[(long long)i * N + k] * C[(long long)j * N + k];
        p += occ[k] * cc;
        q += occ[k] * eps[k] * cc;
      }
      B.P[mo + (long long)i * N + j] = p;
      B.P[mo + (long long)j * N + i] = p;
      B.W[mo + (long long)i * N + j] = q;
      B.W[mo + (long long)j * N + i] = q;
    }
  __syncthreads();
  clk.mark(kStFinal);
}

__global__ void __launch_bounds__(256) scc_kernel(Batch B, Model M, SccOptions opt, int max_nsh, int max_n) {
  extern __shared__ int sm_int[];
  __shared__ SccShared sh;
  __shared__ int next;
  int* sh_atom = sm_int;
  int* sh_k = sh_atom + max_nsh;
  int* sh_ao0 = sh_k + max_nsh;
  int* ao_sh = sh_ao0 + max_nsh;
  int* atom_sh = ao_sh + max_n;  // max_nat + 1
  for (;;) {
    if (threadIdx.x == 0) next = atomicAdd(B.queue, 1);
    __syncthreads();
    const int idx = next;
    __syncthreads();
    if (idx >= B.nmol) break;
    const int m = B.order[idx];
    if (B.status[m] != kOk) continue;  // rejected during setup
    scc_molecule(B, M, opt, m, sh, sh_atom, sh_k, ao_sh, atom_sh, sh_ao0);
  }
}

long long scc_workspace_doubles(int maxn, int maxnsh, int cap, int maxnat) {
  return cta_ws_size(maxn, maxnsh, cap, maxnat);
}

}  // namespace gfn1
