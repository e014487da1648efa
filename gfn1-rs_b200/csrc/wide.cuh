// Large molecules on many SMs ("wide" path): the SCC of gfn1-rs
// `run_scc_with_core` (src/electronic.rs:849-2054) with the matrix algebra of
// one molecule spread over a group of CTAs, batched over every large molecule
// of a call.  No library routine is involved: the Cholesky orthogonaliser, the
// triangular inverse, the congruence products, the Householder
// tridiagonalisation, the eigenvalues, inverse iteration, back-transformation,
// populations and the final density matrices are kernels of this file, the
// matrix products on the FP64 tensor cores (mma.m8n8k4 .f64).  The charge,
// energy, mixing and result stages are the ones of the persistent kernel.
//
// Included at the end of scc.cu (namespace gfn1), so it shares the stage
// functions, the Sturm-count eigenvalue search and the tridiagonal solver.
//
// Layout of one molecule's slot: N x N matrices row-major with leading
// dimension ld = N rounded up to four doubles (32-byte rows):
//   L    Cholesky factor of S (lower triangle, zeros above)
//   Li   L^-1 (lower triangle, zeros above)
//   Hp   H0' = L^-1 H0 L^-T
//   A    working matrix: F' = L^-1 F L^-T, then the Householder reflectors in
//        its strictly lower triangle (column j holds reflector j below the
//        subdiagonal; its first entry is an implicit 1)
//   Z    eigenvectors of F' (columns 0..nocc-1): tridiagonal basis after
//        inverse iteration, orthonormal basis after the back-transformation
//   C    MO coefficients L^-T Z (columns 0..nocc-1)
// plus the factor arrays of inverse iteration (5 N x N, interleaved per
// eigenvector), the panel buffer of the reduction, N-vectors and the SCC
// vectors and Broyden history in the CtaWs layout.
#pragma once

namespace gfn1 {

// ------------------------------------------------------------------ tiles
// One 64 x 64 output tile on the FP64 tensor cores for a CTA of NT threads
// (128 or 256): acc += sum_{k0 <= k < k1} A(i, k) B(k, j) for i in
// [i0, i0 + 64), j in [j0, j0 + 64).  la(i, k) / lb(k, j) return operand
// elements (zero outside the operands' extents and the k range).  AI: the
// operand A is contiguous along i in memory (threads walk i first), else along
// k; BJ: B is contiguous along j, else along k.  The operands go through
// shared memory in chunks of 16 k, double-buffered (loads of the next chunk
// are in flight while the current one is multiplied).  Warps form a 2 x (NT/64)
// grid of 32 x (64 / (NT/64)) warp tiles; acc[mi][nj][c] holds row
// i0 + 32 wi + 8 mi + g, column j0 + WJ wj + 8 nj + 2 t4 + c (g = lane / 4,
// t4 = lane % 4).
constexpr int kTileK = 16;
constexpr int kTilePad = 68;  // shared row length in doubles (bank spread for the fragment loads)
constexpr size_t kTileSmemBytes = sizeof(double) * 2 * 2 * kTileK * kTilePad;

template <int NT>
struct TileShape {
  static constexpr int kWarpsJ = NT / 64;          // 2 (128 threads) or 4 (256 threads)
  static constexpr int kWJ = 64 / kWarpsJ;         // warp tile width: 32 or 16
  static constexpr int kNJ = kWJ / 8;              // 8x8 tiles per warp row: 4 or 2
  static constexpr int kPer = 64 * kTileK / NT;    // operand elements per thread per chunk
};

template <int NT>
__device__ __forceinline__ void tile_zero(double (&acc)[4][TileShape<NT>::kNJ][2]) {
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < TileShape<NT>::kNJ; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
}

template <int NT, bool AI, bool BJ, class LA, class LB>
__device__ __forceinline__ void tile_mma(const LA& la, const LB& lb, int i0, int j0, int k0, int k1,
                                         double (&acc)[4][TileShape<NT>::kNJ][2], double* smem) {
  using TS = TileShape<NT>;
  constexpr int P = TS::kPer;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int wi = wid & 1, wj = wid >> 1;
  const int g = lane >> 2, t4 = lane & 3;
  if (k1 <= k0) return;
  double* As[2] = {smem, smem + kTileK * kTilePad};
  double* Bs[2] = {smem + 2 * kTileK * kTilePad, smem + 3 * kTileK * kTilePad};
  double ra[P], rb[P];
  auto load = [&](int kc) {
#pragma unroll
    for (int r = 0; r < P; ++r) {
      const int e = tid + NT * r;
      const int ai = AI ? (e & 63) : (e >> 4), ak = AI ? (e >> 6) : (e & 15);
      const int bj = BJ ? (e & 63) : (e >> 4), bk = BJ ? (e >> 6) : (e & 15);
      const int ka = kc + ak, kb = kc + bk;
      ra[r] = ka < k1 ? la(i0 + ai, ka) : 0.0;
      rb[r] = kb < k1 ? lb(kb, j0 + bj) : 0.0;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int r = 0; r < P; ++r) {
      const int e = tid + NT * r;
      const int ai = AI ? (e & 63) : (e >> 4), ak = AI ? (e >> 6) : (e & 15);
      const int bj = BJ ? (e & 63) : (e >> 4), bk = BJ ? (e >> 6) : (e & 15);
      As[buf][ak * kTilePad + ai] = ra[r];
      Bs[buf][bk * kTilePad + bj] = rb[r];
    }
  };
  const int nch = (k1 - k0 + kTileK - 1) / kTileK;
  load(k0);
  __syncthreads();  // the previous user of the shared buffers is done
  store(0);
  __syncthreads();
  for (int c = 0; c < nch; ++c) {
    const int buf = c & 1;
    if (c + 1 < nch) load(k0 + (c + 1) * kTileK);
    const double* as = As[buf] + 32 * wi + g;
    const double* bs = Bs[buf] + TS::kWJ * wj + g;
#pragma unroll
    for (int kk = 0; kk < kTileK; kk += 4) {
      double a[4], b[TS::kNJ];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) a[mi] = as[(kk + t4) * kTilePad + 8 * mi];
#pragma unroll
      for (int nj = 0; nj < TS::kNJ; ++nj) b[nj] = bs[(kk + t4) * kTilePad + 8 * nj];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int nj = 0; nj < TS::kNJ; ++nj) dmma_m8n8k4(acc[mi][nj][0], acc[mi][nj][1], a[mi], b[nj]);
    }
    if (c + 1 < nch) store(buf ^ 1);
    __syncthreads();
  }
}

// Visits the tile's elements: f(i, j, value) for the rows and columns this
// thread holds.
template <int NT, class F>
__device__ __forceinline__ void tile_for_each(const double (&acc)[4][TileShape<NT>::kNJ][2], int i0, int j0,
                                              const F& f) {
  using TS = TileShape<NT>;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int wi = wid & 1, wj = wid >> 1;
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int nj = 0; nj < TS::kNJ; ++nj)
#pragma unroll
      for (int c = 0; c < 2; ++c)
        f(i0 + 32 * wi + 8 * mi + g, j0 + TS::kWJ * wj + 8 * nj + 2 * t4 + c, acc[mi][nj][c]);
}

// Lower-triangle tile (I, J), J <= I, of the t-th tile in row order.
__device__ __forceinline__ void lower_tile(int t, int& I, int& J) {
  I = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((I + 1) * (I + 2) / 2 <= t) ++I;
  while (I * (I + 1) / 2 > t) --I;
  J = t - I * (I + 1) / 2;
}

// ------------------------------------------------------------------ group barrier
// Barrier among the n CTAs working on one molecule inside a cooperative launch
// (all CTAs are resident).  Thread 0 of each CTA arrives on a counter; the last
// one resets it and advances the generation, the others wait for the new
// generation.  Every wait is bounded: after kSpinCycles clock cycles (about a
// second), or as soon as any CTA has flagged an error, the waiter raises the
// molecule's error flag and the barrier returns false; the kernel then
// returns, so a lost CTA can never hang the GPU.
struct GroupSync {
  unsigned int count;
  unsigned int gen;
  int err;
  int pad;
};
constexpr int kFlagSlots = 1024;  // per-CTA flags of one molecule's group (at least kWideMaxG)
constexpr long long kSpinCycles = 2000000000LL;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed_i32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Barrier among CTAs 0..n-1 of a group by per-CTA flags: CTA c publishes
// `target` in flags[c] (a release store after its writes), and thread t of
// every CTA waits for flags[t], flags[t + blockDim.x], ... to reach `target`
// (acquire loads), so that no counter is contended.  `target` grows with every
// barrier of every launch (the launch number in the high bits), so flags left
// by earlier launches never satisfy it.  The waits are bounded like those of
// group_barrier; `each(t)` runs in the waiting thread once peer t has arrived
// (the caller reads that peer's published data there).
template <class F>
__device__ __forceinline__ bool flag_barrier(unsigned long long* flags, GroupSync* gs, int c, int n,
                                             unsigned long long target, const F& each) {
  __shared__ int bad_sh;
  if (threadIdx.x == 0) bad_sh = 0;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    st_release_u64(flags + c, target);
  }
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    if (t != c) {
      const long long t0 = clock64();
      while (ld_acquire_u64(flags + t) < target) {
        if (ld_relaxed_i32(&gs->err) != 0 || clock64() - t0 > kSpinCycles) {
          atomicExch(&gs->err, 1);
          bad_sh = 1;
          break;
        }
        __nanosleep(20);
      }
    }
    each(t);
  }
  __syncthreads();
  return bad_sh == 0;
}

__device__ __forceinline__ bool group_barrier(GroupSync* gs, int n) {
  __shared__ int ok_sh;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    if (n > 1) {
      const unsigned g = ld_acquire_u32(&gs->gen);
      __threadfence();
      if (atomicAdd(&gs->count, 1u) == (unsigned)(n - 1)) {
        atomicExch(&gs->count, 0u);
        __threadfence();
        atomicExch(&gs->gen, g + 1u);
      } else {
        const long long t0 = clock64();
        while (ld_acquire_u32(&gs->gen) == g) {
          if (ld_relaxed_i32(&gs->err) != 0 || clock64() - t0 > kSpinCycles) {
            atomicExch(&gs->err, 1);
            ok = 0;
            break;
          }
          __nanosleep(32);
        }
      }
      __threadfence();
    }
    if (ok && ld_relaxed_i32(&gs->err) != 0) ok = 0;
    ok_sh = ok;
  }
  __syncthreads();
  return ok_sh != 0;
}

}  // namespace gfn1

namespace gfn1 {

// ------------------------------------------------------------------ per-molecule slot
// SCC state of one large molecule between kernels (the device counterpart of
// the loop variables of run_scc_with_core).
struct WideState {
  int status;     // kOk, or the molecule's error
  int nocc;       // orbitals with occupation above 1e-30 (prefix length)
  int converged;  // convergence test of the last iteration passed
  int iter;       // SCC iterations of the current rung
  int bro_iter;   // Broyden iteration counter
  int have_e;     // a previous SCC energy exists
  int nneed;      // eigenvalues 0..nneed-1 (and N-1) known
  int have_prev;  // a previous density exists (level shift)
  int spin;
  int rung;       // rung of the fallback ladder being run
  int pad[2];
  double last_e, e_el, e2, e3, ts, mu, rms, nelec, kt, nalpha, nbeta;
  double gl, gu, pivmin, onenrm;  // Gerschgorin interval and norms of the last tridiagonal
};

struct WideMol {
  int m;        // molecule index in the batch
  int N, ld;    // AOs; leading dimension of the slot matrices
  int nblk;     // 64-row blocks
  long long mo; // offset of the batch's S, H0, P, W (leading dimension N)
  double *L, *Li, *Hp, *A, *Z, *C, *iw, *VW;
  double *xbuf, *d, *e, *tau, *esq, *eps, *occ, *pop, *vao, *part, *Tf, *Xp, *popp, *eshift;
  double* ws;   // CtaWs layout with maxn = 1: SCC vectors and Broyden history
  WideState* st;
  GroupSync* sync;  // [2]: column barriers, panel barriers (error flags)
  unsigned long long* flags;  // [2 * kFlagSlots]: per-CTA barrier flags (column, panel)
};

// Per-launch parameters shared by the kernels of the wide path.
struct WideCtx {
  const WideMol* mols;  // [slots]
  const int* act;       // [na] active slots of this launch
  int maxnsh, maxn, maxnat, cap;
};

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }

// Index tables in shared memory and the molecule context (one-CTA stage kernels).
__device__ MolCtx wide_context(const Batch& B, const Model& M, int m, int maxnsh, int maxn, unsigned char* raw) {
  const int a0 = B.atom_off[m], nat = B.atom_off[m + 1] - a0;
  const int sh0 = B.shell_off[m], nsh = B.shell_off[m + 1] - sh0;
  const int N = B.ao_off[m + 1] - B.ao_off[m];
  DenseTables t = dense_tables(raw, maxnsh, maxn);
  if (threadIdx.x == 0) build_index_tables(B, M, a0, nat, t.sh_atom, t.sh_k, t.sh_ao0, t.ao_sh, t.atom_sh);
  __syncthreads();
  return MolCtx{m, a0, nat, sh0, nsh, N, t.sh_atom, t.sh_k, t.sh_ao0, t.ao_sh, t.atom_sh, B.gam + B.gam_off[m]};
}

constexpr int kWideNT = 512;   // one-CTA stage kernels
constexpr int kGemmNT = 128;   // tile kernels
constexpr int kRedNT = 256;    // cooperative reduction kernel

// ------------------------------------------------------------------ orthogonaliser
// Cholesky S = L L^T in 64-column blocks (right-looking, LAPACK dpotrf order):
// the diagonal block by one CTA in shared memory (it also inverts it into the
// diagonal block of L^-1), the panel below as a product with that inverse, the
// trailing lower triangle as a rank-64 update on the tensor cores.  A pivot
// <= 1e-12 rejects the overlap, as the reference rejects an overlap
// eigenvalue <= eigen_tolerance (src/linalg.rs:193-217).
__global__ void __launch_bounds__(256) wide_chol_diag_kernel(WideCtx X, int kblk) {
  extern __shared__ __align__(16) double dsm[];
  double(*a)[65] = reinterpret_cast<double(*)[65]>(dsm);             // 64 x 65
  double(*inv)[65] = reinterpret_cast<double(*)[65]>(dsm + 64 * 65);  // 64 x 65
  __shared__ int bad;
  const WideMol& w = X.mols[X.act[blockIdx.x]];
  const int N = w.N, ld = w.ld, kb = 64 * kblk;
  if (kb >= N || w.st->status != kOk) return;
  const int nb = min(64, N - kb);
  const int tid = threadIdx.x;
  if (tid == 0) bad = 0;
  for (int idx = tid; idx < 64 * 64; idx += 256) {
    const int r = idx >> 6, c = idx & 63;
    a[r][c] = (r < nb && c <= r) ? w.L[(long long)(kb + r) * ld + kb + c] : 0.0;
    inv[r][c] = 0.0;
  }
  __syncthreads();
  for (int c = 0; c < nb; ++c) {
    if (tid == 0) {
      const double p = a[c][c];
      if (!(p > 1e-12)) bad = 1;
      a[c][c] = sqrt(fmax(p, 1e-300));
    }
    __syncthreads();
    const double lc = a[c][c];
    for (int r = c + 1 + tid; r < nb; r += 256) a[r][c] /= lc;
    __syncthreads();
    for (int idx = tid; idx < 64 * 64; idx += 256) {
      const int r = idx >> 6, q = idx & 63;
      if (r > c && q > c && q <= r && r < nb) a[r][q] -= a[r][c] * a[q][c];
    }
    __syncthreads();
  }
  // inverse of the lower-triangular block, one thread per column
  if (tid < nb) {
    const int c = tid;
    for (int r = c; r < nb; ++r) {
      double s = (r == c) ? 1.0 : 0.0;
      for (int q = c; q < r; ++q) s -= a[r][q] * inv[q][c];
      inv[r][c] = s / a[r][r];
    }
  }
  __syncthreads();
  for (int idx = tid; idx < nb * 64; idx += 256) {
    const int r = idx >> 6, c = idx & 63;
    if (c < nb) {
      w.L[(long long)(kb + r) * ld + kb + c] = c <= r ? a[r][c] : 0.0;
      w.Li[(long long)(kb + r) * ld + kb + c] = c <= r ? inv[r][c] : 0.0;
    }
  }
  if (tid == 0 && bad) w.st->status = kErrInvalidInput;
}

// L[i, kb:kb+64] = A[i, kb:kb+64] inv(L_kk)^T for the rows below the block (in place).
__global__ void __launch_bounds__(kGemmNT) wide_chol_panel_kernel(WideCtx X, int kblk) {
  extern __shared__ __align__(16) double tsm[];
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const int N = w.N, ld = w.ld, kb = 64 * kblk;
  if (kb + 64 >= N || w.st->status != kOk) return;
  const int nrt = (N - kb - 64 + 63) / 64;
  const double* L = w.L;
  const double* Li = w.Li;
  for (int t = blockIdx.x; t < nrt; t += gridDim.x) {
    const int i0 = kb + 64 + 64 * t;
    double acc[4][TileShape<kGemmNT>::kNJ][2];
    tile_zero<kGemmNT>(acc);
    auto la = [&](int i, int k) { return i < N ? L[(long long)i * ld + kb + k] : 0.0; };
    auto lb = [&](int k, int c) { return (kb + c < N && k <= c) ? Li[(long long)(kb + c) * ld + kb + k] : 0.0; };
    tile_mma<kGemmNT, false, false>(la, lb, i0, 0, 0, min(64, N - kb), acc, tsm);
    tile_for_each<kGemmNT>(acc, i0, 0, [&](int i, int c, double v) {
      if (i < N && kb + c < N) w.L[(long long)i * ld + kb + c] = v;
    });
  }
}

// Trailing update of the lower triangle: L[i][j] -= sum_t L[i][kb+t] L[j][kb+t].
__global__ void __launch_bounds__(kGemmNT) wide_chol_trail_kernel(WideCtx X, int kblk) {
  extern __shared__ __align__(16) double tsm[];
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const int N = w.N, ld = w.ld, kb = 64 * kblk, r0 = kb + 64;
  if (r0 >= N || w.st->status != kOk) return;
  const int nt = (N - r0 + 63) / 64;
  const int ntiles = nt * (nt + 1) / 2;
  double* L = w.L;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int I, J;
    lower_tile(t, I, J);
    const int i0 = r0 + 64 * I, j0 = r0 + 64 * J;
    double acc[4][TileShape<kGemmNT>::kNJ][2];
    tile_zero<kGemmNT>(acc);
    auto la = [&](int i, int k) { return i < N ? L[(long long)i * ld + kb + k] : 0.0; };
    auto lb = [&](int k, int j) { return j < N ? L[(long long)j * ld + kb + k] : 0.0; };
    tile_mma<kGemmNT, false, false>(la, lb, i0, j0, 0, 64, acc, tsm);
    tile_for_each<kGemmNT>(acc, i0, j0, [&](int i, int j, double v) {
      if (i < N && j <= i) L[(long long)i * ld + j] -= v;
    });
  }
}

// Block row I of L^-1 below the diagonal: Li[I, J] = -inv(L_II) sum_{K=J}^{I-1} L[I, K] Li[K, J].
__global__ void __launch_bounds__(kGemmNT) wide_inv_row_kernel(WideCtx X, int iblk) {
  extern __shared__ __align__(16) double tsm[];
  double* ts = tsm + kTileSmemBytes / sizeof(double);  // 64 x 65 intermediate
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const int N = w.N, ld = w.ld, ib = 64 * iblk;
  if (ib >= N || w.st->status != kOk) return;
  const double* L = w.L;
  double* Li = w.Li;
  for (int J = blockIdx.x; J < iblk; J += gridDim.x) {
    const int j0 = 64 * J;
    double acc[4][TileShape<kGemmNT>::kNJ][2];
    tile_zero<kGemmNT>(acc);
    auto la = [&](int i, int k) { return i < N ? L[(long long)i * ld + k] : 0.0; };
    auto lb = [&](int k, int j) { return Li[(long long)k * ld + j]; };
    tile_mma<kGemmNT, false, true>(la, lb, ib, j0, j0, ib, acc, tsm);
    tile_for_each<kGemmNT>(acc, 0, 0, [&](int i, int j, double v) { ts[i * 65 + j] = v; });
    __syncthreads();
    tile_zero<kGemmNT>(acc);
    auto la2 = [&](int i, int t) { return (ib + i < N && t <= i) ? Li[(long long)(ib + i) * ld + ib + t] : 0.0; };
    auto lb2 = [&](int t, int j) { return ts[t * 65 + j]; };
    tile_mma<kGemmNT, false, true>(la2, lb2, 0, 0, 0, min(64, N - ib), acc, tsm);
    tile_for_each<kGemmNT>(acc, ib, j0, [&](int i, int j, double v) {
      if (i < N) Li[(long long)i * ld + j] = -v;
    });
    __syncthreads();
  }
}

// U = L^-1 H0 (full tiles; U in the Z buffer), then H0' = U L^-T (lower tiles,
// written to both triangles so that H0' is exactly symmetric).
__global__ void __launch_bounds__(kGemmNT) wide_hp1_kernel(Batch B, WideCtx X) {
  extern __shared__ __align__(16) double tsm[];
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const int N = w.N, ld = w.ld;
  if (w.st->status != kOk) return;
  const int nt = (N + 63) / 64;
  const double* Li = w.Li;
  const double* H0 = B.H0 + w.mo;
  for (int t = blockIdx.x; t < nt * nt; t += gridDim.x) {
    const int I = t / nt, J = t - I * nt;
    double acc[4][TileShape<kGemmNT>::kNJ][2];
    tile_zero<kGemmNT>(acc);
    auto la = [&](int i, int k) { return i < N ? Li[(long long)i * ld + k] : 0.0; };
    auto lb = [&](int k, int j) { return j < N ? H0[(long long)k * N + j] : 0.0; };
    tile_mma<kGemmNT, false, true>(la, lb, 64 * I, 64 * J, 0, min(N, 64 * I + 64), acc, tsm);
    tile_for_each<kGemmNT>(acc, 64 * I, 64 * J, [&](int i, int j, double v) {
      if (i < N && j < N) w.Z[(long long)i * ld + j] = v;
    });
  }
}

__global__ void __launch_bounds__(kGemmNT) wide_hp2_kernel(WideCtx X) {
  extern __shared__ __align__(16) double tsm[];
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const int N = w.N, ld = w.ld;
  if (w.st->status != kOk) return;
  const int nt = (N + 63) / 64;
  const double* Li = w.Li;
  const double* U = w.Z;
  for (int t = blockIdx.x; t < nt * (nt + 1) / 2; t += gridDim.x) {
    int I, J;
    lower_tile(t, I, J);
    double acc[4][TileShape<kGemmNT>::kNJ][2];
    tile_zero<kGemmNT>(acc);
    auto la = [&](int i, int k) { return i < N ? U[(long long)i * ld + k] : 0.0; };
    auto lb = [&](int k, int j) { return j < N ? Li[(long long)j * ld + k] : 0.0; };
    tile_mma<kGemmNT, false, false>(la, lb, 64 * I, 64 * J, 0, min(N, 64 * J + 64), acc, tsm);
    tile_for_each<kGemmNT>(acc, 64 * I, 64 * J, [&](int i, int j, double v) {
      if (i < N && j <= i) {
        w.Hp[(long long)i * ld + j] = v;
        w.Hp[(long long)j * ld + i] = v;
      }
    });
  }
}

}  // namespace gfn1

namespace gfn1 {

// ------------------------------------------------------------------ Householder reduction
// F' (slot matrix A, full storage) to tridiagonal form d, e by the blocked
// algorithm of LAPACK dsytrd/dlatrd (lower), spread over the G CTAs of the
// molecule's group.  Per panel of nb columns the trailing rows are split
// evenly among Ga <= G CTAs (Ga shrinks with the trailing size, at least
// min_rows rows each).  Per column j (panel column l):
//   (A) x = A[j+1:, j] - V W[j]^T - W V[j]^T for the CTA's rows, partial sums of
//       |x|^2 and of V^T x, W^T x; group barrier;
//   (B) every CTA sums the partials, forms the reflector (dlarfg: beta, tau,
//       v with v_{j+1} = 1) and for its rows p = tau (A v - V (W^T v) - W (V^T v))
//       with A as of the panel start (row-wise, coalesced, from L2), the
//       partial sum of p.v; group barrier;
//   (C) alpha = -tau (p.v) / 2; w = p + alpha v is kept implicitly (W stores p
//       and alpha until the panel ends).
// At the end of a panel the CTAs finish W and all G CTAs apply the rank-2nb
// update A22 -= V W^T + W V^T to both triangles on the tensor cores.
// Reflector j is stored in column j of A below the subdiagonal (v_{j+1} = 1
// implicit), its factor in tau[j].  CTA 0 finally forms the Gerschgorin
// interval, the 1-norm bound and e^2 for the eigenvalue search.
constexpr int kMaxPanel = 32;
constexpr int kPanelCache = 8192;  // doubles of the per-CTA cache of its rows' panel vectors

struct TridiagSmall {
  double vj[kMaxPanel], wj[kMaxPanel], alpha2[kMaxPanel], vtv[kMaxPanel], wtv[kMaxPanel];
  double vr[2][kMaxPanel], wr[2][kMaxPanel];  // rows j+1 of V and corrected W (double-buffered by column)
  double tot[2 * kMaxPanel + 2];
  double red[32];
  double scal[8];
  double p1;   // p_{j+1} of the last column (w_{j+1} = p_{j+1} + alpha)
  double ajj;  // A[j][j] as of the panel start (CTA 0)
};

// Rows per CTA the cache holds for panel width nb: x, V and W of each row,
// with room left to stage one CTA's 2 nb partial sums.
__host__ __device__ inline int tridiag_rows_cap(int nb) { return (kPanelCache - 2 * nb) / (2 * nb + 1); }

__host__ __device__ inline size_t tridiag_smem_bytes(int maxn) {
  return sizeof(double) * ((size_t)maxn + 8 + kPanelCache) + kTileSmemBytes;
}
// Smallest group size whose CTAs' rows fit the cache.
__host__ __device__ inline int tridiag_min_group(int N, int nb) {
  const int cap = tridiag_rows_cap(nb);
  return (N - 1 + cap - 1) / cap;
}
// CTAs of a group of G that share a panel's nr trailing rows: about
// nr / min_rows of them, but never so few that one gets more rows than its
// cache holds (nr / min_rows rounds down, which alone would leave a CTA up to
// 2 min_rows - 1 rows), and at most G.
__host__ __device__ inline int tridiag_active(int nr, int G, int min_rows, int nb) {
  const int cap = tridiag_rows_cap(nb);
  const int need = (nr + cap - 1) / cap;
  const int want = nr / min_rows > need ? nr / min_rows : need;
  return want < 1 ? 1 : (want < G ? want : G);
}

__global__ void __launch_bounds__(kRedNT) wide_tridiag_kernel(WideCtx X, int G, int nb, int min_rows,
                                                               long long* prof, unsigned long long epoch) {
  extern __shared__ __align__(16) double sm[];
  __shared__ TridiagSmall ss;
  constexpr int NW = kRedNT / 32;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int grp = blockIdx.x / G, c = blockIdx.x - grp * G;
  const WideMol& w = X.mols[X.act[grp]];
  if (w.st->status != kOk) return;
  const int N = w.N, ld = w.ld;
  double* A = w.A;
  double* VW = w.VW;
  double* part = w.part;
  const int PS = 2 * kMaxPanel + 2;  // partial slots per CTA
  double* vs = sm;                                       // v by absolute row index (maxn + 8)
  double* tsm = sm + X.maxn + 8;                         // tensor-core tiles of the trailing update
  double* cache = tsm + kTileSmemBytes / sizeof(double);  // [xs | V rows | W rows] of the CTA's rows
  GroupSync* cs = w.sync;
  GroupSync* ps = w.sync + 1;
  unsigned long long* cflags = w.flags;
  unsigned long long* pflags = w.flags + kFlagSlots;
  unsigned long long cgen = epoch << 24, pgen = epoch << 24;  // barrier targets of this launch
  // optional phase clocks of thread 0 of the first molecule's CTA 0
  const bool timing = prof && blockIdx.x == 0 && tid == 0;
  long long tclk = timing ? clock64() : 0, tph[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  auto mark = [&](int q) {
    if (timing) {
      const long long t = clock64();
      tph[q] += t - tclk;
      tclk = t;
    }
  };
  {  // the first panel needs the most CTAs to fit its rows; the host sizes G for it
    const int nr0 = N - 1, ga0 = tridiag_active(nr0, G, min_rows, nb);
    if ((nr0 + ga0 - 1) / ga0 > tridiag_rows_cap(nb)) {
      if (tid == 0 && c == 0) w.st->status = kErrInvalidInput;
      return;
    }
  }
  bool ok = true;
  for (int k0 = 0; k0 < N - 2 && ok; k0 += nb) {
    const int nbc = min(nb, N - 2 - k0);
    const int nr = N - k0 - 1;
    const int Ga = tridiag_active(nr, G, min_rows, nb);
    const bool active = c < Ga;
    const int r0 = k0 + 1 + (int)(((long long)nr * c) / Ga), r1 = k0 + 1 + (int)(((long long)nr * (c + 1)) / Ga);
    const int R = r1 - r0;  // at most tridiag_rows_cap(nb): Ga >= nr / cap, and G fits the first panel
    double* xs = cache;              // x of the CTA's rows
    double* Vc = cache + R;          // Vc[l * R + (i - r0)]: panel reflectors of the CTA's rows
    double* Wc = Vc + (size_t)nb * R;  // Wc[l * R + (i - r0)]: p of the CTA's rows (w = p + alpha v)
    if (active) {
      // The values every CTA needs from a column's owners ride along with the
      // barrier data (x_{j+1} with the first partial sums, p_{j+1} with the
      // second), row j+1's panel vectors are fetched before the first barrier,
      // and the next column's A entries are prefetched during the
      // matrix-vector product, so that a column costs two barriers and the
      // product, not a chain of dependent loads.
      double xa[4];    // A[i][jx] for this CTA's rows i = max(r0, jx+1) + tid + 256 k
      int xa_col = -1;
      const int Rmax = (nr + Ga - 1) / Ga;
      const bool fuse_x = Rmax <= 32;  // peers' x values copied in the barrier wait
      double* pstage = cache + (size_t)(2 * nb + 1) * R;  // staging of the partial sums
      const int pst_cap = kPanelCache - (2 * nb + 1) * R;
      for (int l = 0; l < nbc; ++l) {
        const int j = k0 + l;
        const int ra = max(r0, j + 1);
        const int par = l & 1;  // ss.vr/ss.wr[par]: row j+1 of V and W (q < l); [par ^ 1]: row j
        // ---- (A) row j's V and W from the previous column (no loads)
        if (tid < l) {
          ss.vj[tid] = tid < l - 1 ? ss.vr[par ^ 1][tid] : 1.0;
          ss.wj[tid] = tid < l - 1 ? ss.wr[par ^ 1][tid] : ss.p1 + ss.alpha2[l - 1];
        } else if (tid >= 32 && tid - 32 < l) {  // row j+1's V and W, needed after the first barrier
          const int q = tid - 32;
          const double v1 = ldcg(VW + (long long)q * ld + j + 1);
          ss.vr[par][q] = v1;
          ss.wr[par][q] = ldcg(VW + (long long)(nb + q) * ld + j + 1) + ss.alpha2[q] * v1;
        } else if (tid == 64 && c == 0) {
          ss.ajj = ldcg(A + (long long)j * ld + j);
        }
        if (xa_col != j) {
          int k = 0;
          for (int i = ra + tid; i < r1 && k < 4; i += kRedNT) xa[k++] = ldcg(A + (long long)i * ld + j);
        }
        __syncthreads();
        {
          int k = 0;
          for (int i = ra + tid; i < r1; i += kRedNT) {
            double x = k < 4 ? xa[k++] : ldcg(A + (long long)i * ld + j);
            const int ri = i - r0;
            for (int q = 0; q < l; ++q) {
              const double vi = Vc[q * R + ri];
              const double wi = Wc[q * R + ri] + ss.alpha2[q] * vi;
              x -= vi * ss.wj[q] + wi * ss.vj[q];
            }
            xs[ri] = x;
            w.xbuf[i] = x;
          }
        }
        __syncthreads();
        const int nq = 2 * l + 1;  // partial sums; slot nq carries x_{j+1} from the CTA that owns row j+1
        const int rs = max(r0, j + 2);  // rows of the reflector's tail
        for (int q = wid; q < nq; q += NW) {
          double sacc = 0.0;
          if (q == 0) {
            for (int i = rs + lane; i < r1; i += 32) sacc += xs[i - r0] * xs[i - r0];
          } else if (q <= l) {
            const double* vq = Vc + (q - 1) * R;
            for (int i = rs + lane; i < r1; i += 32) sacc += vq[i - r0] * xs[i - r0];
          } else {
            const int qq = q - l - 1;
            const double* vq = Vc + qq * R;
            const double* wq = Wc + qq * R;
            const double a2 = ss.alpha2[qq];
            for (int i = rs + lane; i < r1; i += 32) sacc += (wq[i - r0] + a2 * vq[i - r0]) * xs[i - r0];
          }
          sacc = warp_sum(sacc);
          if (lane == 0) part[(long long)c * PS + q] = sacc;
        }
        if (tid == 0) part[(long long)c * PS + nq] = (j + 1 >= r0 && j + 1 < r1) ? xs[j + 1 - r0] : 0.0;
        mark(0);
        // ---- (B) totals of the partials: each waiting thread copies its peer's
        // partials (and, for few rows per CTA, its x values into v) as soon as
        // that peer has arrived
        const int nq1 = nq + 1;
        const bool fused = Ga * nq1 <= pst_cap;
        ok = flag_barrier(cflags, cs, c, Ga, ++cgen, [&](int t) {
          if (fused) {
            const double* src = part + (long long)t * PS;
#pragma unroll 8
            for (int q = 0; q < nq1; ++q) pstage[t * nq1 + q] = ldcg(src + q);
          }
          if (fuse_x) {
            const int t0 = k0 + 1 + (int)(((long long)nr * t) / Ga), t1 = k0 + 1 + (int)(((long long)nr * (t + 1)) / Ga);
            const int u0 = max(t0, j + 2);
            if (t == c) {
              for (int i = u0; i < t1; ++i) vs[i] = xs[i - r0];
            } else {
#pragma unroll 4
              for (int i = u0; i < t1; ++i) vs[i] = ldcg(w.xbuf + i);
            }
          }
        });
        if (!ok) break;
        if (fused) {
          if (tid < nq1) {
            double sacc = 0.0;
            for (int cc = 0; cc < Ga; ++cc) sacc += pstage[cc * nq1 + tid];
            ss.tot[tid] = sacc;
          }
          __syncthreads();
        } else {  // more partials than the staging holds: read them in chunks of CTAs
          const int per = max(1, pst_cap / nq1);
          double sacc = 0.0;
          for (int cb = 0; cb < Ga; cb += per) {
            const int cn = min(per, Ga - cb), tot_n = cn * nq1;
            for (int idx0 = 0; idx0 < tot_n; idx0 += 4 * kRedNT) {
              double t4[4];
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const int idx = idx0 + u * kRedNT + tid;
                t4[u] = idx < tot_n ? ldcg(part + (long long)(cb + idx / nq1) * PS + idx % nq1) : 0.0;
              }
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const int idx = idx0 + u * kRedNT + tid;
                if (idx < tot_n) pstage[idx] = t4[u];
              }
            }
            __syncthreads();
            if (tid < nq1)
              for (int cc = 0; cc < cn; ++cc) sacc += pstage[cc * nq1 + tid];
            __syncthreads();
          }
          if (tid < nq1) ss.tot[tid] = sacc;
          __syncthreads();
        }
        mark(1);
        if (tid == 0) {
          const double x0 = ss.tot[nq];
          const double sq = ss.tot[0];
          double beta = x0, tau = 0.0, scale = 0.0;
          if (sq > 0.0) {
            const double nrm = sqrt(x0 * x0 + sq);
            beta = x0 >= 0.0 ? -nrm : nrm;
            tau = (beta - x0) / beta;
            scale = 1.0 / (x0 - beta);
          }
          ss.scal[0] = tau;
          ss.scal[1] = scale;
          if (c == 0) {
            double dj = ss.ajj;
            for (int q = 0; q < l; ++q) dj -= 2.0 * ss.vj[q] * ss.wj[q];
            w.d[j] = dj;
            w.e[j] = beta;
            w.tau[j] = tau;
          }
        }
        __syncthreads();
        mark(2);
        const double tau = ss.scal[0], scale = ss.scal[1];
        const int kal = (j + 1) & ~1;
        if (fuse_x) {  // v from the x values copied during the barrier
          for (int k = kal + tid; k < N + 2; k += kRedNT)
            vs[k] = k == j + 1 ? 1.0 : ((k > j + 1 && k < N) ? scale * vs[k] : 0.0);
        } else {  // v over rows kal..N+1, four loads in flight per thread
          for (int k0v = kal; k0v < N + 2; k0v += 4 * kRedNT) {
            double t4[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int k = k0v + u * kRedNT + tid;
              t4[u] = (k > j + 1 && k < N) ? ldcg(w.xbuf + k) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int k = k0v + u * kRedNT + tid;
              if (k < N + 2) vs[k] = k == j + 1 ? 1.0 : scale * t4[u];
            }
          }
        }
        if (tid < l) {
          ss.vtv[tid] = ss.vr[par][tid] + scale * ss.tot[1 + tid];
          ss.wtv[tid] = ss.wr[par][tid] + scale * ss.tot[1 + l + tid];
        }
        __syncthreads();
        mark(3);
        // the next column's A entries for this CTA's rows (same panel only:
        // the trailing update changes A between panels)
        if (l + 1 < nbc) {
          int k = 0;
          for (int i = max(r0, j + 2) + tid; i < r1 && k < 4; i += kRedNT) xa[k++] = ldcg(A + (long long)i * ld + j + 1);
          xa_col = j + 1;
        }
        // symv over the CTA's rows: each warp takes two rows at a time, lanes
        // over column pairs, eight loads in flight per lane
        double pv = 0.0, p1 = 0.0;
        const int npair = (N - kal + 1) >> 1;
        const double2* v2 = reinterpret_cast<const double2*>(vs + kal);
        auto finish_row = [&](int i, double t) {
          const int ri = i - r0;
          if (lane < l) {
            const double vi = Vc[lane * R + ri];
            const double wi = Wc[lane * R + ri] + ss.alpha2[lane] * vi;
            t -= vi * ss.wtv[lane] + wi * ss.vtv[lane];
          }
          t = warp_sum(t);
          if (lane == 0) {
            const double p_i = tau * t;
            const double v_i = i == j + 1 ? 1.0 : scale * xs[ri];
            VW[(long long)l * ld + i] = v_i;
            VW[(long long)(nb + l) * ld + i] = p_i;
            Vc[l * R + ri] = v_i;
            Wc[l * R + ri] = p_i;
            if (i >= j + 2) A[(long long)i * ld + j] = v_i;
            pv += p_i * v_i;
            if (i == j + 1) p1 = p_i;
          }
        };
        int i = ra + 2 * wid;
        for (; i + 1 < r1; i += 2 * NW) {
          const double2* rowa = reinterpret_cast<const double2*>(A + (long long)i * ld + kal);
          const double2* rowb = reinterpret_cast<const double2*>(A + (long long)(i + 1) * ld + kal);
          double sa0 = 0.0, sa1 = 0.0, sb0 = 0.0, sb1 = 0.0;
          int p = lane;
          for (; p + 96 < npair; p += 128) {
            const double2 a0 = __ldcg(rowa + p), a1 = __ldcg(rowa + p + 32), a2 = __ldcg(rowa + p + 64),
                          a3 = __ldcg(rowa + p + 96);
            const double2 b0 = __ldcg(rowb + p), b1 = __ldcg(rowb + p + 32), b2 = __ldcg(rowb + p + 64),
                          b3 = __ldcg(rowb + p + 96);
            const double2 c0 = v2[p], c1 = v2[p + 32], c2 = v2[p + 64], c3 = v2[p + 96];
            sa0 += a0.x * c0.x + a0.y * c0.y + a2.x * c2.x + a2.y * c2.y;
            sa1 += a1.x * c1.x + a1.y * c1.y + a3.x * c3.x + a3.y * c3.y;
            sb0 += b0.x * c0.x + b0.y * c0.y + b2.x * c2.x + b2.y * c2.y;
            sb1 += b1.x * c1.x + b1.y * c1.y + b3.x * c3.x + b3.y * c3.y;
          }
          for (; p < npair; p += 32) {
            const double2 a0 = __ldcg(rowa + p), b0 = __ldcg(rowb + p), c0 = v2[p];
            sa0 += a0.x * c0.x + a0.y * c0.y;
            sb0 += b0.x * c0.x + b0.y * c0.y;
          }
          finish_row(i, sa0 + sa1);
          finish_row(i + 1, sb0 + sb1);
        }
        if (i < r1) {  // a last single row
          const double2* rowa = reinterpret_cast<const double2*>(A + (long long)i * ld + kal);
          double sa0 = 0.0, sa1 = 0.0;
          int p = lane;
          for (; p + 32 < npair; p += 64) {
            const double2 a0 = __ldcg(rowa + p), a1 = __ldcg(rowa + p + 32);
            const double2 c0 = v2[p], c1 = v2[p + 32];
            sa0 += a0.x * c0.x + a0.y * c0.y;
            sa1 += a1.x * c1.x + a1.y * c1.y;
          }
          for (; p < npair; p += 32) {
            const double2 a0 = __ldcg(rowa + p), c0 = v2[p];
            sa0 += a0.x * c0.x + a0.y * c0.y;
          }
          finish_row(i, sa0 + sa1);
        }
        if (lane == 0) {
          ss.red[wid] = pv;
          ss.red[NW + wid] = p1;
        }
        __syncthreads();
        if (tid == 0) {
          double sacc = 0.0, s1 = 0.0;
          for (int q = 0; q < NW; ++q) {
            sacc += ss.red[q];
            s1 += ss.red[NW + q];
          }
          part[(long long)c * PS + PS - 1] = sacc;
          part[(long long)c * PS + PS - 2] = s1;  // p_{j+1} from the CTA that owns row j+1, 0 elsewhere
        }
        mark(4);
        {  // ---- (C) alpha = -tau (p.v) / 2 and p_{j+1} from the Ga CTAs' rows
          double* pbuf = tsm;  // the tile area is free here
          ok = flag_barrier(cflags, cs, c, Ga, ++cgen, [&](int t) {
            pbuf[2 * t] = ldcg(part + (long long)t * PS + PS - 1);
            pbuf[2 * t + 1] = ldcg(part + (long long)t * PS + PS - 2);
          });
          if (!ok) break;
          mark(5);
          if (wid == 0) {
            double sacc = 0.0, s1 = 0.0;
            for (int cc = lane; cc < Ga; cc += 32) {
              sacc += pbuf[2 * cc];
              s1 += pbuf[2 * cc + 1];
            }
            sacc = warp_sum(sacc);
            s1 = warp_sum(s1);
            if (lane == 0) {
              ss.alpha2[l] = -0.5 * tau * sacc;
              ss.p1 = s1;
            }
          }
          __syncthreads();
        }
        mark(6);
      }
      if (ok) {  // finish W for the CTA's rows: w = p + alpha v
        for (int idx = tid; idx < nbc * R; idx += kRedNT) {
          const int l = idx / R, ri = idx - l * R, i = r0 + ri;
          if (i >= k0 + l + 1) VW[(long long)(nb + l) * ld + i] = Wc[l * R + ri] + ss.alpha2[l] * Vc[l * R + ri];
        }
      }
    }
    mark(6);
    if (!ok || !(ok = flag_barrier(pflags, ps, c, G, ++pgen, [](int) {}))) break;
    mark(7);
    // ---- trailing update A22 -= V W^T + W V^T (rows and columns >= k1)
    const int k1 = k0 + nbc;
    const int nt = (N - k1 + 63) / 64;
    for (int t = c; t < nt * nt; t += G) {
      const int I = t / nt, J = t - I * nt;
      const int i0 = k1 + 64 * I, j0 = k1 + 64 * J;
      double acc[4][TileShape<kRedNT>::kNJ][2];
      tile_zero<kRedNT>(acc);
      auto la = [&](int i, int k) {
        const int l = k < nb ? k : k - nb;
        return (i < N && l < nbc) ? ldcg(VW + (long long)k * ld + i) : 0.0;
      };
      auto lb = [&](int k, int col) {
        const int l = k < nb ? k : k - nb;
        const int src = k < nb ? nb + k : k - nb;
        return (col < N && l < nbc) ? ldcg(VW + (long long)src * ld + col) : 0.0;
      };
      tile_mma<kRedNT, true, true>(la, lb, i0, j0, 0, 2 * nb, acc, tsm);
      tile_for_each<kRedNT>(acc, i0, j0, [&](int i, int col, double v) {
        if (i < N && col < N) A[(long long)i * ld + col] -= v;
      });
    }
    mark(8);
    if (!(ok = flag_barrier(pflags, ps, c, G, ++pgen, [](int) {}))) break;
    mark(7);
  }
  if (timing)
    for (int q = 0; q < 9; ++q) atomicAdd((unsigned long long*)(prof + q), (unsigned long long)tph[q]);
  if (!ok) {
    if (tid == 0) w.st->status = kErrTimeout;
    return;
  }
  if (c != 0) return;
  // ---- last 2 x 2 block, then the bounds of the eigenvalue search
  if (tid == 0) {
    if (N >= 2) {
      w.d[N - 2] = ldcg(A + (long long)(N - 2) * ld + N - 2);
      w.e[N - 2] = ldcg(A + (long long)(N - 1) * ld + N - 2);
      w.tau[N - 2] = 0.0;
    }
    w.d[N - 1] = ldcg(A + (long long)(N - 1) * ld + N - 1);
    w.e[N - 1] = 0.0;
    w.tau[N - 1] = 0.0;
  }
  __syncthreads();
  double gl = INFINITY, gu = -INFINITY, onenrm = 0.0, emax2 = 0.0;
  for (int i = tid; i < N; i += kRedNT) {
    const double ei = i < N - 1 ? ldcg(w.e + i) : 0.0;
    const double em = i > 0 ? ldcg(w.e + i - 1) : 0.0;
    const double di = ldcg(w.d + i);
    const double off = fabs(em) + fabs(ei);
    gl = fmin(gl, di - off);
    gu = fmax(gu, di + off);
    onenrm = fmax(onenrm, fabs(di) + off);
    if (i < N - 1) {
      w.esq[i] = ei * ei;
      emax2 = fmax(emax2, ei * ei);
    }
  }
  gl = -block_max(-gl, ss.red);
  gu = block_max(gu, ss.red);
  onenrm = block_max(onenrm, ss.red);
  emax2 = block_max(emax2, ss.red);
  if (tid == 0) {
    const double pivmin = DBL_MIN * fmax(1.0, emax2);
    const double span = gu - gl;
    WideState* st = w.st;
    st->gl = gl - (2.1 * DBL_EPSILON * fabs(gl) + 4.0 * DBL_EPSILON * span + pivmin);
    st->gu = gu + (2.1 * DBL_EPSILON * fabs(gu) + 4.0 * DBL_EPSILON * span + pivmin);
    st->pivmin = pivmin;
    st->onenrm = onenrm;
  }
}

}  // namespace gfn1

namespace gfn1 {

// ------------------------------------------------------------------ set-up and rung start
// L = lower triangle of S (zeros above), L^-1 = 0, SCC state from the host-validated status.
__global__ void wide_begin_kernel(Batch B, WideCtx X) {
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const int N = w.N, ld = w.ld;
  const double* S = B.S + w.mo;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)N * ld;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx / ld), j = (int)(idx - (long long)i * ld);
    w.L[idx] = (j <= i && j < N) ? S[(long long)i * N + j] : 0.0;
    w.Li[idx] = 0.0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    WideState* st = w.st;
    st->status = B.status[w.m];
    st->converged = 0;
    st->iter = 0;
    st->nocc = 0;
  }
}

// Start of a rung of the fallback ladder: initial charges, electron counts,
// Broyden and convergence state (src/electronic.rs:1231-1239, :1274).
__global__ void __launch_bounds__(kWideNT, 1) wide_rung_kernel(Batch B, Model M, WideCtx X, SccOptions ro, int rung) {
  extern __shared__ __align__(16) unsigned char raw[];
  const WideMol& w = X.mols[X.act[blockIdx.x]];
  WideState* st = w.st;
  if (st->status != kOk) return;
  const MolCtx c = wide_context(B, M, w.m, X.maxnsh, X.maxn, raw);
  CtaWs ws = cta_ws(w.ws, 1, X.maxnsh, X.cap);
  for (int s = threadIdx.x; s < c.nsh; s += kWideNT) ws.qin[s] = B.init_q ? B.init_q[c.sh0 + s] : 0.0;
  if (threadIdx.x == 0) {
    double nref = 0.0;
    for (int s = 0; s < c.nsh; ++s) nref += M.elem[B.z[c.a0 + c.sh_atom[s]]].refocc[c.sh_k[s]];
    st->nelec = nref - B.charge[w.m];
    st->kt = fmax(ro.etemp, 0.0) * kBoltzmann;
    st->spin = ro.spin_mult > 0;
    st->nalpha = st->spin ? 0.5 * (rint(st->nelec) + (ro.spin_mult - 1)) : 0.0;
    st->nbeta = st->spin ? 0.5 * (rint(st->nelec) - (ro.spin_mult - 1)) : 0.0;
    st->nneed = min(c.N, max(1, (int)ceil(st->spin ? st->nalpha : 0.5 * st->nelec) + 8));
    st->rung = rung;
    st->converged = 0;
    st->iter = 0;
    st->bro_iter = 0;
    st->have_e = 0;
    st->have_prev = 0;
    st->nocc = 0;
    st->last_e = st->e_el = st->e2 = st->e3 = st->ts = st->mu = st->rms = 0.0;
  }
}

// ------------------------------------------------------------------ per iteration
// out[i] = sum_j G[i][j] q[j] over the molecule's nsh x nsh Coulomb matrix, one
// warp per row with the lanes along the row (coalesced), the whole CTA.
__device__ __forceinline__ void coulomb_matvec(const double* G, const double* q, int nsh, double* out) {
  constexpr int NW = kWideNT / 32;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i = wid; i < nsh; i += NW) {
    const double* gi = G + (long long)i * nsh;
    double s0 = 0.0, s1 = 0.0;
    int j = lane;
    for (; j + 32 < nsh; j += 64) {
      s0 += gi[j] * q[j];
      s1 += gi[j + 32] * q[j + 32];
    }
    if (j < nsh) s0 += gi[j] * q[j];
    const double s = warp_sum(s0 + s1);
    if (lane == 0) out[i] = s;
  }
  __syncthreads();
}

// (1) shell potential of the input charges (src/coulomb.rs:140-193), as
// stage_potential with the coalesced Coulomb product.
__global__ void __launch_bounds__(kWideNT, 1) wide_potential_kernel(Batch B, Model M, WideCtx X) {
  extern __shared__ __align__(16) unsigned char raw[];
  const WideMol& w = X.mols[X.act[blockIdx.x]];
  if (w.st->status != kOk) return;
  const MolCtx c = wide_context(B, M, w.m, X.maxnsh, X.maxn, raw);
  CtaWs ws = cta_ws(w.ws, 1, X.maxnsh, X.cap);
  const int tid = threadIdx.x;
  for (int a = tid; a < c.nat; a += kWideNT) {
    double q = 0.0;
    for (int s = c.atom_sh[a]; s < c.atom_sh[a + 1]; ++s) q += ws.qin[s];
    ws.qat[a] = q;
  }
  coulomb_matvec(c.G, ws.qin, c.nsh, ws.vsh);
  for (int i = tid; i < c.nsh; i += kWideNT) {
    const double qa = ws.qat[c.sh_atom[i]];
    ws.vsh[i] += qa * qa * M.elem[B.z[c.a0 + c.sh_atom[i]]].gam3;
  }
  __syncthreads();
  for (int i = tid; i < c.N; i += kWideNT) w.vao[i] = ws.vsh[c.ao_sh[i]];
}

// (9) output charges, energies and rms (src/electronic.rs:2173-2191,
// :3160-3200), as stage_charges_energy with the coalesced Coulomb product.
__device__ void wide_charges_energy(const Batch& B, const Model& M, const MolCtx& c, CtaWs& w, const double* pop,
                                    const double* occ, const double* eps, const double* vao, int nocc, SccShared& sh,
                                    double& e_el, double& e2, double& e3, double& rms) {
  const int tid = threadIdx.x;
  for (int s = tid; s < c.nsh; s += kWideNT) {
    const ElemTable& el = M.elem[B.z[c.a0 + c.sh_atom[s]]];
    const int k = c.sh_k[s];
    double p = 0.0;
    for (int q = 0; q < 2 * el.l[k] + 1; ++q) p += pop[c.sh_ao0[s] + q];
    w.qout[s] = el.refocc[k] - p;
  }
  double part = 0.0;
  for (int i = tid; i < c.N; i += kWideNT) part += (i < nocc ? occ[i] * eps[i] : 0.0) + vao[i] * pop[i];
  e_el = block_sum(part, sh.red);
  for (int a = tid; a < c.nat; a += kWideNT) {
    double q = 0.0;
    for (int s = c.atom_sh[a]; s < c.atom_sh[a + 1]; ++s) q += w.qout[s];
    w.qat[a] = q;
  }
  coulomb_matvec(c.G, w.qout, c.nsh, w.vout);  // G q_out (the third-order part is added below)
  double p2 = 0.0, p3 = 0.0, pr = 0.0;
  for (int i = tid; i < c.nsh; i += kWideNT) {
    const double v = w.vout[i];
    p2 += w.qout[i] * v;
    const int a = c.sh_atom[i];
    const double qa = w.qat[a];
    w.vout[i] = v + qa * qa * M.elem[B.z[c.a0 + a]].gam3;
    const double r = w.qout[i] - w.qin[i];
    pr += r * r;
  }
  for (int a = tid; a < c.nat; a += kWideNT) {
    const double qa = w.qat[a];
    p3 += qa * qa * qa * M.elem[B.z[c.a0 + a]].gam3 / 3.0;
  }
  e2 = 0.5 * block_sum(p2, sh.red);
  e3 = block_sum(p3, sh.red);
  rms = c.nsh ? sqrt(block_sum(pr, sh.red) / c.nsh) : 0.0;
}

// (2) F' = H0' - 1/2 (M + M^T), M = L^-1 diag(v) L lower triangular
// (src/electronic.rs:3133-3158 in the orthonormal basis), written to both
// triangles of the working matrix.
__global__ void __launch_bounds__(kGemmNT) wide_fock_kernel(WideCtx X) {
  extern __shared__ __align__(16) double tsm[];
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  if (w.st->status != kOk) return;
  const int N = w.N, ld = w.ld, nt = (N + 63) / 64;
  const double *Li = w.Li, *L = w.L, *vao = w.vao, *Hp = w.Hp;
  double* A = w.A;
  for (int t = blockIdx.x; t < nt * (nt + 1) / 2; t += gridDim.x) {
    int I, J;
    lower_tile(t, I, J);
    double acc[4][TileShape<kGemmNT>::kNJ][2];
    tile_zero<kGemmNT>(acc);
    auto la = [&](int i, int k) { return i < N ? Li[(long long)i * ld + k] : 0.0; };
    auto lb = [&](int k, int j) { return j < N ? vao[k] * L[(long long)k * ld + j] : 0.0; };
    tile_mma<kGemmNT, false, true>(la, lb, 64 * I, 64 * J, 64 * J, min(N, 64 * I + 64), acc, tsm);
    tile_for_each<kGemmNT>(acc, 64 * I, 64 * J, [&](int i, int j, double mv) {
      if (i < N && j <= i) {
        const double f = Hp[(long long)i * ld + j] - (i == j ? mv : 0.5 * mv);
        A[(long long)i * ld + j] = f;
        A[(long long)j * ld + i] = f;
      }
    });
  }
}

// Level shift F += b (S - S P_prev S / 2) (src/electronic.rs:2125-2137), in the
// orthonormal basis F' += b (I - Z f Z^T / 2) with the previous iteration's
// eigenvectors Z and occupations f.
__global__ void __launch_bounds__(kGemmNT) wide_shift_kernel(WideCtx X, double lshift) {
  extern __shared__ __align__(16) double tsm[];
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const WideState* st = w.st;
  if (st->status != kOk || !st->have_prev) return;
  const int N = w.N, ld = w.ld, nt = (N + 63) / 64, nocc = st->nocc;
  const double *Z = w.Z, *occ = w.occ;
  double* A = w.A;
  for (int t = blockIdx.x; t < nt * (nt + 1) / 2; t += gridDim.x) {
    int I, J;
    lower_tile(t, I, J);
    double acc[4][TileShape<kGemmNT>::kNJ][2];
    tile_zero<kGemmNT>(acc);
    auto la = [&](int i, int k) { return i < N ? Z[(long long)i * ld + k] * occ[k] : 0.0; };
    auto lb = [&](int k, int j) { return j < N ? Z[(long long)j * ld + k] : 0.0; };
    tile_mma<kGemmNT, false, false>(la, lb, 64 * I, 64 * J, 0, nocc, acc, tsm);
    tile_for_each<kGemmNT>(acc, 64 * I, 64 * J, [&](int i, int j, double sp) {
      if (i < N && j <= i) {
        const double val = lshift * ((i == j ? 1.0 : 0.0) - 0.5 * sp);
        A[(long long)i * ld + j] += val;
        if (i != j) A[(long long)j * ld + i] += val;
      }
    });
  }
}

// (4) eigenvalues 0..nneed-1 and N-1 (one thread each), d and e^2 staged in
// shared memory.
constexpr int kEigNT = 32;  // one warp per CTA: the searches spread over the SMs
__global__ void __launch_bounds__(kEigNT) wide_eigval_kernel(WideCtx X) {
  extern __shared__ __align__(16) double dsm[];
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const WideState* st = w.st;
  if (st->status != kOk) return;
  const int N = w.N, nneed = st->nneed;
  const int nlist = nneed < N ? nneed + 1 : N;
  if (blockIdx.x * kEigNT >= nlist) return;
  double* d = dsm;
  double* esq = dsm + N;
  for (int i = threadIdx.x; i < N; i += kEigNT) {
    d[i] = w.d[i];
    esq[i] = i < N - 1 ? w.esq[i] : 0.0;
  }
  __syncthreads();
  const int slot = blockIdx.x * kEigNT + threadIdx.x;
  if (slot < nlist) {  // from the previous iteration's eigenvalue once the rung has one
    const int k = slot < nneed ? slot : N - 1;
    w.eps[k] = eigenvalue_k(d, esq, N, k, st->gl, st->gu, st->pivmin, 4.0 * DBL_EPSILON * st->onenrm, w.eps[k],
                            st->iter > 0);
  }
}

// (5) occupations (src/electronic.rs:3815-3921, spin channels :3930-4045); when
// the known eigenvalues do not decide them, the CTA computes every eigenvalue
// and repeats.  Also the count of orbitals with occupation above 1e-30.
__global__ void __launch_bounds__(kWideNT, 1) wide_fermi_kernel(WideCtx X) {
  __shared__ SccShared sh;
  const WideMol& w = X.mols[X.act[blockIdx.x]];
  WideState* st = w.st;
  if (st->status != kOk) return;
  const int N = w.N, tid = threadIdx.x;
  const double nelec = st->nelec, kt = st->kt;
  int nneed = st->nneed;
  for (int attempt = 0; attempt < 2; ++attempt) {
    if (st->spin) {
      spin_channel_occupations<kWideNT>(w.eps, N, nneed, st->nalpha, st->nbeta, kt, w.occ, w.pop, sh);
    } else if (kt > 0.0 && nelec > 0.0 && nelec < 2.0 * N) {
      double fm, ft;
      bool amb;
      fermi_cta<kWideNT, 2>(w.eps, N, nneed, nelec, kt, w.occ, sh, fm, ft, amb);
      if (tid == 0) {
        sh.scal[1] = fm;
        sh.scal[2] = ft;
        sh.iscal[2] = amb ? 1 : 0;
      }
    } else if (tid < 32) {
      double fm, ft;
      bool amb;
      fermi_warp<2>(w.eps, N, nneed, nelec, kt, w.occ, fm, ft, amb);
      if (tid == 0) {
        sh.scal[1] = fm;
        sh.scal[2] = ft;
        sh.iscal[2] = amb ? 1 : 0;
      }
    }
    __syncthreads();
    if (!sh.iscal[2] || nneed == N) break;
    // the rest of the spectrum, this CTA alone (rare: wide Fermi windows)
    const double atol = 4.0 * DBL_EPSILON * st->onenrm;
    for (int k = nneed + tid; k < N - 1; k += kWideNT)
      w.eps[k] = eigenvalue_k(w.d, w.esq, N, k, st->gl, st->gu, st->pivmin, atol);
    nneed = N;
    __syncthreads();
  }
  int nocc_loc = 0;
  for (int i = tid; i < N; i += kWideNT)
    if ((i < nneed || i == N - 1) && w.occ[i] > 1e-30) nocc_loc = max(nocc_loc, i + 1);
  const int nocc = (int)block_max((double)nocc_loc, sh.red);
  if (tid == 0) {
    st->mu = sh.scal[1];
    st->ts = sh.scal[2];
    st->nocc = nocc;
    st->nneed = nneed;
  }
}

// (6) inverse iteration for the occupied eigenvectors of the tridiagonal (one
// thread per cluster of eigenvalues closer than ortol_rel |T|_1, modified
// Gram-Schmidt inside a cluster), columns of Z with stride ld.
__global__ void __launch_bounds__(64) wide_inviter_kernel(WideCtx X, double ortol_rel, int* stats) {
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const WideState* st = w.st;
  if (st->status != kOk) return;
  const int N = w.N, ld = w.ld, nocc = st->nocc;
  const int j = blockIdx.x * 64 + threadIdx.x;
  if (j >= nocc) return;
  const double* eps = w.eps;
  const double onenrm = st->onenrm;
  const double ortol = ortol_rel * onenrm;
  const double tiny = DBL_EPSILON * fmax(onenrm, 1e-300);
  if (!(j == 0 || eps[j] - eps[j - 1] > ortol)) return;
  int jend = j + 1;
  while (jend < nocc && eps[jend] - eps[jend - 1] <= ortol) ++jend;
  if (stats) {
    atomicMax(stats, jend - j);
    if (jend - j > 1) atomicAdd(stats + 1, 1);
  }
  double* Z = w.Z;
  double* wsv = w.iw + j;
  double lam_prev = -INFINITY;
  for (int jj = j; jj < jend; ++jj) {
    double lam = eps[jj];
    const double pert = 10.0 * DBL_EPSILON * fmax(fabs(lam), onenrm);
    if (jj > j && lam - lam_prev < pert) lam = lam_prev + pert;
    lam_prev = lam;
    double* x = Z + jj;
    if (jend - j == 1) {
      // isolated: the start vector's forward elimination runs with the
      // factorisation, the two solves are not normalised in between (growth
      // below 1e40), and the second one returns |x|^2
      const double cur = tri_factor_rhs(w.d, w.e, N, lam, tiny, wsv, ld, x, ld, (unsigned)jj);
      tri_back(wsv, N, ld, x, ld, cur);
      const double nrm = tri_solve(wsv, N, ld, x, ld);
      const double inv = 1.0 / sqrt(fmax(nrm, 1e-300));
#pragma unroll 8
      for (int i = 0; i < N; ++i) x[(long long)i * ld] *= inv;
      continue;
    }
    tri_factor(w.d, w.e, N, lam, tiny, wsv, ld);
#pragma unroll 8
    for (int i = 0; i < N; ++i) x[(long long)i * ld] = hash_unit(i, jj) + 1e-3;
    const int nit = 4;
    for (int it = 0; it < nit; ++it) {
      tri_solve(wsv, N, ld, x, ld);
      for (int q = j; q < jj; ++q) {
        double dot = 0.0;
#pragma unroll 8
        for (int i = 0; i < N; ++i) dot += Z[(long long)i * ld + q] * x[(long long)i * ld];
#pragma unroll 8
        for (int i = 0; i < N; ++i) x[(long long)i * ld] -= dot * Z[(long long)i * ld + q];
      }
      double nrm = 0.0;
#pragma unroll 8
      for (int i = 0; i < N; ++i) nrm += x[(long long)i * ld] * x[(long long)i * ld];
      const double inv = 1.0 / sqrt(fmax(nrm, 1e-300));
#pragma unroll 8
      for (int i = 0; i < N; ++i) x[(long long)i * ld] *= inv;
    }
  }
}

// (7) back-transformation Z := Q Z, Q = H_0 ... H_{N-3}, in blocks of 64
// reflectors applied last block first as Q_b = I - V T V^T (compact WY,
// LAPACK dlarft forward/columnwise).  V(i, a) of block b: reflector kb + a,
// 1 at row kb + a + 1, A[i][kb + a] below, 0 above.
__device__ __forceinline__ double refl(const double* A, int ld, int N, int kb, int a, int i) {
  const int r = kb + a + 1;
  return (i == r && r < N) ? 1.0 : ((i > r && i < N) ? A[(long long)i * ld + kb + a] : 0.0);
}

// T factors of every block: V^T V on the tensor cores, then the triangular
// recurrence T[0:j, j] = -tau_j T[0:j, 0:j] (V^T V)[0:j, j], T_jj = tau_j.
__global__ void __launch_bounds__(kGemmNT) wide_bt_t_kernel(WideCtx X) {
  extern __shared__ __align__(16) double tsm[];
  double* G = tsm + kTileSmemBytes / sizeof(double);  // 64 x 65
  double* T = G + 64 * 65;                           // 64 x 65
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  if (w.st->status != kOk) return;
  const int N = w.N, ld = w.ld;
  const int nref = N - 2, nblk = (nref + 63) / 64;
  const int b = blockIdx.x;
  if (b >= nblk) return;
  const int kb = 64 * b, nbk = min(64, nref - kb);
  const double* A = w.A;
  double acc[4][TileShape<kGemmNT>::kNJ][2];
  tile_zero<kGemmNT>(acc);
  auto la = [&](int a, int i) { return a < nbk ? refl(A, ld, N, kb, a, i) : 0.0; };
  auto lb = [&](int i, int bb) { return bb < nbk ? refl(A, ld, N, kb, bb, i) : 0.0; };
  tile_mma<kGemmNT, true, true>(la, lb, 0, 0, kb + 1, N, acc, tsm);
  tile_for_each<kGemmNT>(acc, 0, 0, [&](int a, int bb, double v) { G[a * 65 + bb] = v; });
  for (int idx = threadIdx.x; idx < 64 * 65; idx += kGemmNT) T[idx] = 0.0;
  __syncthreads();
  for (int j = 0; j < nbk; ++j) {
    const double tj = w.tau[kb + j];
    double s = 0.0;
    if (threadIdx.x < j)
      for (int q = threadIdx.x; q < j; ++q) s += T[threadIdx.x * 65 + q] * G[q * 65 + j];
    __syncthreads();
    if (threadIdx.x < j) T[threadIdx.x * 65 + j] = -tj * s;
    if (threadIdx.x == j) T[j * 65 + j] = tj;
    __syncthreads();
  }
  double* Tf = w.Tf + (long long)b * 64 * 64;
  for (int idx = threadIdx.x; idx < 64 * 64; idx += kGemmNT) Tf[idx] = T[(idx >> 6) * 65 + (idx & 63)];
}

// Xp[s] = V_b^T Z for the rows of split s (tiles of 64 columns of Z).
__global__ void __launch_bounds__(kGemmNT) wide_bt_x_kernel(WideCtx X, int b, int ksplit) {
  extern __shared__ __align__(16) double tsm[];
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const WideState* st = w.st;
  if (st->status != kOk) return;
  const int N = w.N, ld = w.ld, nocc = st->nocc;
  const int nref = N - 2;
  const int kb = 64 * b;
  if (kb >= nref || nocc <= 0) return;
  const int nbk = min(64, nref - kb);
  const int nct = (nocc + 63) / 64;
  const int rows = N - kb - 1, chunk = (rows + ksplit - 1) / ksplit;
  const double *A = w.A, *Z = w.Z;
  for (int t = blockIdx.x; t < nct * ksplit; t += gridDim.x) {
    const int ct = t / ksplit, s = t - ct * ksplit;
    const int r0 = kb + 1 + s * chunk, r1 = min(N, r0 + chunk);
    double acc[4][TileShape<kGemmNT>::kNJ][2];
    tile_zero<kGemmNT>(acc);
    auto la = [&](int a, int i) { return a < nbk ? refl(A, ld, N, kb, a, i) : 0.0; };
    auto lb = [&](int i, int col) { return col < nocc ? Z[(long long)i * ld + col] : 0.0; };
    if (r0 < r1) tile_mma<kGemmNT, true, true>(la, lb, 0, 64 * ct, r0, r1, acc, tsm);
    tile_for_each<kGemmNT>(acc, 0, 64 * ct, [&](int a, int col, double v) {
      if (col < nocc) w.Xp[((long long)s * 64 + a) * ld + col] = v;
    });
  }
}

// Y = T (sum_s Xp[s]) into Xp[0] (tiles of 64 columns).
__global__ void __launch_bounds__(kGemmNT) wide_bt_y_kernel(WideCtx X, int b, int ksplit) {
  extern __shared__ __align__(16) double tsm[];
  double* Xs = tsm + kTileSmemBytes / sizeof(double);  // 64 x 65
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const WideState* st = w.st;
  if (st->status != kOk) return;
  const int N = w.N, ld = w.ld, nocc = st->nocc;
  if (64 * b >= N - 2 || nocc <= 0) return;
  const int nct = (nocc + 63) / 64;
  const double* Tf = w.Tf + (long long)b * 64 * 64;
  for (int ct = blockIdx.x; ct < nct; ct += gridDim.x) {
    for (int idx = threadIdx.x; idx < 64 * 64; idx += kGemmNT) {
      const int a = idx >> 6, col = 64 * ct + (idx & 63);
      double s = 0.0;
      if (col < nocc)
        for (int q = 0; q < ksplit; ++q) s += w.Xp[((long long)q * 64 + a) * ld + col];
      Xs[a * 65 + (idx & 63)] = s;
    }
    __syncthreads();
    double acc[4][TileShape<kGemmNT>::kNJ][2];
    tile_zero<kGemmNT>(acc);
    auto la = [&](int a, int q) { return Tf[a * 64 + q]; };
    auto lb = [&](int q, int cl) { return Xs[q * 65 + cl]; };
    tile_mma<kGemmNT, false, true>(la, lb, 0, 0, 0, 64, acc, tsm);
    tile_for_each<kGemmNT>(acc, 0, 0, [&](int a, int cl, double v) {
      const int col = 64 * ct + cl;
      if (col < nocc) w.Xp[(long long)a * ld + col] = v;
    });
    __syncthreads();
  }
}

// Z[kb+1:, :] -= V_b Y (tiles of 64 rows x 64 columns).
__global__ void __launch_bounds__(kGemmNT) wide_bt_upd_kernel(WideCtx X, int b) {
  extern __shared__ __align__(16) double tsm[];
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const WideState* st = w.st;
  if (st->status != kOk) return;
  const int N = w.N, ld = w.ld, nocc = st->nocc;
  const int nref = N - 2, kb = 64 * b;
  if (kb >= nref || nocc <= 0) return;
  const int nbk = min(64, nref - kb);
  const int r0 = kb + 1;
  const int nrt = (N - r0 + 63) / 64, nct = (nocc + 63) / 64;
  const double* A = w.A;
  double* Z = w.Z;
  const double* Y = w.Xp;
  for (int t = blockIdx.x; t < nrt * nct; t += gridDim.x) {
    const int rt = t / nct, ct = t - rt * nct;
    const int i0 = r0 + 64 * rt, c0 = 64 * ct;
    double acc[4][TileShape<kGemmNT>::kNJ][2];
    tile_zero<kGemmNT>(acc);
    auto la = [&](int i, int a) { return a < nbk ? refl(A, ld, N, kb, a, i) : 0.0; };
    auto lb = [&](int a, int col) { return col < nocc ? Y[(long long)a * ld + col] : 0.0; };
    tile_mma<kGemmNT, false, true>(la, lb, i0, c0, 0, nbk, acc, tsm);
    tile_for_each<kGemmNT>(acc, i0, c0, [&](int i, int col, double v) {
      if (i < N && col < nocc) Z[(long long)i * ld + col] -= v;
    });
  }
}

// (8) C = L^-T Z, D = L Z and the partial AO populations
// popp[it][mu] = sum_{i in tile it} f_i C[mu][i] D[mu][i]  ((S P)_mu,mu).
__global__ void __launch_bounds__(kGemmNT) wide_cd_kernel(WideCtx X) {
  extern __shared__ __align__(16) double tsm[];
  double* Ds = tsm + kTileSmemBytes / sizeof(double);  // 64 x 65
  double* Cs = Ds + 64 * 65;
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const WideState* st = w.st;
  if (st->status != kOk) return;
  const int N = w.N, ld = w.ld, nocc = st->nocc;
  const int nmt = (N + 63) / 64, nit = (nocc + 63) / 64;
  const double *L = w.L, *Li = w.Li, *Z = w.Z, *occ = w.occ;
  for (int t = blockIdx.x; t < nmt * nit; t += gridDim.x) {
    const int mt = t / nit, it = t - mt * nit;
    const int m0 = 64 * mt, c0 = 64 * it;
    double acc[4][TileShape<kGemmNT>::kNJ][2];
    tile_zero<kGemmNT>(acc);
    auto la = [&](int mu, int k) { return mu < N ? L[(long long)mu * ld + k] : 0.0; };
    auto lz = [&](int k, int col) { return col < nocc ? Z[(long long)k * ld + col] : 0.0; };
    tile_mma<kGemmNT, false, true>(la, lz, m0, c0, 0, min(N, m0 + 64), acc, tsm);
    tile_for_each<kGemmNT>(acc, 0, 0, [&](int r, int cl, double v) { Ds[r * 65 + cl] = v; });
    tile_zero<kGemmNT>(acc);
    auto li = [&](int mu, int k) { return mu < N ? Li[(long long)k * ld + mu] : 0.0; };
    tile_mma<kGemmNT, true, true>(li, lz, m0, c0, m0, N, acc, tsm);
    tile_for_each<kGemmNT>(acc, 0, 0, [&](int r, int cl, double v) {
      Cs[r * 65 + cl] = v;
      const int mu = m0 + r, col = c0 + cl;
      if (mu < N && col < nocc) w.C[(long long)mu * ld + col] = v;
    });
    __syncthreads();
    if (threadIdx.x < 64 && m0 + threadIdx.x < N) {
      const int r = threadIdx.x;
      double s = 0.0;
      for (int cl = 0; cl < 64 && c0 + cl < nocc; ++cl) s += occ[c0 + cl] * Cs[r * 65 + cl] * Ds[r * 65 + cl];
      w.popp[(long long)it * ld + m0 + r] = s;
    }
    __syncthreads();
  }
}

// With a level shift sum(f eps) is not tr(F P): partial sums of
// E_el = tr(H0 P) = sum_k f_k z_k^T H0' z_k per tile of H0' Z.
__global__ void __launch_bounds__(kGemmNT) wide_eshift_kernel(WideCtx X) {
  extern __shared__ __align__(16) double tsm[];
  __shared__ double red[4];
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const WideState* st = w.st;
  if (st->status != kOk) return;
  const int N = w.N, ld = w.ld, nocc = st->nocc;
  const int nrt = (N + 63) / 64, nct = (nocc + 63) / 64;
  const double *Hp = w.Hp, *Z = w.Z, *occ = w.occ;
  for (int t = blockIdx.x; t < nrt * nct; t += gridDim.x) {
    const int rt = t / nct, ct = t - rt * nct;
    double acc[4][TileShape<kGemmNT>::kNJ][2];
    tile_zero<kGemmNT>(acc);
    auto la = [&](int i, int k) { return i < N ? Hp[(long long)i * ld + k] : 0.0; };
    auto lb = [&](int k, int col) { return col < nocc ? Z[(long long)k * ld + col] : 0.0; };
    tile_mma<kGemmNT, false, true>(la, lb, 64 * rt, 64 * ct, 0, N, acc, tsm);
    double part = 0.0;
    tile_for_each<kGemmNT>(acc, 64 * rt, 64 * ct, [&](int i, int col, double v) {
      if (i < N && col < nocc) part += occ[col] * Z[(long long)i * ld + col] * v;
    });
    part = warp_sum(part);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) w.eshift[t] = red[0] + red[1] + red[2] + red[3];
    __syncthreads();
  }
}

// (9)+(10) populations, output charges, energies, convergence test and mixing.
__global__ void __launch_bounds__(kWideNT, 1) wide_energy_mix_kernel(Batch B, Model M, WideCtx X, SccOptions ro,
                                                                     double lshift) {
  extern __shared__ __align__(16) unsigned char raw[];
  __shared__ SccShared sh;
  const WideMol& w = X.mols[X.act[blockIdx.x]];
  WideState* st = w.st;
  if (st->status != kOk) return;
  const MolCtx c = wide_context(B, M, w.m, X.maxnsh, X.maxn, raw);
  CtaWs ws = cta_ws(w.ws, 1, X.maxnsh, X.cap);
  const int N = w.N, ld = w.ld, nocc = st->nocc;
  const int nit = (nocc + 63) / 64;
  for (int mu = threadIdx.x; mu < N; mu += kWideNT) {
    double s = 0.0;
    for (int it = 0; it < nit; ++it) s += w.popp[(long long)it * ld + mu];
    w.pop[mu] = s;
  }
  __syncthreads();
  double e_el, e2, e3, rms;
  wide_charges_energy(B, M, c, ws, w.pop, w.occ, w.eps, w.vao, nocc, sh, e_el, e2, e3, rms);
  if (lshift != 0.0) {
    const int ntile = ((N + 63) / 64) * nit;
    double part = 0.0;
    for (int t = threadIdx.x; t < ntile; t += kWideNT) part += w.eshift[t];
    e_el = block_sum(part, sh.red);
  }
  const double escc = e_el + e2 + e3 + st->ts;
  const double err = st->have_e ? fabs(escc - st->last_e) : INFINITY;
  const bool converged = err < ro.energy_tol && rms < ro.charge_tol;
  __syncthreads();
  if (!converged) {
    int bro = st->bro_iter;
    stage_mix<kWideNT>(ro, c, ws, X.cap, bro, sh);
    if (threadIdx.x == 0) st->bro_iter = bro;
  }
  if (threadIdx.x == 0) {
    st->e_el = e_el;
    st->e2 = e2;
    st->e3 = e3;
    st->rms = rms;
    st->iter += 1;
    st->converged = converged ? 1 : 0;
    if (!converged) {
      st->last_e = escc;
      st->have_e = 1;
      st->have_prev = lshift != 0.0 ? 1 : 0;
    }
  }
}

// ------------------------------------------------------------------ results
// P = C f C^T and W = C f eps C^T of the last diagonalisation (src/linalg.rs:
// 243-273), lower tiles written to both triangles.
__global__ void __launch_bounds__(kGemmNT) wide_pw_kernel(Batch B, WideCtx X) {
  extern __shared__ __align__(16) double tsm[];
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  const WideState* st = w.st;
  if (st->status != kOk) return;
  const int N = w.N, ld = w.ld, nocc = st->nocc, nt = (N + 63) / 64;
  const double *C = w.C, *occ = w.occ, *eps = w.eps;
  double* P = B.P + w.mo;
  double* W = B.W + w.mo;
  for (int t = blockIdx.x; t < nt * (nt + 1) / 2; t += gridDim.x) {
    int I, J;
    lower_tile(t, I, J);
    for (int pass = 0; pass < 2; ++pass) {
      double acc[4][TileShape<kGemmNT>::kNJ][2];
      tile_zero<kGemmNT>(acc);
      auto la = [&](int i, int k) {
        return i < N ? C[(long long)i * ld + k] * (pass ? occ[k] * eps[k] : occ[k]) : 0.0;
      };
      auto lb = [&](int k, int j) { return j < N ? C[(long long)j * ld + k] : 0.0; };
      tile_mma<kGemmNT, false, false>(la, lb, 64 * I, 64 * J, 0, nocc, acc, tsm);
      double* out = pass ? W : P;
      tile_for_each<kGemmNT>(acc, 64 * I, 64 * J, [&](int i, int j, double v) {
        if (i < N && j <= i) {
          out[(long long)i * N + j] = v;
          out[(long long)j * N + i] = v;
        }
      });
    }
  }
}

__global__ void __launch_bounds__(kWideNT, 1) wide_results_kernel(Batch B, Model M, WideCtx X) {
  extern __shared__ __align__(16) unsigned char raw[];
  const WideMol& w = X.mols[X.act[blockIdx.x]];
  const WideState* st = w.st;
  if (st->status != kOk) {
    if (threadIdx.x == 0) {
      B.status[w.m] = st->status;
      B.iterations[w.m] = 0;
    }
    return;
  }
  const MolCtx c = wide_context(B, M, w.m, X.maxnsh, X.maxn, raw);
  CtaWs ws = cta_ws(w.ws, 1, X.maxnsh, X.cap);
  stage_results<kWideNT>(B, c, ws, st->iter, st->converged != 0, st->e_el, st->e2, st->e3, st->ts, st->mu);
  if (B.rung && threadIdx.x == 0) B.rung[w.m] = st->converged ? st->rung : -1;
  if (B.orb_eps) {
    const int ao0 = B.ao_off[w.m], N = w.N, nneed = st->nneed;
    for (int i = threadIdx.x; i < N; i += kWideNT) {
      B.orb_eps[ao0 + i] = (i < nneed || i == N - 1) ? w.eps[i] : __longlong_as_double(0x7ff8000000000000LL);
      B.orb_occ[ao0 + i] = w.occ[i];
    }
  }
}

}  // namespace gfn1

// ================================================================== host side
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace gfn1 {

constexpr int kWideMaxG = 1024;   // CTAs per molecule (partial-sum slots)
constexpr int kWideMaxSplit = 8;  // row splits of the back-transformation's V^T Z

struct WideSlotLayout {
  int ld;
  long long L, Li, Hp, A, Z, C, iw, VW, xbuf, d, e, tau, esq, eps, occ, pop, vao, part, Tf, Xp, popp, eshift, ws;
  long long total;
};

inline long long wide_align4(long long x) { return (x + 31) & ~31LL; }  // 256-byte regions

inline WideSlotLayout wide_slot_layout(int N, int nsh, int nat, int cap) {
  WideSlotLayout s;
  s.ld = (N + 4) & ~3;  // a multiple of four above N: 32-byte rows, one spare column
  const long long n2 = (long long)N * s.ld, nv = s.ld + 4;
  const long long nblk = (N + 63) / 64 + 1;
  long long o = 0;
  auto take = [&](long long nd) {
    const long long at = o;
    o = wide_align4(o + nd);
    return at;
  };
  s.L = take(n2);
  s.Li = take(n2);
  s.Hp = take(n2);
  s.A = take(n2);
  s.Z = take(n2);
  s.C = take(n2);
  s.iw = take(5 * n2);
  s.VW = take(2LL * kMaxPanel * s.ld);
  s.xbuf = take(nv);
  s.d = take(nv);
  s.e = take(nv);
  s.tau = take(nv);
  s.esq = take(nv);
  s.eps = take(nv);
  s.occ = take(nv);
  s.pop = take(nv);
  s.vao = take(nv);
  s.part = take((long long)kWideMaxG * (2 * kMaxPanel + 2));
  s.Tf = take(nblk * 64 * 64);
  s.Xp = take((long long)kWideMaxSplit * 64 * s.ld);
  s.popp = take(nblk * s.ld);
  s.eshift = take(nblk * nblk);
  s.ws = take(cta_ws_size(1, std::max(nsh, 1), cap, std::max(nat, 1)));
  s.total = o;
  return s;
}

// Parameters the autotuner picks per size class: panel width of the
// reduction, minimum rows per CTA (bounds the group size as the trailing
// matrix shrinks) and the measured reduction time.
struct WidePlan {
  int nb = 16, min_rows = 16;
  float tridiag_ms = 0.f;
  bool tuned = false;
};

struct WideRuntime {
  std::vector<WideMol> mols;  // host copies of the slot descriptors
  WideMol* d_mols = nullptr;
  int* d_act = nullptr;
  int* h_act = nullptr;
  WideState* d_state = nullptr;
  WideState* h_state = nullptr;
  GroupSync* d_sync = nullptr;
  unsigned long long* d_flags = nullptr;  // [2 * kFlagSlots] per slot, zero at bind
  int* d_stats = nullptr;  // timing mode: cluster statistics and reduction phase clocks
  int capacity = 0;  // slots the buffers above hold
  WidePlan plan;     // plan of the last run
  int group = 0;     // CTAs per molecule in the last run
};

static std::mutex g_wide_tune_mu;
static std::map<long long, WidePlan> g_wide_plans;  // (device, size class, concurrency class) -> plan

static cudaError_t wide_configure(int dev) {
  static int configured = -1;
  if (configured == dev) return cudaSuccess;
  const int big = 200 * 1024;
  const void* ks[] = {(const void*)wide_chol_diag_kernel,  (const void*)wide_chol_panel_kernel, (const void*)wide_chol_trail_kernel,
                      (const void*)wide_inv_row_kernel,    (const void*)wide_hp1_kernel,
                      (const void*)wide_hp2_kernel,        (const void*)wide_fock_kernel,
                      (const void*)wide_shift_kernel,      (const void*)wide_tridiag_kernel,
                      (const void*)wide_eigval_kernel,     (const void*)wide_bt_t_kernel,
                      (const void*)wide_bt_x_kernel,       (const void*)wide_bt_y_kernel,
                      (const void*)wide_bt_upd_kernel,     (const void*)wide_cd_kernel,
                      (const void*)wide_eshift_kernel,     (const void*)wide_pw_kernel,
                      (const void*)wide_rung_kernel,       (const void*)wide_potential_kernel,
                      (const void*)wide_energy_mix_kernel, (const void*)wide_results_kernel};
  for (const void* k : ks) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e != cudaSuccess) return e;
  }
  configured = dev;
  return cudaSuccess;
}

static std::atomic<unsigned long long> g_tridiag_epoch{0};  // launches of the reduction (barrier flag generations)

static cudaError_t launch_tridiag(const WideCtx& X, int na, int G, int nb, int min_rows, size_t smem, cudaStream_t st,
                                  long long* prof) {
  WideCtx x = X;
  unsigned long long epoch = g_tridiag_epoch.fetch_add(1) + 1;
  void* args[] = {(void*)&x, (void*)&G, (void*)&nb, (void*)&min_rows, (void*)&prof, (void*)&epoch};
  return cudaLaunchCooperativeKernel((const void*)wide_tridiag_kernel, dim3(na * G), dim3(kRedNT), args, smem, st);
}

// The reduction of the na molecules of X.act: G CTAs per molecule, at least
// the group that fits the row cache, at most `gcap`; as many molecules per
// cooperative launch as the resident CTAs allow.  Returns the group size of
// the first launch in *group.
static cudaError_t tridiag_all(const WideCtx& X, int na, int maxn, int nb, int min_rows, int capacity, int gcap,
                               size_t smem, cudaStream_t st, int* group, long long* prof = nullptr) {
  const int gmin = tridiag_min_group(maxn, nb);
  if (gmin > capacity) return cudaErrorInvalidValue;
  const int per = std::max(1, capacity / gmin);
  for (int a0 = 0; a0 < na; a0 += per) {
    const int nn = std::min(per, na - a0);
    const int G = std::max(gmin, std::min(gcap, capacity / nn));
    if (group && a0 == 0) *group = G;
    WideCtx xs = X;
    xs.act = X.act + a0;
    cudaError_t e = launch_tridiag(xs, nn, G, nb, min_rows, smem, st, a0 == 0 ? prof : nullptr);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

__global__ void wide_copy_hp_kernel(WideCtx X) {  // A = H0' (a realistic matrix for the autotuner)
  const WideMol& w = X.mols[X.act[blockIdx.y]];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)w.N * w.ld;
       i += (long long)gridDim.x * blockDim.x)
    w.A[i] = w.Hp[i];
}

// Times the reduction of the current H0' matrices for every candidate
// (panel width x minimum rows per CTA) and keeps the fastest.
static cudaError_t wide_autotune(const WideCtx& X, int na, int capacity, int gcap, size_t smem, int maxn,
                                 cudaStream_t st, WidePlan& plan) {
  const int nbs[] = {8, 16, 32};
  const int mrs[] = {4, 8, 16, 32, 64, 128};
  cudaEvent_t e0, e1;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e != cudaSuccess) return e;
  float best = 1e30f;
  WidePlan bestp;
  const dim3 cg((unsigned)std::min<long long>(((long long)maxn * maxn + 255) / 256, 1024), na);
  for (int warm = 1; warm >= 0 && e == cudaSuccess; --warm)
    for (int nb : nbs)
      for (int mr : mrs) {
        if (warm && (nb != 16 || mr != 16)) continue;
        wide_copy_hp_kernel<<<cg, 256, 0, st>>>(X);
        if ((e = cudaEventRecord(e0, st)) != cudaSuccess) break;
        if ((e = tridiag_all(X, na, maxn, nb, mr, capacity, gcap, smem, st, nullptr)) != cudaSuccess) break;
        if ((e = cudaEventRecord(e1, st)) != cudaSuccess) break;
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (!warm && std::getenv("GFN1_WIDE_TIMING"))
          std::fprintf(stderr, "wide tune N %d molecules %d panel %d min_rows %d: %.3f ms\n", maxn, na, nb, mr, ms);
        if (!warm && ms < best) {
          best = ms;
          bestp.nb = nb;
          bestp.min_rows = mr;
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return e;
  bestp.tridiag_ms = best;
  bestp.tuned = true;
  plan = bestp;
  return cudaSuccess;
}

// Reads the slots' SCC states back (synchronises the stream).
static cudaError_t wide_read_states(WideRuntime& R, int n, cudaStream_t st) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(R.h_state, R.d_state, sizeof(WideState) * n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e;
}

// Per-stage wall time of the large-molecule path, printed to stderr at the end
// of a call when GFN1_WIDE_TIMING=1 (events on the launching stream).
struct WideTimer {
  bool on = false;
  cudaStream_t st = nullptr;
  cudaEvent_t last = nullptr;
  std::map<std::string, double> ms;
  explicit WideTimer(cudaStream_t s) : st(s) {
    const char* v = std::getenv("GFN1_WIDE_TIMING");
    on = v && *v && *v != '0';
    if (on && cudaEventCreate(&last) == cudaSuccess) cudaEventRecord(last, st);
  }
  void mark(const char* name) {
    if (!on) return;
    cudaEvent_t ev;
    if (cudaEventCreate(&ev) != cudaSuccess) return;
    cudaEventRecord(ev, st);
    cudaEventSynchronize(ev);
    float t = 0.f;
    cudaEventElapsedTime(&t, last, ev);
    ms[name] += t;
    cudaEventDestroy(last);
    last = ev;
  }
  ~WideTimer() {
    if (!on) return;
    double tot = 0.0;
    for (auto& kv : ms) tot += kv.second;
    for (auto& kv : ms) std::fprintf(stderr, "wide %-10s %10.3f ms\n", kv.first.c_str(), kv.second);
    std::fprintf(stderr, "wide %-10s %10.3f ms\n", "total", tot);
    if (last) cudaEventDestroy(last);
  }
};

// One pass of the SCC over the molecules listed in R.h_act[0..na): the whole
// large-molecule path for a call.  Synchronises `st` once per SCC iteration
// (the convergence flags).
cudaError_t run_wide(const Batch& B, const Model& M, const SccOptions& opt, WideRuntime& R, int nslots, int maxn,
                     int maxnsh, int maxnat, int cap, int num_sms, cudaStream_t st) {
  if (nslots == 0) return cudaSuccess;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaError_t e = wide_configure(dev);
  if (e != cudaSuccess) return e;
  WideCtx X{R.d_mols, R.d_act, maxnsh, maxn, maxnat, cap};
  WideTimer tm(st);
  // Eigenvalues closer than ortol_rel |T|_1 form a cluster whose vectors are
  // re-orthogonalised (modified Gram-Schmidt).  Inverse iteration alone leaves
  // an overlap of about eps |T| / gap between two vectors, at most 2e-9 here;
  // a wider threshold (LAPACK dstein: 1e-3) chains hundreds of the dense
  // levels of a large molecule into clusters one thread would orthogonalise.
  double ortol_rel = 1e-7;
  if (const char* v = std::getenv("GFN1_WIDE_ORTOL")) ortol_rel = std::atof(v);
  if (tm.on && !R.d_stats) {
    if ((e = cudaMalloc(&R.d_stats, sizeof(int) * 64)) != cudaSuccess) return e;
  }
  if (tm.on && (e = cudaMemsetAsync(R.d_stats, 0, sizeof(int) * 64, st)) != cudaSuccess) return e;
  const size_t tsm = kTileSmemBytes;
  const size_t tsm1 = kTileSmemBytes + sizeof(double) * 64 * 65;
  const size_t tsm2 = kTileSmemBytes + 2 * sizeof(double) * 64 * 65;
  const size_t rsm = dense_table_bytes(maxnsh, maxn, maxnat);
  const size_t trsm = tridiag_smem_bytes(maxn);
  if (rsm > 200 * 1024 || trsm > 200 * 1024) return cudaErrorInvalidValue;
  auto upload_act = [&](int na) {
    return cudaMemcpyAsync(R.d_act, R.h_act, sizeof(int) * na, cudaMemcpyHostToDevice, st);
  };
  auto gx = [&](long long tiles, int na) {
    return (unsigned)std::max<long long>(1, std::min<long long>(tiles, std::max(1, 8 * num_sms / std::max(na, 1))));
  };
  const int nblk = (maxn + 63) / 64;
  const long long mt = (long long)nblk * (nblk + 1) / 2;
  // ---- all slots: orthogonaliser and H0'
  int na = nslots;
  for (int q = 0; q < na; ++q) R.h_act[q] = q;
  if ((e = upload_act(na)) != cudaSuccess) return e;
  wide_begin_kernel<<<dim3(gx(((long long)maxn * maxn + 255) / 256, na), na), 256, 0, st>>>(B, X);
  for (int k = 0; k < nblk; ++k) {
    wide_chol_diag_kernel<<<na, 256, 2 * sizeof(double) * 64 * 65, st>>>(X, k);
    wide_chol_panel_kernel<<<dim3(gx(nblk, na), na), kGemmNT, tsm, st>>>(X, k);
    wide_chol_trail_kernel<<<dim3(gx(mt, na), na), kGemmNT, tsm, st>>>(X, k);
  }
  for (int I = 1; I < nblk; ++I) wide_inv_row_kernel<<<dim3(gx(I, na), na), kGemmNT, tsm1, st>>>(X, I);
  wide_hp1_kernel<<<dim3(gx((long long)nblk * nblk, na), na), kGemmNT, tsm, st>>>(B, X);
  wide_hp2_kernel<<<dim3(gx(mt, na), na), kGemmNT, tsm, st>>>(X);
  tm.mark("orth");
  // ---- group size and the reduction plan (autotuned once per size class)
  int occ = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, wide_tridiag_kernel, kRedNT, trsm)) != cudaSuccess)
    return e;
  if (occ < 1) return cudaErrorInvalidConfiguration;
  const int capacity = occ * num_sms;
  const int gcap = std::min(num_sms, kWideMaxG);
  {
    const int nab = na <= 1 ? 1 : na <= 4 ? 4 : na <= 16 ? 16 : na <= 64 ? 64 : 1024;
    const long long key = ((long long)dev << 40) | ((long long)((maxn + 127) / 128) << 16) | nab;
    std::lock_guard<std::mutex> lk(g_wide_tune_mu);
    auto it = g_wide_plans.find(key);
    const char* env_nb = std::getenv("GFN1_WIDE_PANEL");
    if (env_nb && *env_nb) {  // fixed plan (sweeps)
      R.plan.nb = std::max(1, std::min(kMaxPanel, std::atoi(env_nb)));
      const char* env_mr = std::getenv("GFN1_WIDE_MIN_ROWS");
      R.plan.min_rows = env_mr && *env_mr ? std::max(1, std::atoi(env_mr)) : 16;
      R.plan.tuned = false;
    } else if (it != g_wide_plans.end()) {
      R.plan = it->second;
    } else {
      if ((e = wide_autotune(X, na, capacity, gcap, trsm, maxn, st, R.plan)) != cudaSuccess) return e;
      g_wide_plans[key] = R.plan;
    }
  }
  tm.mark("tune");
  if ((e = wide_read_states(R, nslots, st)) != cudaSuccess) return e;
  std::vector<int> done(nslots, 0);  // converged on an earlier rung, or failed
  for (int q = 0; q < nslots; ++q) done[q] = R.h_state[q].status != kOk;
  // ---- the fallback ladder (src/electronic.rs:1390-1447): rung 0 with the
  // requested options, then linear mixing with a level shift, then T_el >= 3000 K
  for (int rung = 0; rung <= 3; ++rung) {
    na = 0;
    for (int q = 0; q < nslots; ++q)
      if (!done[q]) R.h_act[na++] = q;
    if (na == 0) break;
    SccOptions ro = opt;
    double lshift = opt.level_shift;
    if (rung == 1 || rung == 2) {
      ro.broyden = 0;
      ro.mixing = rung == 1 ? 0.20 : 0.10;
      lshift = std::max(opt.level_shift, rung == 1 ? 0.20 : 0.10);
      ro.max_scc = std::max(opt.max_scc, 800);
    } else if (rung == 3) {
      ro.etemp = std::max(opt.etemp, 3000.0);
      ro.max_scc = std::max(opt.max_scc, 250);
      lshift = 0.0;
    }
    if ((e = upload_act(na)) != cudaSuccess) return e;
    wide_rung_kernel<<<na, kWideNT, rsm, st>>>(B, M, X, ro, rung);
    for (int iter = 1; iter <= ro.max_scc && na > 0; ++iter) {
      tm.mark("host");
      wide_potential_kernel<<<na, kWideNT, rsm, st>>>(B, M, X);
      tm.mark("potential");
      wide_fock_kernel<<<dim3(gx(mt, na), na), kGemmNT, tsm, st>>>(X);
      if (lshift != 0.0) wide_shift_kernel<<<dim3(gx(mt, na), na), kGemmNT, tsm, st>>>(X, lshift);
      tm.mark("fock");
      if ((e = tridiag_all(X, na, maxn, R.plan.nb, R.plan.min_rows, capacity, gcap, trsm, st, &R.group,
                           tm.on ? (long long*)(R.d_stats + 32) : nullptr)) != cudaSuccess)
        return e;
      tm.mark("tridiag");
      wide_eigval_kernel<<<dim3((maxn + kEigNT) / kEigNT, na), kEigNT, sizeof(double) * 2 * maxn, st>>>(X);
      tm.mark("eigval");
      wide_fermi_kernel<<<na, kWideNT, 0, st>>>(X);
      tm.mark("fermi");
      wide_inviter_kernel<<<dim3((maxn + 63) / 64, na), 64, 0, st>>>(X, ortol_rel, tm.on ? R.d_stats : nullptr);
      tm.mark("inviter");
      const int nref_blk = (std::max(maxn - 2, 0) + 63) / 64;
      wide_bt_t_kernel<<<dim3(std::max(nref_blk, 1), na), kGemmNT, tsm + 2 * sizeof(double) * 64 * 65, st>>>(X);
      const int nct = nblk;
      const int ksplit = std::max(1, std::min(kWideMaxSplit, num_sms / std::max(1, na * nct)));
      for (int b = nref_blk - 1; b >= 0; --b) {
        wide_bt_x_kernel<<<dim3(gx((long long)nct * ksplit, na), na), kGemmNT, tsm, st>>>(X, b, ksplit);
        wide_bt_y_kernel<<<dim3(gx(nct, na), na), kGemmNT, tsm1, st>>>(X, b, ksplit);
        wide_bt_upd_kernel<<<dim3(gx((long long)nblk * nct, na), na), kGemmNT, tsm, st>>>(X, b);
      }
      tm.mark("backtr");
      wide_cd_kernel<<<dim3(gx((long long)nblk * nct, na), na), kGemmNT, tsm2, st>>>(X);
      if (lshift != 0.0) wide_eshift_kernel<<<dim3(gx((long long)nblk * nct, na), na), kGemmNT, tsm, st>>>(X);
      tm.mark("cd");
      wide_energy_mix_kernel<<<na, kWideNT, rsm, st>>>(B, M, X, ro, lshift);
      tm.mark("energy");
      if ((e = wide_read_states(R, nslots, st)) != cudaSuccess) return e;
      int nn = 0;
      for (int a = 0; a < na; ++a) {
        const int q = R.h_act[a];
        const WideState& s = R.h_state[q];
        if (s.status != kOk || s.converged) done[q] = 1;
        else R.h_act[nn++] = q;
      }
      if (nn != na) {
        na = nn;
        if (na > 0 && (e = upload_act(na)) != cudaSuccess) return e;
      }
    }
  }
  // ---- results for every slot: P, W of the last diagonalisation, energies, charges
  for (int q = 0; q < nslots; ++q) R.h_act[q] = q;
  if ((e = upload_act(nslots)) != cudaSuccess) return e;
  wide_pw_kernel<<<dim3(gx(mt, nslots), nslots), kGemmNT, tsm, st>>>(B, X);
  wide_results_kernel<<<nslots, kWideNT, rsm, st>>>(B, M, X);
  tm.mark("final");
  if (tm.on) {
    int hs[64];
    if (cudaMemcpy(hs, R.d_stats, sizeof(hs), cudaMemcpyDeviceToHost) == cudaSuccess) {
      std::fprintf(stderr, "wide clusters: largest %d, clusters of two or more %d (ortol %.1e |T|)\n", hs[0], hs[1],
                   ortol_rel);
      const char* names[] = {"A", "bar1", "B-tot", "B-v", "symv", "bar2", "C", "panelbar", "trail"};
      for (int q = 0; q < 9; ++q)
        std::fprintf(stderr, "wide tridiag phase %-8s %12.0f kcycles (CTA 0 of the first molecule)\n", names[q],
                     ((long long*)(hs + 32))[q] / 1e3);
    }
  }
  return cudaGetLastError();
}

// Slot descriptors for the large molecules of a batch over one device buffer
// (`base`, wide_slot_layout(...).total doubles per slot at `slot_off`).
cudaError_t wide_bind(WideRuntime& R, const std::vector<int>& ids, const std::vector<int>& Ns,
                      const std::vector<long long>& mos, const std::vector<int>& nshs, const std::vector<int>& nats,
                      int cap, double* base, const std::vector<long long>& slot_off) {
  const int n = (int)ids.size();
  cudaError_t e = cudaSuccess;
  if (n > R.capacity) {
    if (R.d_mols) cudaFree(R.d_mols);
    if (R.d_act) cudaFree(R.d_act);
    if (R.d_state) cudaFree(R.d_state);
    if (R.d_sync) cudaFree(R.d_sync);
    if (R.d_flags) cudaFree(R.d_flags);
    if (R.h_act) cudaFreeHost(R.h_act);
    if (R.h_state) cudaFreeHost(R.h_state);
    R.d_flags = nullptr;
    R.d_mols = nullptr;
    R.d_act = nullptr;
    R.d_state = nullptr;
    R.d_sync = nullptr;
    R.h_act = nullptr;
    R.h_state = nullptr;
    R.capacity = 0;
    if ((e = cudaMalloc(&R.d_mols, sizeof(WideMol) * n)) != cudaSuccess ||
        (e = cudaMalloc(&R.d_act, sizeof(int) * n)) != cudaSuccess ||
        (e = cudaMalloc(&R.d_state, sizeof(WideState) * n)) != cudaSuccess ||
        (e = cudaMalloc(&R.d_sync, sizeof(GroupSync) * 2 * n)) != cudaSuccess ||
        (e = cudaMalloc(&R.d_flags, sizeof(unsigned long long) * 2 * kFlagSlots * n)) != cudaSuccess ||
        (e = cudaHostAlloc((void**)&R.h_act, sizeof(int) * n, cudaHostAllocDefault)) != cudaSuccess ||
        (e = cudaHostAlloc((void**)&R.h_state, sizeof(WideState) * n, cudaHostAllocDefault)) != cudaSuccess)
      return e;
    R.capacity = n;
  }
  R.mols.resize(n);
  for (int q = 0; q < n; ++q) {
    const WideSlotLayout s = wide_slot_layout(Ns[q], nshs[q], nats[q], cap);
    double* p = base + slot_off[q];
    WideMol& w = R.mols[q];
    w.m = ids[q];
    w.N = Ns[q];
    w.ld = s.ld;
    w.nblk = (Ns[q] + 63) / 64;
    w.mo = mos[q];
    w.L = p + s.L;
    w.Li = p + s.Li;
    w.Hp = p + s.Hp;
    w.A = p + s.A;
    w.Z = p + s.Z;
    w.C = p + s.C;
    w.iw = p + s.iw;
    w.VW = p + s.VW;
    w.xbuf = p + s.xbuf;
    w.d = p + s.d;
    w.e = p + s.e;
    w.tau = p + s.tau;
    w.esq = p + s.esq;
    w.eps = p + s.eps;
    w.occ = p + s.occ;
    w.pop = p + s.pop;
    w.vao = p + s.vao;
    w.part = p + s.part;
    w.Tf = p + s.Tf;
    w.Xp = p + s.Xp;
    w.popp = p + s.popp;
    w.eshift = p + s.eshift;
    w.ws = p + s.ws;
    w.st = R.d_state + q;
    w.sync = R.d_sync + 2 * q;
    w.flags = R.d_flags + (size_t)2 * kFlagSlots * q;
  }
  if ((e = cudaMemcpy(R.d_mols, R.mols.data(), sizeof(WideMol) * n, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
  if ((e = cudaMemset(R.d_sync, 0, sizeof(GroupSync) * 2 * n)) != cudaSuccess) return e;
  if ((e = cudaMemset(R.d_flags, 0, sizeof(unsigned long long) * 2 * kFlagSlots * n)) != cudaSuccess) return e;
  return cudaMemset(R.d_state, 0, sizeof(WideState) * n);
}

void wide_release(WideRuntime& R) {
  if (R.d_stats) cudaFree(R.d_stats);
  if (R.d_flags) cudaFree(R.d_flags);
  if (R.d_mols) cudaFree(R.d_mols);
  if (R.d_act) cudaFree(R.d_act);
  if (R.d_state) cudaFree(R.d_state);
  if (R.d_sync) cudaFree(R.d_sync);
  if (R.h_act) cudaFreeHost(R.h_act);
  if (R.h_state) cudaFreeHost(R.h_state);
  R = WideRuntime();
}

long long wide_slot_doubles(int N, int nsh, int nat, int cap) { return wide_slot_layout(N, nsh, nat, cap).total; }

}  // namespace gfn1

namespace gfn1 {
// Opaque handles for the host code of the C ABI.
WideRuntime* wide_runtime_new() { return new WideRuntime(); }
void wide_runtime_delete(WideRuntime* r) {
  if (!r) return;
  wide_release(*r);
  delete r;
}
cudaError_t wide_bind_runtime(WideRuntime* r, const std::vector<int>& ids, const std::vector<int>& Ns,
                              const std::vector<long long>& mos, const std::vector<int>& nshs,
                              const std::vector<int>& nats, int cap, double* base,
                              const std::vector<long long>& slot_off) {
  return wide_bind(*r, ids, Ns, mos, nshs, nats, cap, base, slot_off);
}
cudaError_t wide_run(const Batch& B, const Model& M, const SccOptions& opt, WideRuntime* r, int nslots, int maxn,
                     int maxnsh, int maxnat, int cap, int num_sms, cudaStream_t st) {
  return run_wide(B, M, opt, *r, nslots, maxn, maxnsh, maxnat, cap, num_sms, st);
}
void wide_plan_info(const WideRuntime* r, int* nb, int* min_rows, int* group, float* ms, int* tuned) {
  if (nb) *nb = r ? r->plan.nb : 0;
  if (min_rows) *min_rows = r ? r->plan.min_rows : 0;
  if (group) *group = r ? r->group : 0;
  if (ms) *ms = r ? r->plan.tridiag_ms : 0.f;
  if (tuned) *tuned = r && r->plan.tuned ? 1 : 0;
}
}  // namespace gfn1

namespace gfn1 {
size_t dense_table_bytes_host(int maxnsh, int maxn, int maxnat) { return dense_table_bytes(maxnsh, maxn, maxnat); }
}  // namespace gfn1
