// Learned SCC initial guess: descriptor, inference, projection and training
// kernels (see guess.cuh).  Training uses FP32 master weights; inference reads
// BF16 copies of the weights and keeps activations in BF16 with FP32
// accumulation.
#include <cuda_bf16.h>
#include <math.h>

#include "../../include/gfn1_b200.h"
#include "guess.cuh"

namespace gfn1 {

namespace {

__device__ __forceinline__ int elem_channel(int z) {
  return z == 1 ? 0 : (z == 6 ? 1 : (z == 7 ? 2 : (z == 8 ? 3 : -1)));
}

__device__ __forceinline__ float silu_f(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float dsilu_f(float z) {
  const float s = 1.0f / (1.0f + expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// ------------------------------------------------------------------ descriptors
// One CTA per molecule, one warp per atom.  Lanes own radial features lane and
// lane + 32 (channels 0-1 and 2-3, centre lane & 15); lanes 0..15 own the
// angular pair (channel lane >> 2, radial function lane & 3).  The neighbour
// geometry (distance, cutoff function, unit vector, channel) is formed once per
// neighbour, by the lane j - j0 of a 32-neighbour chunk, and broadcast to the
// warp in neighbour order, so every feature sums its terms in the order of
// the neighbours.
__global__ void __launch_bounds__(128, 4) guess_features_kernel(int nmol, const int* __restrict__ atom_off,
                                                             const int* __restrict__ z,
                                                             const double* __restrict__ xyz,
                                                             const float* __restrict__ mean,
                                                             const float* __restrict__ stdv, float* __restrict__ x) {
  const int m = blockIdx.x;
  if (m >= nmol) return;
  const int a0 = atom_off[m], a1 = atom_off[m + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double rc = kGuessCutoff, pi = 3.141592653589793;
  const int k = lane & 15;
  const double mu = 0.5 + 5.5 * k / 15.0;
  const int c0 = lane >> 4, c1 = (lane + 32) >> 4;
  const int ca = lane >> 2, b = lane & 3;
  const double nu = (b == 0) ? 1.0 : (b == 1 ? 2.0 : (b == 2 ? 3.0 : 4.5));
  for (int i = a0 + wid; i < a1; i += nw) {
    float* xi = x + (long long)i * kGuessIn;
    const int ci = elem_channel(z[i]);
    if (ci < 0) {
      for (int f = lane; f < kGuessIn; f += 32) xi[f] = 0.0f;
      continue;
    }
    const double xa = xyz[3LL * i], ya = xyz[3LL * i + 1], za = xyz[3LL * i + 2];
    double g0 = 0.0, g1 = 0.0;
    double vx = 0.0, vy = 0.0, vz = 0.0, sxx = 0.0, syy = 0.0, szz = 0.0, sxy = 0.0, sxz = 0.0, syz = 0.0, sw = 0.0;
    for (int j0 = a0; j0 < a1; j0 += 32) {
      // neighbour j0 + lane: channel (-1: none), distance, cutoff function, unit vector
      int cjl = -1;
      double rl = 0.0, fcl = 0.0, uxl = 0.0, uyl = 0.0, uzl = 0.0;
      const int jl = j0 + lane;
      if (jl < a1 && jl != i) {
        const int cj = elem_channel(z[jl]);
        const double dx = xyz[3LL * jl] - xa, dy = xyz[3LL * jl + 1] - ya, dz = xyz[3LL * jl + 2] - za;
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (cj >= 0 && r2 < rc * rc && r2 != 0.0) {
          cjl = cj;
          rl = sqrt(r2);
          fcl = 0.5 * (cos(pi * rl / rc) + 1.0);
          uxl = dx / rl;
          uyl = dy / rl;
          uzl = dz / rl;
        }
      }
      const int nj = min(32, a1 - j0);
      for (int t = 0; t < nj; ++t) {
        const int cj = __shfl_sync(0xffffffffu, cjl, t);
        if (cj < 0) continue;
        const double r = __shfl_sync(0xffffffffu, rl, t);
        const double fc = __shfl_sync(0xffffffffu, fcl, t);
        const double gr = exp(-4.0 * (r - mu) * (r - mu)) * fc;
        if (cj == c0) g0 += gr;
        if (cj == c1) g1 += gr;
        const double ux = __shfl_sync(0xffffffffu, uxl, t);
        const double uy = __shfl_sync(0xffffffffu, uyl, t);
        const double uz = __shfl_sync(0xffffffffu, uzl, t);
        if (lane < 16 && cj == ca) {
          const double w = exp(-(r - nu) * (r - nu)) * fc;
          vx += w * ux;
          vy += w * uy;
          vz += w * uz;
          sxx += w * ux * ux;
          syy += w * uy * uy;
          szz += w * uz * uz;
          sxy += w * ux * uy;
          sxz += w * ux * uz;
          syz += w * uy * uz;
          sw += w;
        }
      }
    }
    auto put = [&](int f, double v) {
      xi[f] = mean ? (float)((v - (double)mean[f]) / (double)stdv[f]) : (float)v;
    };
    put(lane, g0);
    put(lane + 32, g1);
    if (lane < 16) {
      const double t3 = sw / 3.0;
      const double txx = sxx - t3, tyy = syy - t3, tzz = szz - t3;
      put(64 + lane, vx * vx + vy * vy + vz * vz);
      put(80 + lane, txx * txx + tyy * tyy + tzz * tzz + 2.0 * (sxy * sxy + sxz * sxz + syz * syz));
    }
    if (lane < 4) xi[kGuessDesc + lane] = (lane == ci) ? 1.0f : 0.0f;
  }
}

// ------------------------------------------------------------------ inference
// Tensor-core MLP on 64-atom tiles: each hidden layer is a [64 x K] x [K x 128]
// product of BF16 activations and weights with FP32 accumulation
// (mma.sync.m16n8k16, 8 warps: warp w takes rows 16 (w & 3).. and columns
// 64 (w >> 2)..), then bias and SiLU in FP32, rounded to BF16 for the next
// layer.  Weights sit transposed in shared memory ([n][k], rows padded by 8
// elements so that the fragment loads of the 8 row groups fall in distinct
// banks); the first layer's K = 100 is padded with zeros to 112.
constexpr int kTile = 64;                  // atoms per tile
constexpr int kInferNT = 256;              // 8 warps
constexpr int kK1 = 112;                   // kGuessIn rounded up to the MMA's k = 16
constexpr int kLd1 = kK1 + 8;              // row stride (elements) of the input tile and W1^T
constexpr int kLdH = kGuessHid + 8;        // row stride of hidden activations, W2^T and W3^T
static_assert(kGuessIn <= kK1 && kK1 % 16 == 0, "first-layer padding");

struct InferSmem {
  static constexpr size_t w1 = 0;                                                    // W1^T [128][kLd1]
  static constexpr size_t w2 = w1 + sizeof(uint16_t) * kGuessHid * kLd1;             // W2^T [128][kLdH]
  static constexpr size_t w3 = w2 + sizeof(uint16_t) * kGuessHid * kLdH;             // W3^T [128][kLdH]
  static constexpr size_t w4 = w3 + sizeof(uint16_t) * kGuessHid * kLdH;             // W4 [128][2]
  static constexpr size_t bias = w4 + sizeof(uint16_t) * kGuessHid * kGuessOut;      // b1 b2 b3 b4 (FP32)
  static constexpr size_t xin = bias + sizeof(float) * (3 * kGuessHid + 4);          // [64][kLd1]
  static constexpr size_t h0 = xin + sizeof(uint16_t) * kTile * kLd1;                // [64][kLdH]
  static constexpr size_t h1 = h0 + sizeof(uint16_t) * kTile * kLdH;                 // [64][kLdH]
  static constexpr size_t total = h1 + sizeof(uint16_t) * kTile * kLdH;
};
static_assert(InferSmem::w2 % 16 == 0 && InferSmem::w3 % 16 == 0 && InferSmem::w4 % 16 == 0 &&
                  InferSmem::bias % 16 == 0 && InferSmem::xin % 16 == 0 && InferSmem::h0 % 16 == 0 &&
                  InferSmem::h1 % 16 == 0,
              "16-byte aligned regions");

__device__ __forceinline__ float bf2f(uint16_t h) { return __uint_as_float(((unsigned)h) << 16); }
__device__ __forceinline__ uint16_t f2bf(float f) {
  const __nv_bfloat16 b = __float2bfloat16_rn(f);
  return *reinterpret_cast<const uint16_t*>(&b);
}
__device__ __forceinline__ uint32_t lds32(const uint16_t* p) { return *reinterpret_cast<const uint32_t*>(p); }

// D += A B for one 16x8 tile, k = 16: A row-major (a0: rows g, k 2t..2t+1;
// a1: rows g + 8; a2, a3: k + 8), B column-major (b0: k 2t..2t+1 of column
// g; b1: k + 8), D (d0, d1: row g, columns 2t, 2t + 1; d2, d3: row g + 8),
// g = lane / 4, t = lane % 4.
__device__ __forceinline__ void mma_bf16_16x8x16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                                 uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// One hidden layer on a 64-atom tile: out = SiLU(in W + b); in [64][LDI],
// wt = W^T [128][LDI], out [64][kLdH], K a multiple of 16.
template <int K, int LDI>
__device__ __forceinline__ void infer_layer(const uint16_t* __restrict__ in, const uint16_t* __restrict__ wt,
                                            const float* __restrict__ bias, uint16_t* __restrict__ out) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int r0 = (wid & 3) * 16, n0 = (wid >> 2) * 64;
  float acc[8][4];
#pragma unroll
  for (int q = 0; q < 8; ++q)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[q][c] = 0.0f;
#pragma unroll
  for (int k0 = 0; k0 < K; k0 += 16) {
    const uint16_t* ar = in + (r0 + g) * LDI + k0 + 2 * t;
    const uint32_t a0 = lds32(ar), a1 = lds32(ar + 8 * LDI), a2 = lds32(ar + 8), a3 = lds32(ar + 8 * LDI + 8);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const uint16_t* br = wt + (n0 + 8 * q + g) * LDI + k0 + 2 * t;
      mma_bf16_16x8x16(acc[q], a0, a1, a2, a3, lds32(br), lds32(br + 8));
    }
  }
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int col = n0 + 8 * q + 2 * t;
    const float b0 = bias[col], b1 = bias[col + 1];
    const uint32_t lo = (uint32_t)f2bf(silu_f(acc[q][0] + b0)) | ((uint32_t)f2bf(silu_f(acc[q][1] + b1)) << 16);
    const uint32_t hi = (uint32_t)f2bf(silu_f(acc[q][2] + b0)) | ((uint32_t)f2bf(silu_f(acc[q][3] + b1)) << 16);
    *reinterpret_cast<uint32_t*>(out + (r0 + g) * kLdH + col) = lo;
    *reinterpret_cast<uint32_t*>(out + (r0 + g + 8) * kLdH + col) = hi;
  }
}

__global__ void __launch_bounds__(kInferNT, 1) guess_infer_kernel(const float* __restrict__ params,
                                                                 const uint16_t* __restrict__ wbf16,
                                                                 long long natoms, const float* __restrict__ x,
                                                                 float* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint16_t* sw1 = reinterpret_cast<uint16_t*>(smem + InferSmem::w1);
  uint16_t* sw2 = reinterpret_cast<uint16_t*>(smem + InferSmem::w2);
  uint16_t* sw3 = reinterpret_cast<uint16_t*>(smem + InferSmem::w3);
  uint16_t* sw4 = reinterpret_cast<uint16_t*>(smem + InferSmem::w4);
  float* sb = reinterpret_cast<float*>(smem + InferSmem::bias);
  uint16_t* sx = reinterpret_cast<uint16_t*>(smem + InferSmem::xin);
  uint16_t* sh0 = reinterpret_cast<uint16_t*>(smem + InferSmem::h0);
  uint16_t* sh1 = reinterpret_cast<uint16_t*>(smem + InferSmem::h1);
  const int tid = threadIdx.x;
  // weights: W1..W3 read in their global order [k][n] and stored transposed,
  // the padding columns zero; W4 as it is
  const uint16_t* gw1 = wbf16;
  const uint16_t* gw2 = gw1 + kGuessIn * kGuessHid;
  const uint16_t* gw3 = gw2 + kGuessHid * kGuessHid;
  const uint16_t* gw4 = gw3 + kGuessHid * kGuessHid;
  for (int i = tid; i < kGuessHid * kLd1; i += kInferNT) {
    const int n = i / kLd1, k = i - n * kLd1;
    if (k >= kGuessIn) sw1[i] = 0;
  }
  for (int i = tid; i < kGuessHid * kLdH; i += kInferNT) {
    const int n = i / kLdH, k = i - n * kLdH;
    if (k >= kGuessHid) sw2[i] = sw3[i] = 0;
  }
  for (int i = tid; i < kGuessIn * kGuessHid; i += kInferNT) {
    const int k = i / kGuessHid, n = i - k * kGuessHid;
    sw1[n * kLd1 + k] = gw1[i];
  }
  for (int i = tid; i < kGuessHid * kGuessHid; i += kInferNT) {
    const int k = i / kGuessHid, n = i - k * kGuessHid;
    sw2[n * kLdH + k] = gw2[i];
    sw3[n * kLdH + k] = gw3[i];
  }
  for (int i = tid; i < kGuessHid * kGuessOut; i += kInferNT) sw4[i] = gw4[i];
  // biases from the FP32 parameter vector
  const float* pb1 = params + 2 * kGuessDesc + kGuessIn * kGuessHid;
  const float* pb2 = pb1 + kGuessHid + kGuessHid * kGuessHid;
  const float* pb3 = pb2 + kGuessHid + kGuessHid * kGuessHid;
  const float* pb4 = pb3 + kGuessHid + kGuessHid * kGuessOut;
  for (int i = tid; i < kGuessHid; i += kInferNT) {
    sb[i] = pb1[i];
    sb[kGuessHid + i] = pb2[i];
    sb[2 * kGuessHid + i] = pb3[i];
  }
  if (tid < kGuessOut) sb[3 * kGuessHid + tid] = pb4[tid];
  const long long ntiles = (natoms + kTile - 1) / kTile;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long row0 = tile * kTile;
    __syncthreads();
    for (int i = tid; i < kTile * kLd1; i += kInferNT) {
      const int r = i / kLd1, c = i - r * kLd1;
      sx[i] = f2bf((c < kGuessIn && row0 + r < natoms) ? x[(row0 + r) * kGuessIn + c] : 0.0f);
    }
    __syncthreads();
    infer_layer<kK1, kLd1>(sx, sw1, sb, sh0);
    __syncthreads();
    infer_layer<kGuessHid, kLdH>(sh0, sw2, sb + kGuessHid, sh1);
    __syncthreads();
    infer_layer<kGuessHid, kLdH>(sh1, sw3, sb + 2 * kGuessHid, sh0);
    __syncthreads();
    if (tid < kTile * kGuessOut) {
      const int a = tid >> 1, o = tid & 1;
      float s = sb[3 * kGuessHid + o];
      for (int k = 0; k < kGuessHid; ++k) s += bf2f(sh0[a * kLdH + k]) * bf2f(sw4[k * kGuessOut + o]);
      if (row0 + a < natoms) y[(row0 + a) * kGuessOut + o] = s;
    }
  }
}

__global__ void guess_bf16_kernel(const float* __restrict__ params, uint16_t* __restrict__ out) {
  // weight matrices W1..W4 in order, skipping the biases
  const long long n1 = (long long)kGuessIn * kGuessHid, n2 = (long long)kGuessHid * kGuessHid,
                  n4 = (long long)kGuessHid * kGuessOut;
  const float* w1 = params + 2 * kGuessDesc;
  const float* w2 = w1 + n1 + kGuessHid;
  const float* w3 = w2 + n2 + kGuessHid;
  const float* w4 = w3 + n2 + kGuessHid;
  const long long tot = n1 + 2 * n2 + n4;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    float v;
    if (i < n1)
      v = w1[i];
    else if (i < n1 + n2)
      v = w2[i - n1];
    else if (i < n1 + 2 * n2)
      v = w3[i - n1 - n2];
    else
      v = w4[i - n1 - 2 * n2];
    out[i] = f2bf(v);
  }
}

// One warp per molecule: shift the predicted shell charges to the molecule's
// charge and write them in the engine's shell layout.
__global__ void guess_project_kernel(int nmol, const int* __restrict__ atom_off, const int* __restrict__ shell_off,
                                     const int* __restrict__ z, const float* __restrict__ y,
                                     const double* __restrict__ charge, double* __restrict__ init_q) {
  const int lane = threadIdx.x & 31;
  const int m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (m >= nmol) return;
  const int a0 = atom_off[m], a1 = atom_off[m + 1];
  const int s0 = shell_off[m], s1 = shell_off[m + 1];
  bool ok = (s1 - s0) == 2 * (a1 - a0);
  double s = 0.0;
  for (int a = a0 + lane; a < a1; a += 32) {
    if (elem_channel(z[a]) < 0) ok = false;
    s += (double)y[2LL * a] + (double)y[2LL * a + 1];
  }
  ok = __all_sync(0xffffffffu, ok);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (!ok) {
    for (int q = s0 + lane; q < s1; q += 32) init_q[q] = 0.0;
    return;
  }
  const int n = 2 * (a1 - a0);
  const double shift = n ? ((charge ? charge[m] : 0.0) - s) / n : 0.0;
  for (int q = lane; q < n; q += 32) init_q[s0 + q] = (double)y[2LL * a0 + q] + shift;
}

// ------------------------------------------------------------------ training
// C[MxN] = op(A)[MxK] op(B)[KxN] over the K range of blockIdx.z, 64x64 tiles,
// 16x16 threads with 4x4 outputs each.  op(A)(m,k) = TA ? A[k lda + m] :
// A[m lda + k]; op(B)(k,n) = TB ? B[n ldb + k] : B[k ldb + n].
enum Epi : int { kEpiPartial = 0, kEpiBiasSilu = 1, kEpiBias = 2, kEpiDsilu = 3 };

template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(256) mlp_gemm_kernel(int M, int N, int K, const float* __restrict__ A, int lda,
                                                       const float* __restrict__ B, int ldb,
                                                       const float* __restrict__ bias,
                                                       const float* __restrict__ zprev, int ldz,
                                                       float* __restrict__ C, float* __restrict__ Z, int ldc,
                                                       int kchunk) {
  __shared__ __align__(16) float As[16][64];
  __shared__ __align__(16) float Bs[16][64];
  const int tid = threadIdx.x;
  const int tm = tid >> 4, tn = tid & 15;
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  const long long kbeg = (long long)blockIdx.z * kchunk;
  const long long kend = min((long long)K, kbeg + kchunk);
  float acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = 0.0f;
  for (long long k0 = kbeg; k0 < kend; k0 += 16) {
    for (int e = tid; e < 1024; e += 256) {
      const int mm = TA ? (e & 63) : (e >> 4);
      const int kk = TA ? (e >> 6) : (e & 15);
      const long long gm = m0 + mm, gk = k0 + kk;
      float v = 0.0f;
      if (gm < M && gk < kend) v = TA ? A[gk * lda + gm] : A[gm * lda + gk];
      As[kk][mm] = v;
    }
    for (int e = tid; e < 1024; e += 256) {
      const int nn = TB ? (e >> 4) : (e & 63);
      const int kk = TB ? (e & 15) : (e >> 6);
      const long long gn = n0 + nn, gk = k0 + kk;
      float v = 0.0f;
      if (gn < N && gk < kend) v = TB ? B[gn * ldb + gk] : B[gk * ldb + gn];
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      const float4 a = *reinterpret_cast<const float4*>(&As[kk][tm * 4]);
      const float4 bv = *reinterpret_cast<const float4*>(&Bs[kk][tn * 4]);
      const float av[4] = {a.x, a.y, a.z, a.w}, bw[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] += av[r] * bw[c];
    }
    __syncthreads();
  }
  float* Cz = C + (EPI == kEpiPartial ? (long long)blockIdx.z * M * ldc : 0LL);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const long long gm = m0 + tm * 4 + r;
    if (gm >= M) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int gn = n0 + tn * 4 + c;
      if (gn >= N) continue;
      const float v = acc[r][c];
      if (EPI == kEpiPartial) {
        Cz[gm * ldc + gn] = v;
      } else if (EPI == kEpiBiasSilu) {
        const float zz = v + bias[gn];
        Z[gm * ldc + gn] = zz;
        C[gm * ldc + gn] = silu_f(zz);
      } else if (EPI == kEpiBias) {
        C[gm * ldc + gn] = v + bias[gn];
      } else {
        C[gm * ldc + gn] = v * dsilu_f(zprev[gm * ldz + gn]);
      }
    }
  }
}

__global__ void mlp_reduce_kernel(int nz, long long stride, const float* __restrict__ part, float* __restrict__ out,
                                  long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int q = 0; q < nz; ++q) s += part[q * stride + i];
    out[i] = s;
  }
}

// part[z][n] = sum over rows of chunk z of Y[m][n] (column sums for bias gradients)
__global__ void mlp_colsum_kernel(int M, int N, const float* __restrict__ Y, int ldy, int mchunk,
                                  float* __restrict__ part) {
  const int zc = blockIdx.x;
  const long long mb = (long long)zc * mchunk, me = min((long long)M, mb + mchunk);
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    float s = 0.0f;
    for (long long m = mb; m < me; ++m) s += Y[m * ldy + n];
    part[(long long)zc * N + n] = s;
  }
}

// One warp per molecule: projection, squared error and the gradient through
// the projection, gy = gq - mean_molecule(gq) with gq = 2 (q - label) inv_nsh.
__global__ void mlp_project_loss_kernel(int nmol, const int* __restrict__ atom_off, const float* __restrict__ y,
                                        const double* __restrict__ charge, const float* __restrict__ label,
                                        double inv_nsh, float* __restrict__ gy, float* __restrict__ q,
                                        double* __restrict__ loss_mol) {
  const int lane = threadIdx.x & 31;
  const int m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (m >= nmol) return;
  const long long e0 = 2LL * atom_off[m], e1 = 2LL * atom_off[m + 1];
  const int n = (int)(e1 - e0);
  double s = 0.0;
  for (long long e = e0 + lane; e < e1; e += 32) s += (double)y[e];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  const double shift = n ? ((charge ? charge[m] : 0.0) - s) / n : 0.0;
  double l2 = 0.0, gs = 0.0;
  for (long long e = e0 + lane; e < e1; e += 32) {
    const double qq = (double)y[e] + shift;
    if (q) q[e] = (float)qq;
    if (label) {
      const double r = qq - (double)label[e];
      l2 += r * r;
      gs += 2.0 * r * inv_nsh;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    l2 += __shfl_xor_sync(0xffffffffu, l2, o);
    gs += __shfl_xor_sync(0xffffffffu, gs, o);
  }
  if (label && gy) {
    const double gmean = n ? gs / n : 0.0;
    for (long long e = e0 + lane; e < e1; e += 32) {
      const double r = (double)y[e] + shift - (double)label[e];
      gy[e] = (float)(2.0 * r * inv_nsh - gmean);
    }
  }
  if (lane == 0 && loss_mol) loss_mol[m] = l2 * inv_nsh;
}

__global__ void mlp_adam_kernel(long long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
}

}  // namespace

size_t guess_infer_smem_bytes() { return InferSmem::total; }

cudaError_t launch_guess_features(int nmol, const int* atom_off, const int* z, const double* xyz, const float* mean,
                                  const float* stdv, float* x, cudaStream_t st) {
  if (nmol <= 0) return cudaSuccess;
  guess_features_kernel<<<nmol, 128, 0, st>>>(nmol, atom_off, z, xyz, mean, stdv, x);
  return cudaGetLastError();
}

cudaError_t launch_guess_infer(const GuessModel& g, long long natoms, const float* x, float* y, cudaStream_t st) {
  if (natoms <= 0) return cudaSuccess;
  static int configured_dev = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (configured_dev != dev) {
    cudaError_t e = cudaFuncSetAttribute(guess_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)InferSmem::total);
    if (e != cudaSuccess) return e;
    configured_dev = dev;
  }
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long ntiles = (natoms + kTile - 1) / kTile;
  const int grid = (int)(ntiles < nsm ? ntiles : nsm);
  guess_infer_kernel<<<grid, kInferNT, InferSmem::total, st>>>(g.params, g.wbf16, natoms, x, y);
  return cudaGetLastError();
}

cudaError_t launch_guess_project(int nmol, const int* atom_off, const int* shell_off, const int* z, const float* y,
                                 const double* charge, double* init_q, cudaStream_t st) {
  if (nmol <= 0) return cudaSuccess;
  const int threads = 256;
  const long long blocks = ((long long)nmol * 32 + threads - 1) / threads;
  guess_project_kernel<<<(unsigned)blocks, threads, 0, st>>>(nmol, atom_off, shell_off, z, y, charge, init_q);
  return cudaGetLastError();
}

cudaError_t guess_model_upload(const float* host_params, GuessModel& g) {
  g.params = nullptr;
  g.wbf16 = nullptr;
  const long long nw = (long long)kGuessIn * kGuessHid + 2LL * kGuessHid * kGuessHid + kGuessHid * kGuessOut;
  cudaError_t e = cudaMalloc(&g.params, sizeof(float) * kGuessParams);
  if (e == cudaSuccess) e = cudaMalloc(&g.wbf16, sizeof(uint16_t) * nw);
  if (e == cudaSuccess) e = cudaMemcpy(g.params, host_params, sizeof(float) * kGuessParams, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    guess_bf16_kernel<<<64, 256>>>(g.params, g.wbf16);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) guess_model_free(g);
  return e;
}

void guess_model_free(GuessModel& g) {
  if (g.params) cudaFree(g.params);
  if (g.wbf16) cudaFree(g.wbf16);
  g.params = nullptr;
  g.wbf16 = nullptr;
}

}  // namespace gfn1

// ------------------------------------------------------------------ C ABI: training primitives
using namespace gfn1;

static int cuda_status(cudaError_t e) { return e == cudaSuccess ? GFN1_OK : GFN1_E_DEVICE; }

extern "C" int gfn1_mlp_gemm(int ta, int tb, int epi, int M, int N, int K, const float* A, int lda, const float* B,
                             int ldb, const float* bias, const float* zprev, int ldz, float* C, float* Z, int ldc,
                             int ksplit, void* stream) {
  if (M < 0 || N < 0 || K < 0 || !A || !B || !C || epi < 0 || epi > 3 || ksplit < 1) return GFN1_E_INVALID_INPUT;
  if ((epi == kEpiBiasSilu && (!bias || !Z)) || (epi == kEpiBias && !bias) || (epi == kEpiDsilu && !zprev))
    return GFN1_E_INVALID_INPUT;
  if (epi != kEpiPartial && ksplit != 1) return GFN1_E_INVALID_INPUT;
  if (M == 0 || N == 0) return GFN1_OK;
  const int kchunk = (int)((((long long)K + ksplit - 1) / ksplit + 15) / 16 * 16);
  const int nz = K == 0 ? 1 : (int)(((long long)K + kchunk - 1) / kchunk);
  dim3 grid((N + 63) / 64, (M + 63) / 64, nz);
  cudaStream_t st = (cudaStream_t)stream;
#define GFN1_GEMM_CASE(TA_, TB_, E_)                                                                        \
  if (ta == TA_ && tb == TB_ && epi == E_) {                                                                \
    mlp_gemm_kernel<TA_, TB_, E_><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, bias, zprev, ldz, C, Z, ldc, \
                                                        kchunk);                                          \
    return cuda_status(cudaGetLastError());                                                                 \
  }
  GFN1_GEMM_CASE(false, false, kEpiBiasSilu)
  GFN1_GEMM_CASE(false, false, kEpiBias)
  GFN1_GEMM_CASE(false, true, kEpiDsilu)
  GFN1_GEMM_CASE(false, true, kEpiPartial)
  GFN1_GEMM_CASE(true, false, kEpiPartial)
  GFN1_GEMM_CASE(false, false, kEpiPartial)
#undef GFN1_GEMM_CASE
  return GFN1_E_INVALID_INPUT;
}

extern "C" int gfn1_mlp_gemm_splits(int K, int ksplit) {
  if (K <= 0 || ksplit < 1) return 1;
  const long long kchunk = (((long long)K + ksplit - 1) / ksplit + 15) / 16 * 16;
  return (int)(((long long)K + kchunk - 1) / kchunk);
}

extern "C" int gfn1_mlp_reduce(int nz, int64_t stride, const float* part, float* out, int64_t n, void* stream) {
  if (nz < 1 || n < 0 || !part || !out) return GFN1_E_INVALID_INPUT;
  if (n == 0) return GFN1_OK;
  const long long blocks = (n + 255) / 256;
  mlp_reduce_kernel<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0, (cudaStream_t)stream>>>(nz, stride, part,
                                                                                                  out, n);
  return cuda_status(cudaGetLastError());
}

extern "C" int gfn1_mlp_colsum(int M, int N, const float* Y, int ldy, int mchunk, float* part, void* stream) {
  if (M < 0 || N < 1 || N > 1024 || mchunk < 1 || !Y || !part) return GFN1_E_INVALID_INPUT;
  const int nz = M == 0 ? 1 : (M + mchunk - 1) / mchunk;
  mlp_colsum_kernel<<<nz, N < 128 ? 128 : N, 0, (cudaStream_t)stream>>>(M, N, Y, ldy, mchunk, part);
  return cuda_status(cudaGetLastError());
}

extern "C" int gfn1_mlp_project_loss(int nmol, const int32_t* atom_off, const float* y, const double* charge,
                                     const float* label, double inv_nsh, float* gy, float* q, double* loss_mol,
                                     void* stream) {
  if (nmol < 0 || !atom_off || !y) return GFN1_E_INVALID_INPUT;
  if (nmol == 0) return GFN1_OK;
  const long long blocks = ((long long)nmol * 32 + 255) / 256;
  mlp_project_loss_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(nmol, atom_off, y, charge, label,
                                                                              inv_nsh, gy, q, loss_mol);
  return cuda_status(cudaGetLastError());
}

extern "C" int gfn1_mlp_adam(int64_t n, float* p, const float* g, float* m, float* v, float lr, float beta1,
                             float beta2, float eps, float c1, float c2, void* stream) {
  if (n < 0 || !p || !g || !m || !v) return GFN1_E_INVALID_INPUT;
  if (n == 0) return GFN1_OK;
  const long long blocks = (n + 255) / 256;
  mlp_adam_kernel<<<(unsigned)(blocks < 2048 ? blocks : 2048), 256, 0, (cudaStream_t)stream>>>(n, p, g, m, v, lr,
                                                                                               beta1, beta2, eps, c1, c2);
  return cuda_status(cudaGetLastError());
}

extern "C" int gfn1_guess_features_device(int nmol, const int32_t* atom_off, const int32_t* z, const double* xyz,
                                          const float* mean, const float* stdv, float* x, void* stream) {
  if (nmol < 0 || (nmol > 0 && (!atom_off || !z || !xyz || !x)) || ((mean == nullptr) != (stdv == nullptr)))
    return GFN1_E_INVALID_INPUT;
  return cuda_status(launch_guess_features(nmol, atom_off, z, xyz, mean, stdv, x, (cudaStream_t)stream));
}

extern "C" int64_t gfn1_guess_param_count(void) { return kGuessParams; }
