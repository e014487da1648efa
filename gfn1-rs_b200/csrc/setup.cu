// Per-molecule setup kernel: one CTA per molecule builds everything that depends
// on the geometry only.
//
//  * coordination numbers with the exponential count, k = 16, cutoff 30 bohr for
//    H0 and 25 bohr for D3 (src/coordination.rs:51-106, src/dispersion.rs:1245-1251);
//  * self energies se = h - kcn*CN (src/hamiltonian.rs:98-104);
//  * the overlap S and H0 = S * 1/2 (se_i + se_j) * hscale * Pi(R) for every shell
//    pair inside the 30 bohr integral cutoff (src/integrals.rs:133-243,
//    src/hamiltonian.rs:91-134).  Each unordered shell pair is evaluated once and
//    mirrored, where the reference evaluates both directed atom pairs;
//  * the shell-resolved Klopman-Ohno matrix (src/coulomb.rs:82-107);
//  * repulsion energy and gradient (src/repulsion.rs:39-59, :139-159);
//  * D3(BJ) two-body energy and gradient with its CN chain
//    (src/dispersion.rs:1232-1360, :1629-1692, :1753-1787);
//  * the halogen-bond correction, energy and gradient (src/halogen.rs:64-160).
//
// Per-atom sums run one thread per atom over all partners in a fixed order, so
// the results are bitwise reproducible (no floating-point atomics).
#include "common.cuh"
#include "model.cuh"
#include "overlap.cuh"

namespace gfn1 {

__device__ __forceinline__ void tri_inverse(long long w, int& i, int& j) {
  long long ii = (long long)((sqrt(8.0 * (double)w + 1.0) - 1.0) * 0.5);
  while (ii * (ii + 1) / 2 > w) --ii;
  while ((ii + 1) * (ii + 2) / 2 <= w) ++ii;
  i = (int)ii;
  j = (int)(w - ii * (ii + 1) / 2);
}

// S and H0 entries of one shell pair (both triangles); LA, LB are the shells'
// angular momenta, so the overlap block stays in registers.
template <int LA, int LB>
__device__ __forceinline__ void shell_pair_sh0(const ElemTable& ea, int ka, const double* xa, const ElemTable& eb, int kb,
                                               const double* xb, bool zero, double hij, double* S, double* H0, int N,
                                               int mu0, int nu0) {
  double Sb[2 * LA + 1][2 * LB + 1];
  double dummy[2 * LA + 1][2 * LB + 1][3];
  if (!zero)
    overlap_block_any<LA, LB, false>(ea.nprim[ka], ea.alpha[ka], ea.coef[ka], xa, eb.nprim[kb], eb.alpha[kb],
                                     eb.coef[kb], xb, 2, Sb, dummy);
#pragma unroll
  for (int x = 0; x < 2 * LA + 1; ++x)
#pragma unroll
    for (int y = 0; y < 2 * LB + 1; ++y) {
      const double sv = zero ? 0.0 : Sb[x][y];
      const long long i1 = (long long)(mu0 + x) * N + (nu0 + y);
      const long long i2 = (long long)(nu0 + y) * N + (mu0 + x);
      S[i1] = sv;
      S[i2] = sv;
      H0[i1] = sv * hij;
      H0[i2] = sv * hij;
    }
}

// Halogen-bond energy of one molecule; adds its gradient to gc [nat*3].  For
// each donor X with strength c = 0.1 CXB, K is the nearest other atom within
// 20 bohr and every acceptor J (N, O, P, S) within 20 bohr contributes
//   E = c b^6 (u^2 - xbdamp u) / (1 + u^2),  b = 1/2 - T/4,  u = (r0 / r_JX)^6,
// T = (r_KX^2 + r_JX^2 - r_JK^2) / (r_KX r_JX), r0 = xbrad (R_X + R_J), with the
// reference's +1e-18 on r_JX and r_KX.  The gradient is taken through the
// three squared distances.
__device__ double halogen_term(const Model& M, const int* zs, const double* xyz, int nat, double* gc) {
  const double cut2 = 400.0, eps = 1e-18;
  const double damp = M.g.xbdamp, rscale = M.g.xbrad;
  double e = 0.0;
  for (int x = 0; x < nat; ++x) {
    const int zx = zs[x];
    const double c = M.elem[zx].xb;
    if (c == 0.0 || !(zx == 17 || zx == 35 || zx == 53 || zx == 85)) continue;
    int k = -1;  // nearest other atom inside the cutoff (first of equals)
    double kr2 = 0.0;
    for (int j = 0; j < nat; ++j) {
      if (j == x) continue;
      const double dx = xyz[3 * j] - xyz[3 * x], dy = xyz[3 * j + 1] - xyz[3 * x + 1], dz = xyz[3 * j + 2] - xyz[3 * x + 2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 <= 1e-24 || r2 > cut2) continue;
      if (k < 0 || r2 < kr2) {
        k = j;
        kr2 = r2;
      }
    }
    if (k < 0) continue;
    for (int j = 0; j < nat; ++j) {
      const int zj = zs[j];
      if (j == x || !(zj == 7 || zj == 8 || zj == 15 || zj == 16)) continue;
      double vjx[3], vkx[3], vjk[3];
      for (int q = 0; q < 3; ++q) {
        vjx[q] = xyz[3 * j + q] - xyz[3 * x + q];
        vkx[q] = xyz[3 * k + q] - xyz[3 * x + q];
        vjk[q] = xyz[3 * j + q] - xyz[3 * k + q];
      }
      const double djx = vjx[0] * vjx[0] + vjx[1] * vjx[1] + vjx[2] * vjx[2];
      const double dkx = vkx[0] * vkx[0] + vkx[1] * vkx[1] + vkx[2] * vkx[2];
      const double djk = vjk[0] * vjk[0] + vjk[1] * vjk[1] + vjk[2] * vjk[2];
      if (djx <= 1e-24 || djx > cut2 || djx <= eps || dkx <= eps) continue;
      const double rjx = sqrt(djx) + eps, rkx = sqrt(dkx) + eps;
      const double xy = sqrt(dkx * djx);
      if (xy <= eps) continue;
      const double T = (dkx + djx - djk) / xy;
      const double b = 0.5 - 0.25 * T;
      const double b2 = b * b, b5 = b2 * b2 * b, b6 = b5 * b;
      const double r0 = rscale * (M.elem[zx].rad + M.elem[zj].rad);
      const double t1 = r0 / rjx, t3 = t1 * t1 * t1, u = t3 * t3;
      const double num = u * u - damp * u, den = 1.0 + u * u;
      const double L = num / den;
      e += c * b6 * L;
      const double dL = (6.0 * u * (damp - 2.0 * u) / den + 12.0 * u * u * num / (den * den)) / rjx;
      const double dET = -1.5 * c * b5 * L;  // dE/dT
      const double gjx = dET * (1.0 / (rkx * rjx) - 0.5 * T / (rjx * rjx)) + 0.5 * c * b6 * dL / rjx;
      const double gkx = dET * (1.0 / (rkx * rjx) - 0.5 * T / (rkx * rkx));
      const double gjk = -dET / xy;
      for (int q = 0; q < 3; ++q) {
        gc[3 * j + q] += 2.0 * (gjx * vjx[q] + gjk * vjk[q]);
        gc[3 * x + q] -= 2.0 * (gjx * vjx[q] + gkx * vkx[q]);
        gc[3 * k + q] += 2.0 * (gkx * vkx[q] - gjk * vjk[q]);
      }
    }
  }
  return e;
}

// 128-thread CTAs, four per SM (128 registers): the s/p pairs fit, pairs with
// a d shell (rare) keep part of their blocks in local memory.
// Molecule blockIdx.x of `mols` (or of the batch when null).  Large molecules
// are launched with gridDim.y > 1: every CTA of a molecule computes the
// coordination numbers and self energies (cheap, identical), then takes every
// gridDim.y-th block of its shell pairs for S, H0 and the Coulomb matrix; the
// classical terms (repulsion, D3, halogen bonds) stay with blockIdx.y == 0.
// MaxL: the highest shell angular momentum of the batch; the s/p
// instantiation (MaxL = 1) leaves out the d-shell blocks and their registers.
template <int MaxL>
__global__ void __launch_bounds__(128, 4) setup_kernel(Batch B, Model M, int enable_dispersion, int max_nsh,
                                                        const int* mols) {
  extern __shared__ double smem[];
  const int m = mols ? mols[blockIdx.x] : blockIdx.x;
  if (B.status[m] != kOk) return;  // rejected by the host-side validation
  const int split = blockIdx.y, nsplit = gridDim.y;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int a0 = B.atom_off[m], nat = B.atom_off[m + 1] - a0;
  const int sh0 = B.shell_off[m], nsh = B.shell_off[m + 1] - sh0;
  const int N = B.ao_off[m + 1] - B.ao_off[m];
  const int maxn = B.max_nat;
  double* xyz = smem;                 // 3*maxn
  double* cn = xyz + 3 * maxn;        // maxn
  double* cnd = cn + maxn;            // maxn
  double* dedcn = cnd + maxn;         // maxn
  double* gw = dedcn + maxn;          // kMaxRef*maxn
  double* dgw = gw + kMaxRef * maxn;  // kMaxRef*maxn
  double* red = dgw + kMaxRef * maxn; // 32
  int* zs = (int*)(red + 32);         // maxn
  int* atom_sh = zs + maxn;           // maxn+1
  int* atom_ao = atom_sh + maxn + 1;  // maxn+1
  int* sh_atom = atom_ao + maxn + 1;  // max_nsh
  int* sh_k = sh_atom + max_nsh;      // max_nsh

  for (int i = tid; i < nat; i += nt) {
    zs[i] = B.z[a0 + i];
    xyz[3 * i] = B.xyz[3 * (a0 + i)];
    xyz[3 * i + 1] = B.xyz[3 * (a0 + i) + 1];
    xyz[3 * i + 2] = B.xyz[3 * (a0 + i) + 2];
  }
  __syncthreads();
  if (tid == 0) {
    int s = 0, o = 0;
    for (int a = 0; a < nat; ++a) {
      const ElemTable& e = M.elem[zs[a]];
      atom_sh[a] = s;
      atom_ao[a] = o;
      for (int k = 0; k < e.nsh; ++k) {
        sh_atom[s + k] = a;
        sh_k[s + k] = k;
      }
      s += e.nsh;
      o += e.nao;
    }
    atom_sh[nat] = s;
    atom_ao[nat] = o;
  }
  // coordination numbers (both cutoffs), one thread per atom
  for (int i = tid; i < nat; i += nt) {
    const double ri = M.elem[zs[i]].rcov;
    double c30 = 0.0, c25 = 0.0;
    for (int j = 0; j < nat; ++j) {
      if (j == i) continue;
      const double dx = xyz[3 * j] - xyz[3 * i], dy = xyz[3 * j + 1] - xyz[3 * i + 1], dz = xyz[3 * j + 2] - xyz[3 * i + 2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 <= 1e-24 || r2 > 900.0) continue;
      const double rc = ri + M.elem[zs[j]].rcov;
      double v, dv;
      exp_count(sqrt(r2), rc, v, dv);
      c30 += v;
      if (r2 <= 625.0) c25 += v;
    }
    cn[i] = c30;
    cnd[i] = c25;
    B.cn[a0 + i] = c30;
  }
  __syncthreads();
  for (int s = tid; s < nsh; s += nt) {
    const int a = sh_atom[s], k = sh_k[s];
    const ElemTable& e = M.elem[zs[a]];
    B.se[sh0 + s] = e.hdiag[k] - e.kcn[k] * cn[a];
  }
  __syncthreads();

  // ---- S and H0, one work item per unordered shell pair
  double* S = B.S + B.mat_off[m];
  double* H0 = B.H0 + B.mat_off[m];
  const long long npairs = (long long)nsh * (nsh + 1) / 2;
  for (long long w = tid + (long long)split * nt; w < npairs; w += (long long)nt * nsplit) {
    int si, sj;
    tri_inverse(w, si, sj);
    const int a = sh_atom[si], b = sh_atom[sj];
    const int za = zs[a], zb = zs[b];
    const int ka = sh_k[si], kb = sh_k[sj];
    const ElemTable& ea = M.elem[za];
    const ElemTable& eb = M.elem[zb];
    const int la = ea.l[ka], lb = eb.l[kb];
    const int mu0 = atom_ao[a] + ea.ao_first[ka], nu0 = atom_ao[b] + eb.ao_first[kb];
    const double sei = B.se[sh0 + si], sej = B.se[sh0 + sj];
    double hij = 0.0;
    bool zero = false;
    if (a == b) {
      hij = 0.5 * (sei + sej);
    } else {
      const double dx = xyz[3 * a] - xyz[3 * b], dy = xyz[3 * a + 1] - xyz[3 * b + 1], dz = xyz[3 * a + 2] - xyz[3 * b + 2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 <= 1e-24 || r2 > 900.0) {
        zero = true;
      } else {
        const double rr = sqrt(sqrt(r2) / (ea.rad + eb.rad));
        const double poly = (1.0 + ea.poly[ka] * rr) * (1.0 + eb.poly[kb] * rr);
        hij = 0.5 * (sei + sej) * hscale(M, za, ka, zb, kb) * poly;
      }
    }
    if constexpr (MaxL < 2) {
      switch (la * 2 + lb) {
        case 0: shell_pair_sh0<0, 0>(ea, ka, &xyz[3 * a], eb, kb, &xyz[3 * b], zero, hij, S, H0, N, mu0, nu0); break;
        case 1: shell_pair_sh0<0, 1>(ea, ka, &xyz[3 * a], eb, kb, &xyz[3 * b], zero, hij, S, H0, N, mu0, nu0); break;
        case 2: shell_pair_sh0<1, 0>(ea, ka, &xyz[3 * a], eb, kb, &xyz[3 * b], zero, hij, S, H0, N, mu0, nu0); break;
        default: shell_pair_sh0<1, 1>(ea, ka, &xyz[3 * a], eb, kb, &xyz[3 * b], zero, hij, S, H0, N, mu0, nu0); break;
      }
    } else
    switch (la * 3 + lb) {
      case 0: shell_pair_sh0<0, 0>(ea, ka, &xyz[3 * a], eb, kb, &xyz[3 * b], zero, hij, S, H0, N, mu0, nu0); break;
      case 1: shell_pair_sh0<0, 1>(ea, ka, &xyz[3 * a], eb, kb, &xyz[3 * b], zero, hij, S, H0, N, mu0, nu0); break;
      case 2: shell_pair_sh0<0, 2>(ea, ka, &xyz[3 * a], eb, kb, &xyz[3 * b], zero, hij, S, H0, N, mu0, nu0); break;
      case 3: shell_pair_sh0<1, 0>(ea, ka, &xyz[3 * a], eb, kb, &xyz[3 * b], zero, hij, S, H0, N, mu0, nu0); break;
      case 4: shell_pair_sh0<1, 1>(ea, ka, &xyz[3 * a], eb, kb, &xyz[3 * b], zero, hij, S, H0, N, mu0, nu0); break;
      case 5: shell_pair_sh0<1, 2>(ea, ka, &xyz[3 * a], eb, kb, &xyz[3 * b], zero, hij, S, H0, N, mu0, nu0); break;
      case 6: shell_pair_sh0<2, 0>(ea, ka, &xyz[3 * a], eb, kb, &xyz[3 * b], zero, hij, S, H0, N, mu0, nu0); break;
      case 7: shell_pair_sh0<2, 1>(ea, ka, &xyz[3 * a], eb, kb, &xyz[3 * b], zero, hij, S, H0, N, mu0, nu0); break;
      default: shell_pair_sh0<2, 2>(ea, ka, &xyz[3 * a], eb, kb, &xyz[3 * b], zero, hij, S, H0, N, mu0, nu0); break;
    }
  }

  // ---- Klopman-Ohno matrix (exactly symmetric: G_ij and G_ji come from the
  // same commutative expression, which the SCC's column reads rely on)
  double* G = B.gam + B.gam_off[m];
  for (long long w = tid + (long long)split * nt; w < (long long)nsh * nsh; w += (long long)nt * nsplit) {
    const int i = (int)(w / nsh), j = (int)(w % nsh);
    const int a = sh_atom[i], b = sh_atom[j];
    const double g = harmonic_avg(M.elem[zs[a]].hard[sh_k[i]], M.elem[zs[b]].hard[sh_k[j]]);
    double v;
    if (a == b) v = g;
    else {
      const double dx = xyz[3 * a] - xyz[3 * b], dy = xyz[3 * a + 1] - xyz[3 * b + 1], dz = xyz[3 * a + 2] - xyz[3 * b + 2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      v = 1.0 / sqrt(r2 + 1.0 / (g * g));
    }
    G[w] = v;
  }

  if (split != 0) return;  // the classical terms: one CTA per molecule
  // ---- repulsion (pairs within 25 bohr), one thread per atom
  double erep = 0.0;
  for (int i = tid; i < nat; i += nt) {
    const ElemTable& ei = M.elem[zs[i]];
    double gx = 0, gy = 0, gz = 0, e = 0;
    for (int j = 0; j < nat; ++j) {
      if (j == i) continue;
      const ElemTable& ej = M.elem[zs[j]];
      const double dx = xyz[3 * j] - xyz[3 * i], dy = xyz[3 * j + 1] - xyz[3 * i + 1], dz = xyz[3 * j + 2] - xyz[3 * i + 2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 <= 1e-24 || r2 > 625.0) continue;
      const double r = sqrt(r2);
      const double alpha = sqrt(ei.repa * ej.repa);
      const double zeff = ei.repb * ej.repb;
      const double k = (zs[i] <= 2 && zs[j] <= 2) ? M.g.kexplight : M.g.kexp;
      const double rk = pow(r, k);
      const double en = zeff * exp(-alpha * rk) / r;
      const double pref = (alpha * rk * k + 1.0) * en / r2;
      e += 0.5 * en;
      gx += dx * pref;
      gy += dy * pref;
      gz += dz * pref;
    }
    erep += e;
    B.grad_classic[3 * (a0 + i)] = gx;
    B.grad_classic[3 * (a0 + i) + 1] = gy;
    B.grad_classic[3 * (a0 + i) + 2] = gz;
  }
  erep = block_sum(erep, red);

  // ---- D3(BJ)
  double edisp = 0.0;
  if (enable_dispersion) {
    for (int i = tid; i < nat; i += nt) {  // reference weights, src/dispersion.rs:1629-1692
      const ElemTable& e = M.elem[zs[i]];
      const int nr = e.d3_nref;
      double logit[kMaxRef], mx = -INFINITY;
      for (int k = 0; k < nr; ++k) {
        const double d = cnd[i] - e.d3_cnref[k];
        logit[k] = -4.0 * d * d;
        mx = fmax(mx, logit[k]);
      }
      double raw[kMaxRef], norm = 0.0, dnorm = 0.0;
      for (int k = 0; k < nr; ++k) {
        raw[k] = exp(logit[k] - mx);
        norm += raw[k];
        dnorm += 8.0 * (e.d3_cnref[k] - cnd[i]) * raw[k];
      }
      const double ninv = 1.0 / norm;
      for (int k = 0; k < kMaxRef; ++k) {
        double gwk = 0.0, dgk = 0.0;
        if (k < nr) {
          const double expd = 8.0 * (e.d3_cnref[k] - cnd[i]) * raw[k];
          gwk = raw[k] * ninv;
          dgk = expd * ninv - raw[k] * dnorm * ninv * ninv;
          if (!isfinite(gwk)) gwk = 0.0;
          if (!isfinite(dgk)) dgk = 0.0;
        }
        gw[k * maxn + i] = gwk;
        dgw[k * maxn + i] = dgk;
      }
    }
    __syncthreads();
    const double s6 = M.g.s6, s8 = M.g.s8, a1 = M.g.a1, a2 = M.g.a2;
    for (int i = tid; i < nat; i += nt) {  // pair terms, src/dispersion.rs:1260-1297
      const int zi = zs[i];
      const ElemTable& ei = M.elem[zi];
      double gx = 0, gy = 0, gz = 0, e = 0, dc = 0;
      for (int j = 0; j < nat; ++j) {
        if (j == i) continue;
        const int zj = zs[j];
        const ElemTable& ej = M.elem[zj];
        const double dx = xyz[3 * i] - xyz[3 * j], dy = xyz[3 * i + 1] - xyz[3 * j + 1], dz = xyz[3 * i + 2] - xyz[3 * j + 2];
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 <= 1e-24 || r2 > 2500.0 || r2 <= 1e-14) continue;
        const double* c6r = M.c6ref + (long long)(zi * kNZ + zj) * (kMaxRef * kMaxRef);
        double c6 = 0.0, dc6 = 0.0;
        for (int ra = 0; ra < ei.d3_nref; ++ra) {
          double rowc = 0.0;
          for (int rb = 0; rb < ej.d3_nref; ++rb) rowc += gw[rb * maxn + j] * c6r[ra * kMaxRef + rb];
          c6 += gw[ra * maxn + i] * rowc;
          dc6 += dgw[ra * maxn + i] * rowc;
        }
        const double r4r2ij = 3.0 * ei.r4r2 * ej.r4r2;
        const double r0 = a1 * sqrt(r4r2ij) + a2;
        const double r02 = r0 * r0, r06 = r02 * r02 * r02, r08 = r06 * r02;
        const double r4 = r2 * r2;
        const double t6 = 1.0 / (r4 * r2 + r06);
        const double t8 = 1.0 / (r4 * r4 + r08);
        const double d6 = -6.0 * r4 * t6 * t6;
        const double d8 = -8.0 * r4 * r2 * t8 * t8;
        const double ed = s6 * t6 + s8 * r4r2ij * t8;
        const double gd = s6 * d6 + s8 * r4r2ij * d8;
        e -= 0.5 * c6 * ed;
        gx += dx * (-c6 * gd);
        gy += dy * (-c6 * gd);
        gz += dz * (-c6 * gd);
        dc -= dc6 * ed;
      }
      edisp += e;
      dedcn[i] = dc;
      B.grad_classic[3 * (a0 + i)] += gx;
      B.grad_classic[3 * (a0 + i) + 1] += gy;
      B.grad_classic[3 * (a0 + i) + 2] += gz;
    }
    __syncthreads();
    for (int i = tid; i < nat; i += nt) {  // CN chain, src/dispersion.rs:1330-1342
      const double ri = M.elem[zs[i]].rcov;
      double gx = 0, gy = 0, gz = 0;
      for (int j = 0; j < nat; ++j) {
        if (j == i) continue;
        const double dx = xyz[3 * i] - xyz[3 * j], dy = xyz[3 * i + 1] - xyz[3 * j + 1], dz = xyz[3 * i + 2] - xyz[3 * j + 2];
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 <= 1e-24 || r2 > 625.0) continue;
        const double r = sqrt(r2);
        double v, dv;
        exp_count(r, ri + M.elem[zs[j]].rcov, v, dv);
        const double pref = (dedcn[i] + dedcn[j]) * dv / r;
        gx += dx * pref;
        gy += dy * pref;
        gz += dz * pref;
      }
      B.grad_classic[3 * (a0 + i)] += gx;
      B.grad_classic[3 * (a0 + i) + 1] += gy;
      B.grad_classic[3 * (a0 + i) + 2] += gz;
    }
    edisp = block_sum(edisp, red);
  }
  // ---- halogen bonds (src/halogen.rs:64-160, triples :716-786).  Donors
  // (Cl, Br, I, At with a CXB entry) are rare, so one thread sums every triple
  // in atom order and adds the gradient after the per-atom terms above.
  __syncthreads();
  if (tid == 0) {
    const double ehal = halogen_term(M, zs, xyz, nat, B.grad_classic + 3LL * a0);
    double* t = B.terms + (long long)m * kTerms;
    for (int k = 0; k < kTerms; ++k) t[k] = 0.0;
    t[2] = erep;
    t[7] = edisp;
    t[8] = ehal;
  }
}

// Launches the setup kernel for a batch whose highest shell angular momentum
// is max_l (the s/p instantiation below 2).
cudaError_t launch_setup(int max_l, dim3 grid, int nt, size_t smem, cudaStream_t st, const Batch& B, const Model& M,
                         int enable_dispersion, int max_nsh, const int* mols) {
  auto* k = max_l >= 2 ? setup_kernel<2> : setup_kernel<1>;
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k<<<grid, nt, smem, st>>>(B, M, enable_dispersion, max_nsh, mols);
  return cudaGetLastError();
}

}  // namespace gfn1
