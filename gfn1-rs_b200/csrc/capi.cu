// Host side of the engine: table loading, per-element device tables, batch
// layout and the C ABI declared in include/gfn1_b200.h.
//
// Element preparation follows gfn1-rs BasisSet::build (src/basis.rs:121-233):
// STO-nG expansion with normalised primitives (src/sto.rs:790-881), the GFN1
// primitive-count rule (src/basis.rs:251-279), same-centre orthogonalisation of
// a second shell of the same angular momentum (src/basis.rs:318-344), the CN
// shift (src/basis.rs:281-293) and the legacy eV->Eh factor (src/basis.rs:18).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/gfn1_b200.h"
#include "common.cuh"
#include "guess.cuh"
#include "optimize.cuh"
#include "model.cuh"

namespace gfn1 {
cudaError_t launch_setup(int max_l, dim3 grid, int nt, size_t smem, cudaStream_t st, const Batch& B, const Model& M,
                         int enable_dispersion, int max_nsh, const int* mols);
cudaError_t launch_grad(int max_l, dim3 grid, size_t smem, cudaStream_t st, const Batch& B, const Model& M,
                        const int* mols, int phases);
long long scc_workspace_doubles(int maxn, int maxnsh, int cap, int maxnat);
size_t scc_smem_bytes(int maxnsh, int maxn, int maxnat, int matrix_n);
size_t scc_max_dynamic_smem(int nt);
cudaError_t launch_scc(int nt, int grid, size_t smem, cudaStream_t st, const Batch& B, const Model& M,
                       const SccOptions& opt, const SccLaunch& SL);
cudaError_t launch_scc_robust(int nt, int grid, size_t smem, cudaStream_t st, const Batch& B, const Model& M,
                              const SccOptions& opt, const SccLaunch& SL);
// large molecules on many SMs (wide.cuh)
struct WideRuntime;
WideRuntime* wide_runtime_new();
void wide_runtime_delete(WideRuntime* r);
long long wide_slot_doubles(int N, int nsh, int nat, int cap);
cudaError_t wide_bind_runtime(WideRuntime* r, const std::vector<int>& ids, const std::vector<int>& Ns,
                              const std::vector<long long>& mos, const std::vector<int>& nshs,
                              const std::vector<int>& nats, int cap, double* base,
                              const std::vector<long long>& slot_off);
cudaError_t wide_run(const Batch& B, const Model& M, const SccOptions& opt, WideRuntime* r, int nslots, int maxn,
                     int maxnsh, int maxnat, int cap, int num_sms, cudaStream_t st);
void wide_plan_info(const WideRuntime* r, int* nb, int* min_rows, int* group, float* ms, int* tuned);
size_t dense_table_bytes_host(int maxnsh, int maxn, int maxnat);
}  // namespace gfn1

using namespace gfn1;

namespace {

const double kEvToHartreeModel = 1.0 / 27.21138505;  // src/basis.rs:18
const double kAngstromToBohr = 1.8897261246257702;   // src/constants.rs:27
const double kPiHost = 3.14159265358979323846;

thread_local std::string t_error;

struct Tables {
  std::map<std::string, std::vector<double>> kv;
  bool has(const std::string& k) const { return kv.count(k) != 0; }
  const std::vector<double>* get(const std::string& k) const {
    auto it = kv.find(k);
    return it == kv.end() ? nullptr : &it->second;
  }
  double scalar(const std::string& k, double d) const {
    auto p = get(k);
    return p && !p->empty() ? (*p)[0] : d;
  }
};

// C stdio on purpose: the host process may already hold a different libstdc++.
bool load_tables(const char* path, Tables& t, std::string& err) {
  FILE* fp = std::fopen(path, "rb");
  if (!fp) {
    err = std::string("cannot open tables file ") + path;
    return false;
  }
  std::string text;
  char buf[1 << 16];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof buf, fp)) > 0) text.append(buf, got);
  std::fclose(fp);
  size_t pos = 0;
  while (pos < text.size()) {
    size_t eol = text.find('\n', pos);
    if (eol == std::string::npos) eol = text.size();
    std::string line = text.substr(pos, eol - pos);
    pos = eol + 1;
    if (line.empty() || line[0] == '#') continue;
    const char* c = line.c_str();
    while (*c == ' ') ++c;
    const char* ks = c;
    while (*c && *c != ' ') ++c;
    std::string key(ks, c - ks);
    char* end = nullptr;
    long n = std::strtol(c, &end, 10);
    if (end == c || n < 0) {
      err = "bad table line for `" + key + "`";
      return false;
    }
    c = end;
    std::vector<double> v((size_t)n);
    for (long i = 0; i < n; ++i) {
      v[i] = std::strtod(c, &end);
      if (end == c) {
        err = "bad table value for `" + key + "`";
        return false;
      }
      c = end;
    }
    t.kv[key] = std::move(v);
  }
  return true;
}

struct Prim {
  double a, c;
};

// src/sto.rs:790-881
bool sto_ng(const Tables& t, int ng, int n, int l, double zeta, std::vector<Prim>& out) {
  bool special = (n == 6 && ng == 6 && l <= 1);
  if (ng < 1 || ng > 6 || ((n > 5 || n <= l) && !special) || zeta <= 0) return false;
  std::vector<double> alpha(ng), coeff(ng);
  if (special) {
    auto a = t.get(l == 0 ? "sto.alpha6s" : "sto.alpha6p");
    auto c = t.get(l == 0 ? "sto.coeff6s" : "sto.coeff6p");
    if (!a || !c) return false;
    for (int i = 0; i < 6; ++i) {
      alpha[i] = (*a)[i];
      coeff[i] = (*c)[i];
    }
  } else {
    int ityp1 = (l == 0) ? n : (l == 1 ? 4 + n : (l == 2 ? 7 + n : (l == 3 ? 9 + n : 10 + n)));
    if (ityp1 < 1 || ityp1 > 15) return false;
    auto a = t.get("sto.alpha." + std::to_string(ng));
    auto c = t.get("sto.coeff." + std::to_string(ng));
    if (!a || !c) return false;
    for (int i = 0; i < ng; ++i) {
      alpha[i] = (*a)[(ityp1 - 1) * ng + i];
      coeff[i] = (*c)[(ityp1 - 1) * ng + i];
    }
  }
  static const double dfact[8] = {1.0, 1.0, 3.0, 15.0, 105.0, 945.0, 10395.0, 135135.0};
  out.resize(ng);
  for (int i = 0; i < ng; ++i) {
    const double al = alpha[i] * zeta * zeta;
    out[i].a = al;
    out[i].c = coeff[i] * std::pow(2.0 / kPiHost * al, 0.75) * std::pow(std::sqrt(4.0 * al), l) / std::sqrt(dfact[l]);
  }
  return true;
}

// src/basis.rs:318-344
void orthogonalize(const std::vector<Prim>& ref, std::vector<Prim>& sh) {
  double ov = 0.0;
  for (auto& a : ref)
    for (auto& b : sh) ov += a.c * b.c * std::pow(std::sqrt(kPiHost / (a.a + b.a)), 3);
  for (auto& a : ref) sh.push_back({a.a, -ov * a.c});
  double nrm = 0.0;
  for (auto& a : sh)
    for (auto& b : sh) nrm += a.c * b.c * std::pow(std::sqrt(kPiHost / (a.a + b.a)), 3);
  const double sc = 1.0 / std::sqrt(nrm);
  for (auto& p : sh) p.c *= sc;
}

int gfn1_kind(int z) {  // src/basis.rs:295-302
  if (z == 1 || z == 2 || (z >= 6 && z <= 10) || (z >= 14 && z <= 18) || (z >= 32 && z <= 36) ||
      (z >= 50 && z <= 54) || (z >= 82 && z <= 86))
    return 1;
  if (z >= 21 && z <= 24) return 2;
  return 0;
}

// Grow-only device buffer.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  bool ensure(size_t count) {
    if (count <= n && p) return true;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    size_t want = std::max<size_t>(count, 1);
    if (cudaMalloc(&p, want * sizeof(T)) != cudaSuccess) return false;
    n = want;
    return true;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// Grow-only pinned host buffer.
struct HostBuf {
  unsigned char* p = nullptr;
  size_t n = 0;
  bool ensure(size_t bytes) {
    if (bytes <= n && p) return true;
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
    if (cudaHostAlloc((void**)&p, std::max<size_t>(bytes, 256), cudaHostAllocDefault) != cudaSuccess) return false;
    n = std::max<size_t>(bytes, 256);
    return true;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
  }
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Makes `dev` the current device for the scope of an entry point and puts the
// caller's current device back on exit, so that no call of the C ABI leaves
// the calling thread on another device.
struct DeviceGuard {
  int prev = -1;
  cudaError_t status = cudaSuccess;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) status = cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
};

}  // namespace


struct gfn1_batch;

// A learned initial-guess model on the engine's device (FP32 parameters and
// BF16 weight copies).
struct gfn1_guess {
  gfn1_engine* eng = nullptr;
  GuessModel model{};
};

struct gfn1_engine {
  int device = 0;
  int num_sms = 148;
  std::string error;
  ElemTable elem[kNZ];
  bool device_ok[kNZ];
  double refocc_total[kNZ];
  Globals glob;
  std::vector<double> pair_scaling, c6ref;
  ElemTable* d_elem = nullptr;
  double* d_pair = nullptr;
  double* d_c6 = nullptr;
  cudaStream_t stream = nullptr;
  gfn1_batch* oneshot = nullptr;  // reused by gfn1_batch_energy_gradient / gfn1_run
  gfn1_guess* guess = nullptr;    // default initial guess of new batches (not owned)
  Model model() const {
    Model m;
    m.elem = d_elem;
    m.pair_scaling = d_pair;
    m.c6ref = d_c6;
    m.g = glob;
    return m;
  }
};

// Layout of the per-batch input blob (one host->device copy) and output blob
// (one device->host copy); byte offsets, 256-byte aligned.
struct BlobLayout {
  size_t atom_off, shell_off, ao_off, mat_off, gam_off, pair_off, order, status0, z, charge, xyz, init_q, in_bytes;
  size_t terms, grad, shell_q, atom_q, dipole, fermi, iterations, status, rung, out_bytes;
};

struct gfn1_batch {
  gfn1_engine* eng = nullptr;
  int nmol = 0;
  long long natoms = 0, nshells = 0, naos = 0, mat_total = 0, gam_total = 0, pair_total = 0;
  int max_nat = 0, max_nsh = 0, max_n = 0, cap = 0;
  int max_l = 0;  // highest shell angular momentum of the batch (selects the s/p setup and gradient kernels)
  // SCC size classes: [0] molecules above the split size, [1] the rest
  struct SccClass {
    int q_begin = 0, q_end = 0, n_cta = 0, nt = 256, maxn = 0, maxnsh = 0, maxnat = 0;
    long long ws_offset = 0, ws_stride = 0;
    size_t smem = 0;
  } cls[2];
  SccClass robust;  // fallback ladder: workspace for the batch's largest molecule, a few CTAs
  DevBuf<int> failed;
  cudaStream_t side = nullptr;  // second stream for the concurrent class launch
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  gfn1_options opt;
  bool has_init_q = false;
  bool profiling = false;
  DevBuf<int> shift_list;  // with a requested level shift: the molecules for the ladder kernel
  DevBuf<int> shift_count; // their number (copied into queue[3])
  int n_shift = 0;
  std::string host_err;   // message of the first molecule the host validation rejected
  int host_err_mol = -1;  // that molecule, or -1
  // inputs of the last prepare() that gfn1_batch_energy_gradient ran on this
  // batch; a call with the same topology, charges, options, large-molecule
  // threshold and learned guess reuses its layout and only stages the new
  // coordinates (prepare() clears it)
  struct TopologyKey {
    bool valid = false;
    std::vector<int32_t> atom_offsets;
    std::vector<uint8_t> z;
    std::vector<double> charge;  // empty: no charges given
    gfn1_options opt;
    int dense_n = 0;
    gfn1_guess* guess = nullptr;
  } last_topology;
  gfn1_guess* guess = nullptr;       // learned guess used when no initial charges are set
  DevBuf<float> gx, gy;              // guess features [natoms x 100] and outputs [natoms x 2]
  DevBuf<double> gq;                 // guessed initial shell charges [nshells]
  // molecules above the wide threshold: SCC with each molecule on a group of SMs
  std::vector<int> wide_ids;
  int n_dense = 0;  // leading entries of the processing order above the threshold (their setup and gradient split over CTAs)
  int wide_maxn = 0, wide_maxnsh = 0, wide_maxnat = 0;
  WideRuntime* wide = nullptr;
  DevBuf<double> wide_buf;
  BlobLayout lay;
  HostBuf h_in, h_out;               // pinned staging
  DevBuf<unsigned char> d_in, d_out; // device blobs
  DevBuf<double> S, H0, P, W, ws, gam, pairbuf, cn, shell_pot, shell_pot_in, se, grad_classic, orb_eps, orb_occ;
  DevBuf<int> queue;
  // geometry optimisation on the device (gfn1_batch_optimize)
  const int* opt_skip = nullptr;  // molecules the engine kernels skip this round, or null
  DevBuf<unsigned char> opt_mol;
  DevBuf<double> opt_x, opt_g, opt_d, opt_S, opt_Y, opt_q;
  DevBuf<int> opt_flags;          // skip[nmol] | active count
  DevBuf<unsigned long long> stage;
  template <class T>
  T* din(size_t off) const { return (T*)(d_in.p + off); }
  template <class T>
  T* dout(size_t off) const { return (T*)(d_out.p + off); }
  template <class T>
  T* hin(size_t off) const { return (T*)(h_in.p + off); }
  template <class T>
  T* hout(size_t off) const { return (T*)(h_out.p + off); }
  Batch dev() const {
    Batch B;
    std::memset(&B, 0, sizeof B);
    B.nmol = nmol;
    B.max_nat = max_nat;
    B.atom_off = din<int>(lay.atom_off);
    B.shell_off = din<int>(lay.shell_off);
    B.ao_off = din<int>(lay.ao_off);
    B.mat_off = din<long long>(lay.mat_off);
    B.gam_off = din<long long>(lay.gam_off);
    B.pair_off = din<long long>(lay.pair_off);
    B.order = din<int>(lay.order);
    B.z = din<int>(lay.z);
    B.xyz = din<double>(lay.xyz);
    B.charge = din<double>(lay.charge);
    B.init_q = has_init_q ? din<double>(lay.init_q) : (guess ? gq.p : nullptr);
    B.S = S.p;
    B.H0 = H0.p;
    B.P = P.p;
    B.W = W.p;
    B.ws = ws.p;
    B.ws_stride = 0;
    B.ws_maxn = max_n;
    B.ws_maxnsh = max_nsh;
    B.ws_cap = cap;
    B.gam = gam.p;
    B.pairbuf = pairbuf.p;
    B.cn = cn.p;
    B.shell_q = dout<double>(lay.shell_q);
    B.shell_pot = shell_pot.p;
    B.shell_pot_in = shell_pot_in.p;
    B.atom_q = dout<double>(lay.atom_q);
    B.se = se.p;
    B.terms = dout<double>(lay.terms);
    B.grad = dout<double>(lay.grad);
    B.grad_classic = grad_classic.p;
    B.dipole = dout<double>(lay.dipole);
    B.fermi = dout<double>(lay.fermi);
    B.iterations = dout<int>(lay.iterations);
    B.status = dout<int>(lay.status);
    B.rung = dout<int>(lay.rung);
    B.orb_eps = orb_eps.p;
    B.orb_occ = orb_occ.p;
    B.queue = queue.p;
    B.failed = failed.p;
    B.stage_cycles = profiling ? stage.p : nullptr;
    return B;
  }
  void release() {
    h_in.release();
    h_out.release();
    d_in.release();
    d_out.release();
    for (DevBuf<double>* d : {&S, &H0, &P, &W, &ws, &gam, &pairbuf, &cn, &shell_pot, &shell_pot_in, &se, &grad_classic, &orb_eps, &orb_occ})
      d->release();
    queue.release();
    stage.release();
    failed.release();
    gx.release();
    gy.release();
    gq.release();
    wide_buf.release();
    opt_mol.release();
    for (DevBuf<double>* d : {&opt_x, &opt_g, &opt_d, &opt_S, &opt_Y, &opt_q}) d->release();
    opt_flags.release();
    if (wide) wide_runtime_delete(wide);
    wide = nullptr;
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
    ev_fork = ev_join = nullptr;
    side = nullptr;
  }
};

namespace {

int fail(const gfn1_engine* eng, int code, const std::string& msg) {
  t_error = msg;
  if (eng) const_cast<gfn1_engine*>(eng)->error = msg;
  return code;
}

int cuda_fail(const gfn1_engine* eng, cudaError_t e, const char* what) {
  return fail(eng, GFN1_E_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
}

std::string default_tables_path() {
  // <package>/data/gfn1_tables.txt next to <package>/lib/libgfn1_b200.so is
  // resolved by the Python layer; the C ABI accepts an explicit path or the
  // GFN1_B200_TABLES environment variable.
  const char* envp = std::getenv("GFN1_B200_TABLES");
  if (envp && *envp) return envp;
  return "gfn1_tables.txt";
}

bool build_elements(gfn1_engine* eng, const Tables& t, std::string& err) {
  Globals& g = eng->glob;
  g.ks = t.scalar("glob.ks", 1.85);
  g.kp = t.scalar("glob.kp", 2.25);
  g.kd = t.scalar("glob.kd", 2.00);
  g.ksp = t.scalar("glob.ksp", 2.08);
  g.kdiff = t.scalar("glob.kdiff", 2.85);
  g.enscale = t.scalar("glob.enscale", -0.7);
  g.kexp = t.scalar("glob.kexp", 1.5);
  g.kexplight = t.scalar("glob.kexplight", g.kexp);
  g.s6 = t.scalar("glob.s6", 1.0);
  for (const char* k : {"glob.a1", "glob.a2", "glob.s8", "glob.s9", "glob.xbdamp", "glob.xbrad"}) {
    if (!t.has(k)) {
      err = std::string("missing required $globpar entry `") + (k + 5) + "`";
      return false;
    }
  }
  g.a1 = t.scalar("glob.a1", 0);
  g.a2 = t.scalar("glob.a2", 0);
  g.s8 = t.scalar("glob.s8", 0);
  g.xbdamp = t.scalar("glob.xbdamp", 0);  // src/halogen.rs:68-69
  g.xbrad = t.scalar("glob.xbrad", 0);
  if (std::fabs(t.scalar("glob.s9", 0.0)) > 1e-15) {
    err = "D3 three-body term (s9 != 0) is outside the device path";
    return false;
  }
  const double cns = t.scalar("glob.cns", 0.6), cnp = t.scalar("glob.cnp", -0.3);
  const double cnd1 = t.scalar("glob.cnd1", -0.5), cnd2 = t.scalar("glob.cnd2", 0.5);
  auto refocc = t.get("refocc");
  auto radius = t.get("atomic_radius_ang");
  auto covrad = t.get("covrad_ang");
  auto en = t.get("pauling_en");
  auto nref = t.get("d3.nref");
  auto r4r2 = t.get("d3.r4r2");
  if (!refocc || !radius || !covrad || !en || !nref || !r4r2) {
    err = "tables file lacks element data";
    return false;
  }
  for (int z = 0; z < kNZ; ++z) {
    std::memset(&eng->elem[z], 0, sizeof(ElemTable));
    eng->device_ok[z] = false;
    eng->refocc_total[z] = 0.0;
  }
  for (int z = 1; z <= kMaxZ; ++z) {
    const std::string p = "elem." + std::to_string(z) + ".";
    auto ao = t.get(p + "ao");
    auto lev = t.get(p + "lev");
    auto ex = t.get(p + "exp");
    if (!ao || !lev || !ex) continue;
    const int nsh = (int)ao->size() / 2;
    bool ok = nsh <= kMaxShAtom;
    for (int k = 0; k < nsh && ok; ++k)
      if ((int)(*ao)[2 * k + 1] > 2) ok = false;  // device path: s, p and d shells
    if (!ok) continue;
    ElemTable& e = eng->elem[z];
    e.nsh = nsh;
    const double gam = t.scalar(p + "gam", 0.0);
    const double lpar[3] = {t.scalar(p + "lpars", 0.0), t.scalar(p + "lparp", 0.0), t.scalar(p + "lpard", 0.0)};
    const double poly[3] = {t.scalar(p + "polys", 0.0), t.scalar(p + "polyp", 0.0), t.scalar(p + "polyd", 0.0)};
    bool seen[3] = {false, false, false};
    std::vector<Prim> ref[3];
    int nao = 0;
    for (int k = 0; k < nsh; ++k) {
      const int n = (int)(*ao)[2 * k], l = (int)(*ao)[2 * k + 1];
      const bool valence = !seen[l];
      // src/basis.rs:251-279: d shells take 4 primitives
      const int np = (z <= 2) ? (l == 0 ? (n == 1 ? 4 : 3) : (l == 1 ? 3 : 4)) : (l <= 1 ? 6 : 4);
      std::vector<Prim> prims;
      if (!sto_ng(t, np, n, l, (*ex)[k], prims)) {
        ok = false;
        break;
      }
      if (seen[l]) orthogonalize(ref[l], prims);
      else ref[l] = prims;
      seen[l] = true;
      if ((int)prims.size() > kMaxPrim) {
        ok = false;
        break;
      }
      e.l[k] = l;
      e.nprim[k] = (int)prims.size();
      e.valence[k] = valence ? 1 : 0;
      e.ao_first[k] = nao;
      nao += 2 * l + 1;
      for (size_t i = 0; i < prims.size(); ++i) {
        e.alpha[k][i] = prims[i].a;
        e.coef[k][i] = prims[i].c;
      }
      e.hdiag[k] = (*lev)[k] * kEvToHartreeModel;
      const int kind = gfn1_kind(z);
      const double f = kind == 0 ? 0.0 : (l == 0 ? cns : (l == 1 ? cnp : (kind == 1 ? cnd1 : cnd2)));
      e.kcn[k] = -(*lev)[k] * kEvToHartreeModel * f * 0.01;
      e.poly[k] = poly[l] * 0.01;
      e.refocc[k] = valence ? (*refocc)[3 * z + l] : 0.0;
      e.hard[k] = gam * (1.0 + 0.1 * lpar[l]);  // src/params.rs:152-161
      eng->refocc_total[z] += e.refocc[k];
    }
    if (!ok) {
      std::memset(&e, 0, sizeof(ElemTable));
      eng->refocc_total[z] = 0.0;
      continue;
    }
    e.nao = nao;
    e.gam3 = 0.1 * t.scalar(p + "gam3", 0.0);
    e.repa = t.scalar(p + "repa", 0.0);
    e.repb = t.scalar(p + "repb", 0.0);
    e.xb = 0.1 * t.scalar(p + "cxb", 0.0);  // src/halogen.rs:775-786
    e.en = (*en)[z];
    e.rad = (*radius)[z] * kAngstromToBohr;
    e.rcov = (4.0 / 3.0) * (*covrad)[z] * kAngstromToBohr;
    e.r4r2 = std::sqrt(0.5 * (*r4r2)[z - 1] * std::sqrt((double)z));
    e.d3_nref = (int)(*nref)[z - 1];
    auto cref = t.get("d3.cnref." + std::to_string(z));
    if (!cref || e.d3_nref > kMaxRef || e.d3_nref < 1 || e.rad <= 0 || e.rcov <= 0) {
      std::memset(&e, 0, sizeof(ElemTable));
      eng->refocc_total[z] = 0.0;
      continue;
    }
    for (int r = 0; r < e.d3_nref; ++r) e.d3_cnref[r] = (*cref)[r];
    eng->device_ok[z] = true;
  }
  // pair scaling (src/params.rs:361-367, :694-710)
  eng->pair_scaling.assign(kNZ * kNZ, 1.0);
  for (int a = 1; a <= kMaxZ; ++a)
    for (int b = 1; b <= kMaxZ; ++b) {
      auto drow = [](int zz) {
        if (zz >= 21 && zz < 30) return 1.1;
        if (zz >= 39 && zz < 48) return 1.2;
        if (zz >= 57 && zz < 80) return 1.2;
        return -1.0;
      };
      double v = (drow(a) > 0 && drow(b) > 0) ? 0.5 * (drow(a) + drow(b)) : 1.0;
      const std::string key = "pair." + std::to_string(std::min(a, b)) + "." + std::to_string(std::max(a, b));
      if (t.has(key)) v = t.scalar(key, v);
      eng->pair_scaling[a * kNZ + b] = v;
    }
  // D3 reference C6, stored for both element orders (src/dispersion.rs:3145-3164)
  eng->c6ref.assign((size_t)kNZ * kNZ * kMaxRef * kMaxRef, 0.0);
  for (int a = 1; a <= kMaxZ; ++a)
    for (int b = 1; b <= kMaxZ; ++b) {
      if (!eng->device_ok[a] || !eng->device_ok[b]) continue;
      const int hi = std::max(a, b), lo = std::min(a, b);
      auto blk = t.get("d3.c6." + std::to_string(hi) + "." + std::to_string(lo));
      if (!blk) continue;
      const int nhi = eng->elem[hi].d3_nref, nlo = eng->elem[lo].d3_nref;
      for (int ra = 0; ra < eng->elem[a].d3_nref; ++ra)
        for (int rb = 0; rb < eng->elem[b].d3_nref; ++rb) {
          // lookup rule of D3Reference::c6: the larger element's reference first
          int ia, ib;
          if (a > b) {
            ia = ra;
            ib = rb;
          } else {
            ia = rb;
            ib = ra;
          }
          (void)nhi;
          eng->c6ref[((size_t)(a * kNZ + b)) * kMaxRef * kMaxRef + ra * kMaxRef + rb] = (*blk)[ia * nlo + ib];
        }
    }
  return true;
}

void fill_default(gfn1_options* o) {
  o->max_scc = 250;
  o->energy_tolerance = 1e-6;
  o->charge_tolerance = 2e-5;
  o->mixing = 0.4;
  o->scc_broyden = 1;
  o->scc_broyden_size = 250;
  o->electronic_temperature = 300.0;
  o->enable_dispersion = 1;
  o->compute_gradient = 1;
  o->spin_multiplicity = 0;
  o->level_shift = 0.0;
}

// Checks of a requested spin multiplicity (resolve_spin_channels,
// src/electronic.rs:545-598); returns an empty string when it is usable.
std::string spin_multiplicity_error(int mult, double nelec, int norb) {
  if (mult == 0) return "";
  if (mult < 1) return "spin multiplicity must be at least 1";
  const double rounded = std::round(nelec);
  if (std::fabs(nelec - rounded) > 1e-8) return "spin multiplicity requires an integer electron count";
  const long long ne = (long long)rounded, unpaired = mult - 1;
  if (unpaired > ne) return "spin multiplicity needs more unpaired electrons than the system has";
  if ((ne - unpaired) % 2 != 0) return "spin multiplicity " + std::to_string(mult) + " is incompatible with " +
                                       std::to_string(ne) + " electrons";
  if ((ne + unpaired) / 2 > norb) return "spin multiplicity needs more orbitals than the basis has";
  return "";
}

}  // namespace


namespace {

// Fills the topology part of a batch (sizes, offsets, order, element check,
// electron count) into the pinned input blob and grows every buffer.  Buffers
// are never shrunk, so a reused batch allocates only when a larger batch comes.
// Molecules above this many AOs run on groups of SMs (wide.cuh); GFN1_DENSE_N
// overrides the default of 256.
int dense_threshold() {
  int n = 256;
  if (const char* dn = std::getenv("GFN1_DENSE_N"))
    if (*dn) n = std::max(2, std::atoi(dn));
  return n;
}

int prepare(gfn1_batch* b, int nmol, const int32_t* atom_offsets, const uint8_t* z, const double* charge,
            const gfn1_options* opt, std::string& first_err, int& worst) {
  gfn1_engine* eng = b->eng;
  b->last_topology.valid = false;
  gfn1_options o;
  if (opt) o = *opt;
  else fill_default(&o);
  if (o.max_scc < 1) return fail(eng, GFN1_E_INVALID_INPUT, "max_scc must be at least 1");
  if (atom_offsets[0] != 0) return fail(eng, GFN1_E_INVALID_INPUT, "atom_offsets[0] must be 0");
  for (int m = 0; m < nmol; ++m)
    if (atom_offsets[m + 1] < atom_offsets[m]) return fail(eng, GFN1_E_INVALID_INPUT, "atom_offsets must be non-decreasing");
  b->nmol = nmol;
  b->opt = o;
  b->has_init_q = false;
  const long long natoms = atom_offsets[nmol];
  b->natoms = natoms;
  b->max_nat = b->max_nsh = b->max_n = 0;
  b->max_l = 0;
  // sizes first (for the blob layout)
  std::vector<int> nsh_m(nmol), n_m(nmol), st_m(nmol, GFN1_OK);
  std::vector<double> nref_m(nmol, 0.0);
  long long nshells = 0, naos = 0, mat_total = 0, gam_total = 0, pair_total = 0;
  worst = GFN1_OK;
  for (int m = 0; m < nmol; ++m) {
    const int a0 = atom_offsets[m], a1 = atom_offsets[m + 1];
    int n = 0, s = 0, st = GFN1_OK;
    if (a1 <= a0) {
      st = GFN1_E_INVALID_INPUT;
      if (first_err.empty()) first_err = "molecule " + std::to_string(m) + ": cannot run GFN1 SCC for an empty basis";
    }
    for (int a = a0; a < a1; ++a) {
      const int zz = z[a];
      if (zz < 1 || zz > kMaxZ) {
        st = GFN1_E_MISSING_ELEMENT;
        if (first_err.empty()) first_err = "missing GFN1 parameter block for Z=" + std::to_string(zz);
        continue;
      }
      if (!eng->device_ok[zz]) {
        st = std::max(st, (int)GFN1_E_UNSUPPORTED);
        if (first_err.empty()) first_err = "element Z=" + std::to_string(zz) + " is outside the device path";
        continue;
      }
      n += eng->elem[zz].nao;
      s += eng->elem[zz].nsh;
      nref_m[m] += eng->refocc_total[zz];
      for (int k = 0; k < eng->elem[zz].nsh; ++k) b->max_l = std::max(b->max_l, eng->elem[zz].l[k]);
    }
    const double ch = charge ? charge[m] : 0.0;
    const double nelec = nref_m[m] - ch;  // src/electronic.rs:491-510
    if (st == GFN1_OK && (!std::isfinite(nelec) || nelec < -1e-8 || nelec > 2.0 * n + 1e-8)) {
      st = GFN1_E_INVALID_INPUT;
      if (first_err.empty()) first_err = "molecule " + std::to_string(m) + ": invalid electron count";
    }
    if (st == GFN1_OK) {
      const std::string se = spin_multiplicity_error(o.spin_multiplicity, nelec, n);
      if (!se.empty()) {
        st = GFN1_E_INVALID_INPUT;
        if (first_err.empty()) first_err = "molecule " + std::to_string(m) + ": " + se;
      }
    }
    st_m[m] = st;
    worst = std::max(worst, st);
    nsh_m[m] = s;
    n_m[m] = n;
    nshells += s;
    naos += n;
    mat_total += (((long long)n * n + 31) / 32) * 32;
    gam_total += (long long)s * s;
    pair_total += (long long)(a1 - a0) * (a1 - a0 - 1) / 2;
    b->max_nat = std::max(b->max_nat, a1 - a0);
    b->max_nsh = std::max(b->max_nsh, s);
    b->max_n = std::max(b->max_n, n);
  }
  b->nshells = nshells;
  b->naos = naos;
  b->host_err = first_err;
  b->host_err_mol = -1;
  for (int m = 0; m < nmol && b->host_err_mol < 0; ++m)
    if (st_m[m] != GFN1_OK) b->host_err_mol = m;
  b->mat_total = mat_total;
  b->gam_total = gam_total;
  b->pair_total = pair_total;
  // blob layout
  BlobLayout& L = b->lay;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t at = off;
    off = align256(off + bytes);
    return at;
  };
  L.atom_off = take(sizeof(int) * (nmol + 1));
  L.shell_off = take(sizeof(int) * (nmol + 1));
  L.ao_off = take(sizeof(int) * (nmol + 1));
  L.mat_off = take(sizeof(long long) * (nmol + 1));
  L.gam_off = take(sizeof(long long) * (nmol + 1));
  L.pair_off = take(sizeof(long long) * (nmol + 1));
  L.order = take(sizeof(int) * nmol);
  L.status0 = take(sizeof(int) * nmol);
  L.z = take(sizeof(int) * std::max<long long>(natoms, 1));
  L.charge = take(sizeof(double) * nmol);
  L.xyz = take(sizeof(double) * 3 * std::max<long long>(natoms, 1));
  L.init_q = take(sizeof(double) * std::max<long long>(nshells, 1));
  L.in_bytes = off;
  off = 0;
  L.terms = take(sizeof(double) * kTerms * nmol);
  L.grad = take(sizeof(double) * 3 * std::max<long long>(natoms, 1));
  L.shell_q = take(sizeof(double) * std::max<long long>(nshells, 1));
  L.atom_q = take(sizeof(double) * std::max<long long>(natoms, 1));
  L.dipole = take(sizeof(double) * 3 * nmol);
  L.fermi = take(sizeof(double) * nmol);
  L.iterations = take(sizeof(int) * nmol);
  L.status = take(sizeof(int) * nmol);
  L.rung = take(sizeof(int) * nmol);
  L.out_bytes = off;
  if (!b->h_in.ensure(L.in_bytes) || !b->h_out.ensure(L.out_bytes))
    return fail(eng, GFN1_E_DEVICE, "pinned host allocation failed");
  int* h_atom = b->hin<int>(L.atom_off);
  int* h_shell = b->hin<int>(L.shell_off);
  int* h_ao = b->hin<int>(L.ao_off);
  long long* h_mat = b->hin<long long>(L.mat_off);
  long long* h_gam = b->hin<long long>(L.gam_off);
  long long* h_pair = b->hin<long long>(L.pair_off);
  int* h_order = b->hin<int>(L.order);
  int* h_st = b->hin<int>(L.status0);
  int* h_z = b->hin<int>(L.z);
  double* h_ch = b->hin<double>(L.charge);
  h_atom[0] = h_shell[0] = h_ao[0] = 0;
  h_mat[0] = h_gam[0] = h_pair[0] = 0;
  for (int m = 0; m < nmol; ++m) {
    const int a0 = atom_offsets[m], a1 = atom_offsets[m + 1];
    h_atom[m + 1] = a1;
    h_shell[m + 1] = h_shell[m] + nsh_m[m];
    h_ao[m + 1] = h_ao[m] + n_m[m];
    h_mat[m + 1] = h_mat[m] + (((long long)n_m[m] * n_m[m] + 31) / 32) * 32;
    h_gam[m + 1] = h_gam[m] + (long long)nsh_m[m] * nsh_m[m];
    h_pair[m + 1] = h_pair[m] + (long long)(a1 - a0) * (a1 - a0 - 1) / 2;
    h_st[m] = st_m[m];
    h_ch[m] = charge ? charge[m] : 0.0;
    for (int a = a0; a < a1; ++a) {
      const int zz = z[a];
      h_z[a] = (zz >= 1 && zz <= kMaxZ && eng->device_ok[zz]) ? zz : 1;  // rejected molecules are skipped
    }
  }
  // most expensive molecules first (cost ~ N^3)
  for (int m = 0; m < nmol; ++m) h_order[m] = m;
  std::stable_sort(h_order, h_order + nmol, [&](int x, int y) { return n_m[x] > n_m[y]; });
  b->cap = std::max(1, std::min(std::max(o.scc_broyden_size, 2), o.max_scc));
  // two size classes over the sorted order (class 0: N > kSplitN), each with its
  // CTA size; 512 / nt CTAs share an SM, so several molecules interleave on it.
  // Measured on the 4096-molecule batch (SCC stage, zero guess): one 512-thread
  // CTA per SM above 96 AOs 141 ms, 256 threads 126 ms, 128 threads 113 ms,
  // 64 threads 139 ms: four molecules per SM hide each other's barrier and
  // latency stalls, while smaller CTAs lose too much per-molecule parallelism.
  // A class whose vectors do not fit the per-CTA shared memory gets larger CTAs.
  const int kSplitN = 96;
  const int kClassNt[2] = {128, 128};
  // above kDenseN AOs one SM per molecule is too slow: those molecules run on
  // groups of SMs (wide.cuh).  GFN1_DENSE_N overrides the threshold (the tests
  // use it to run both paths on the same molecules).
  const int kDenseN = dense_threshold();
  constexpr int kWideMaxN = 8192;  // the reduction keeps two N-vectors per CTA in shared memory
  int n_dense = 0;
  while (n_dense < nmol && n_m[h_order[n_dense]] > kDenseN) ++n_dense;
  b->n_dense = n_dense;
  b->wide_ids.clear();
  b->wide_maxn = b->wide_maxnsh = b->wide_maxnat = 0;
  for (int q = 0; q < n_dense; ++q) {
    const int mm = h_order[q];
    if (st_m[mm] != GFN1_OK) continue;
    if (n_m[mm] > kWideMaxN) {
      h_st[mm] = st_m[mm] = GFN1_E_INVALID_INPUT;
      worst = std::max(worst, (int)GFN1_E_INVALID_INPUT);
      if (first_err.empty())
        first_err = "molecule " + std::to_string(mm) + ": more than " + std::to_string(kWideMaxN) + " basis functions";
      continue;
    }
    b->wide_ids.push_back(mm);
    b->wide_maxn = std::max(b->wide_maxn, n_m[mm]);
    b->wide_maxnsh = std::max(b->wide_maxnsh, nsh_m[mm]);
    b->wide_maxnat = std::max(b->wide_maxnat, atom_offsets[mm + 1] - atom_offsets[mm]);
  }
  b->n_shift = 0;
  if (o.level_shift != 0.0) {
    if (!std::isfinite(o.level_shift)) return fail(eng, GFN1_E_INVALID_INPUT, "level shift must be finite");
    // molecules on one SM go to the ladder kernel from rung 0; the wide path
    // applies the shift itself
    std::vector<int> lst;
    for (int q = n_dense; q < nmol; ++q) {
      const int mm = h_order[q];
      if (h_st[mm] != GFN1_OK) continue;
      lst.push_back(mm);
    }
    b->n_shift = (int)lst.size();
    if (!b->shift_list.ensure(std::max<size_t>(lst.size(), 1)) || !b->shift_count.ensure(1) ||
        (!lst.empty() && cudaMemcpy(b->shift_list.p, lst.data(), sizeof(int) * lst.size(), cudaMemcpyHostToDevice) !=
                             cudaSuccess) ||
        cudaMemcpy(b->shift_count.p, &b->n_shift, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(eng, GFN1_E_DEVICE, "device copy of the level-shift list failed");
  }
  b->host_err = first_err;
  b->host_err_mol = -1;
  for (int m = 0; m < nmol && b->host_err_mol < 0; ++m)
    if (h_st[m] != GFN1_OK) b->host_err_mol = m;
  int n_large = n_dense;
  while (n_large < nmol && n_m[h_order[n_large]] > kSplitN) ++n_large;
  long long ws_total = 0;
  for (int c = 0; c < 2; ++c) {
    gfn1_batch::SccClass& K = b->cls[c];
    K.q_begin = c == 0 ? n_dense : n_large;
    K.q_end = c == 0 ? n_large : nmol;
    K.nt = kClassNt[c];
    K.maxn = K.maxnsh = K.maxnat = 0;
    for (int q = K.q_begin; q < K.q_end; ++q) {
      const int mm = h_order[q];
      K.maxn = std::max(K.maxn, n_m[mm]);
      K.maxnsh = std::max(K.maxnsh, nsh_m[mm]);
      K.maxnat = std::max(K.maxnat, atom_offsets[mm + 1] - atom_offsets[mm]);
    }
    const int count = K.q_end - K.q_begin;
    const size_t fixed = scc_smem_bytes(K.maxnsh, K.maxn, K.maxnat, 0);
    while (K.nt < 512 && fixed > scc_max_dynamic_smem(K.nt)) K.nt *= 2;  // vectors of big molecules need room
    K.n_cta = count == 0 ? 0 : std::max(1, std::min(count, (kSccThreadsPerSm / K.nt) * eng->num_sms));
    K.ws_stride = count == 0 ? 0 : scc_workspace_doubles(std::max(K.maxn, 1), std::max(K.maxnsh, 1), b->cap,
                                                           std::max(K.maxnat, 1));
    K.ws_offset = ws_total;
    ws_total += K.ws_stride * K.n_cta;
    // Shared memory holds the index tables and vectors only; the working matrix
    // stays in global memory, cached by the L1 that the small carve-out leaves
    // (with four CTAs per SM this measured faster than giving each CTA room for
    // the matrix: 98 vs 105 ms for the SCC stage of the 4096-molecule batch).
    K.smem = fixed;
  }
  {  // fallback ladder: molecules the rung-0 launches leave unconverged, rerun by a few CTAs
    gfn1_batch::SccClass& R = b->robust;
    R.maxn = R.maxnsh = R.maxnat = 0;
    for (int q = n_dense; q < nmol; ++q) {
      const int mm = h_order[q];
      R.maxn = std::max(R.maxn, n_m[mm]);
      R.maxnsh = std::max(R.maxnsh, nsh_m[mm]);
      R.maxnat = std::max(R.maxnat, atom_offsets[mm + 1] - atom_offsets[mm]);
    }
    const int count = nmol - n_dense;
    R.nt = 128;
    const size_t fixed = scc_smem_bytes(R.maxnsh, R.maxn, R.maxnat, 0);
    while (R.nt < 512 && fixed > scc_max_dynamic_smem(R.nt)) R.nt *= 2;
    // a requested level shift runs every molecule on this kernel: full width
    const int width = o.level_shift != 0.0 ? (kSccThreadsPerSm / R.nt) * eng->num_sms : 64;
    R.n_cta = count == 0 ? 0 : std::min(count, width);
    R.ws_stride = count == 0 ? 0 : scc_workspace_doubles(std::max(R.maxn, 1), std::max(R.maxnsh, 1), b->cap,
                                                           std::max(R.maxnat, 1));
    R.ws_offset = ws_total;
    ws_total += R.ws_stride * R.n_cta;
    R.smem = fixed;
  }
  if (!b->side) {
    if (cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) != cudaSuccess)
      return fail(eng, GFN1_E_DEVICE, "stream creation failed");
  }
  bool ok = b->d_in.ensure(L.in_bytes) && b->d_out.ensure(L.out_bytes) && b->queue.ensure(4) &&
            b->failed.ensure((size_t)nmol) &&
            b->stage.ensure(kStages) && b->S.ensure(mat_total) && b->H0.ensure(mat_total) && b->P.ensure(mat_total) &&
            b->W.ensure(mat_total) && b->ws.ensure((size_t)std::max<long long>(ws_total, 1)) && b->gam.ensure(gam_total) &&
            b->pairbuf.ensure(8 * std::max<long long>(pair_total, 1)) && b->cn.ensure(natoms) &&
            b->shell_pot.ensure(nshells) && b->shell_pot_in.ensure(nshells) && b->se.ensure(nshells) && b->grad_classic.ensure(3 * natoms) &&
            b->orb_eps.ensure(std::max<long long>(naos, 1)) && b->orb_occ.ensure(std::max<long long>(naos, 1));
  if (!ok) return fail(eng, GFN1_E_DEVICE, "device allocation failed for the batch workspace");
  if (!b->wide_ids.empty()) {
    std::vector<int> Ns, nshs, nats;
    std::vector<long long> mos, slot_off;
    long long tot = 0;
    for (int mm : b->wide_ids) {  // the SCC vectors of every slot use the CtaWs layout of the largest molecule
      Ns.push_back(n_m[mm]);
      nshs.push_back(b->wide_maxnsh);
      nats.push_back(b->wide_maxnat);
      mos.push_back(h_mat[mm]);
      slot_off.push_back(tot);
      tot += wide_slot_doubles(n_m[mm], b->wide_maxnsh, b->wide_maxnat, b->cap);
    }
    if (!b->wide) b->wide = wide_runtime_new();
    if (!b->wide_buf.ensure((size_t)std::max<long long>(tot, 1)))
      return fail(eng, GFN1_E_DEVICE, "device allocation failed for the large-molecule path");
    if (dense_table_bytes_host(b->wide_maxnsh, b->wide_maxn, b->wide_maxnat) > 200 * 1024)
      return fail(eng, GFN1_E_INVALID_INPUT, "molecule too large for the large-molecule path's index tables");
    cudaError_t e = wide_bind_runtime(b->wide, b->wide_ids, Ns, mos, nshs, nats, b->cap, b->wide_buf.p, slot_off);
    if (e != cudaSuccess) return cuda_fail(eng, e, "large-molecule path set-up");
  }
  b->guess = eng->guess;
  if (b->guess && !(b->gx.ensure((size_t)kGuessIn * std::max<long long>(natoms, 1)) &&
                    b->gy.ensure((size_t)kGuessOut * std::max<long long>(natoms, 1)) &&
                    b->gq.ensure((size_t)std::max<long long>(nshells, 1))))
    return fail(eng, GFN1_E_DEVICE, "device allocation failed for the learned guess");
  return GFN1_OK;
}

// Copies the whole input blob (topology, coordinates, optional initial charges).
int upload_inputs(gfn1_batch* b, cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync(b->d_in.p, b->h_in.p, b->lay.in_bytes, cudaMemcpyHostToDevice, st);
  return e == cudaSuccess ? GFN1_OK : cuda_fail(b->eng, e, "host to device copy");
}

int launch_stage(gfn1_batch* b, int stage, cudaStream_t st) {
  gfn1_engine* eng = b->eng;
  const Batch B = b->dev();
  const Model M = eng->model();
  const int nt = 128;  // setup CTA: four per SM (measured 8.9 against 9.0 ms with 256 threads)
  cudaError_t e = cudaSuccess;
  if (stage == 0) {
    // reset status from the host-validated copy and the work counter
    if ((e = cudaMemcpyAsync(B.status, b->din<int>(b->lay.status0), sizeof(int) * b->nmol, cudaMemcpyDeviceToDevice,
                             st)) != cudaSuccess ||
        (e = cudaMemsetAsync(b->queue.p, 0, sizeof(int) * 4, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(B.rung, 0, sizeof(int) * b->nmol, st)) != cudaSuccess)
      return cuda_fail(eng, e, "batch reset");
    if (b->opt_skip && (e = launch_opt_skip(b->nmol, b->opt_skip, B.status, st)) != cudaSuccess)
      return cuda_fail(eng, e, "optimiser skip list");
    if (b->profiling && (e = cudaMemsetAsync(b->stage.p, 0, sizeof(unsigned long long) * kStages, st)) != cudaSuccess)
      return cuda_fail(eng, e, "batch reset");
    if (b->guess && !b->has_init_q) {  // learned initial shell charges from the device coordinates
      const GuessModel& g = b->guess->model;
      if ((e = launch_guess_features(b->nmol, B.atom_off, B.z, B.xyz, g.params, g.params + kGuessDesc, b->gx.p, st)) !=
              cudaSuccess ||
          (e = launch_guess_infer(g, b->natoms, b->gx.p, b->gy.p, st)) != cudaSuccess ||
          (e = launch_guess_project(b->nmol, B.atom_off, B.shell_off, B.z, b->gy.p, B.charge, b->gq.p, st)) !=
              cudaSuccess)
        return cuda_fail(eng, e, "learned guess");
    }
    const size_t smem = sizeof(double) * (16 * (size_t)b->max_nat + 32) +
                        sizeof(int) * (3 * (size_t)b->max_nat + 2 + 2 * (size_t)b->max_nsh);
    // one CTA per molecule; large molecules (the leading entries of the
    // processing order) with their shell pairs split over many CTAs; the s/p
    // instantiation unless the batch has a d shell
    const int nd = b->n_dense, ns = b->nmol - nd;
    if (ns > 0 && (e = launch_setup(b->max_l, dim3(ns, 1), nt, smem, st, B, M, b->opt.enable_dispersion, b->max_nsh,
                                    B.order + nd)) != cudaSuccess)
      return cuda_fail(eng, e, "setup launch");
    if (nd > 0 && (e = launch_setup(b->max_l, dim3(nd, std::max(1, 4 * eng->num_sms / nd)), nt, smem, st, B, M,
                                    b->opt.enable_dispersion, b->max_nsh, B.order)) != cudaSuccess)
      return cuda_fail(eng, e, "setup launch");
  } else if (stage == 1) {
    SccOptions so;
    so.max_scc = b->opt.max_scc;
    so.broyden = b->opt.scc_broyden;
    so.broyden_size = b->opt.scc_broyden_size;
    so.enable_dispersion = b->opt.enable_dispersion;
    so.energy_tol = b->opt.energy_tolerance;
    so.charge_tol = b->opt.charge_tolerance;
    so.mixing = b->opt.mixing;
    so.etemp = b->opt.electronic_temperature;
    so.spin_mult = b->opt.spin_multiplicity;
    so.level_shift = b->opt.level_shift;
    // fork: the small-molecule class runs on the side stream next to the large one
    if ((e = cudaEventRecord(b->ev_fork, st)) != cudaSuccess || (e = cudaStreamWaitEvent(b->side, b->ev_fork, 0)) != cudaSuccess)
      return cuda_fail(eng, e, "stream fork");
    if (so.level_shift != 0.0 && b->n_shift > 0) {  // every molecule to the ladder kernel, from rung 0
      if ((e = cudaMemcpyAsync(b->failed.p, b->shift_list.p, sizeof(int) * b->n_shift, cudaMemcpyDeviceToDevice, st)) !=
              cudaSuccess ||
          (e = cudaMemcpyAsync(b->queue.p + 3, b->shift_count.p, sizeof(int), cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
        return cuda_fail(eng, e, "level-shift list");
    }
    for (int c = 0; c < 2 && so.level_shift == 0.0; ++c) {
      const gfn1_batch::SccClass& K = b->cls[c];
      if (K.n_cta == 0) continue;
      SccLaunch SL;
      SL.q_begin = K.q_begin;
      SL.q_end = K.q_end;
      SL.counter = b->queue.p + c;
      SL.ws = b->ws.p + K.ws_offset;
      SL.ws_stride = K.ws_stride;
      SL.maxn = K.maxn;
      SL.maxnsh = K.maxnsh;
      SL.maxnat = K.maxnat;
      SL.cap = b->cap;
      SL.smem_bytes = (int)K.smem;
      if ((e = launch_scc(K.nt, K.n_cta, K.smem, c == 0 ? st : b->side, B, M, so, SL)) != cudaSuccess)
        return cuda_fail(eng, e, "scc launch");
    }
    if ((e = cudaEventRecord(b->ev_join, b->side)) != cudaSuccess || (e = cudaStreamWaitEvent(st, b->ev_join, 0)) != cudaSuccess)
      return cuda_fail(eng, e, "stream join");
    if (b->robust.n_cta > 0) {  // rungs 1-3 for whatever rung 0 left unconverged (exits at once if nothing)
      const gfn1_batch::SccClass& R = b->robust;
      SccLaunch SL;
      SL.q_begin = 0;
      SL.q_end = 0;
      SL.counter = b->queue.p + 2;
      SL.ws = b->ws.p + R.ws_offset;
      SL.ws_stride = R.ws_stride;
      SL.maxn = R.maxn;
      SL.maxnsh = R.maxnsh;
      SL.maxnat = R.maxnat;
      SL.cap = b->cap;
      SL.smem_bytes = (int)R.smem;
      if ((e = launch_scc_robust(R.nt, R.n_cta, R.smem, st, B, M, so, SL)) != cudaSuccess)
        return cuda_fail(eng, e, "scc fallback launch");
    }
    if (!b->wide_ids.empty()) {  // large molecules on groups of SMs, after the one-SM classes
      if ((e = wide_run(B, M, so, b->wide, (int)b->wide_ids.size(), b->wide_maxn, b->wide_maxnsh, b->wide_maxnat,
                        b->cap, eng->num_sms, st)) != cudaSuccess)
        return cuda_fail(eng, e, "large-molecule SCC");
    }
  } else if (stage == 2) {
    if (!b->opt.compute_gradient) return GFN1_OK;
    const size_t smem = sizeof(double) * 7 * (size_t)b->max_nat + sizeof(int) * (3 * (size_t)b->max_nat + 2);
    const int nd = b->n_dense, ns = b->nmol - nd;
    if (ns > 0 && (e = launch_grad(b->max_l, dim3(ns, 1), smem, st, B, M, B.order + nd, 3)) != cudaSuccess)
      return cuda_fail(eng, e, "gradient launch");
    if (nd > 0) {  // large molecules: atom pairs over many CTAs, then the per-atom sums
      if ((e = launch_grad(b->max_l, dim3(nd, std::max(1, 4 * eng->num_sms / nd)), smem, st, B, M, B.order, 1)) !=
              cudaSuccess ||
          (e = launch_grad(b->max_l, dim3(nd, 1), smem, st, B, M, B.order, 2)) != cudaSuccess)
        return cuda_fail(eng, e, "gradient launch");
    }
  } else {
    return fail(eng, GFN1_E_INVALID_INPUT, "unknown stage");
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(eng, e, "kernel launch");
  return GFN1_OK;
}

// Synchronises `st`, scatters the output blob into the caller's buffers and
// turns per-molecule statuses into the call's return code.
int finish(gfn1_batch* b, const gfn1_outputs* out, cudaStream_t st) {
  gfn1_engine* eng = b->eng;
  const BlobLayout& L = b->lay;
  cudaError_t e = cudaMemcpyAsync(b->h_out.p, b->d_out.p, L.out_bytes, cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return cuda_fail(eng, e, "device to host copy");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(eng, e, "batch execution");
  const double* terms = b->hout<double>(L.terms);
  const int* status = b->hout<int>(L.status);
  if (out) {
    const int nmol = b->nmol;
    if (out->energy)
      for (int m = 0; m < nmol; ++m) out->energy[m] = terms[(size_t)kTerms * m];
    if (out->terms) std::memcpy(out->terms, terms, sizeof(double) * kTerms * nmol);
    if (out->gradient && b->opt.compute_gradient)
      std::memcpy(out->gradient, b->hout<double>(L.grad), sizeof(double) * 3 * b->natoms);
    if (out->shell_charges) std::memcpy(out->shell_charges, b->hout<double>(L.shell_q), sizeof(double) * b->nshells);
    if (out->atomic_charges) std::memcpy(out->atomic_charges, b->hout<double>(L.atom_q), sizeof(double) * b->natoms);
    if (out->dipole) std::memcpy(out->dipole, b->hout<double>(L.dipole), sizeof(double) * 3 * nmol);
    if (out->fermi_level) std::memcpy(out->fermi_level, b->hout<double>(L.fermi), sizeof(double) * nmol);
    if (out->iterations) std::memcpy(out->iterations, b->hout<int>(L.iterations), sizeof(int) * nmol);
    if (out->status) std::memcpy(out->status, status, sizeof(int) * nmol);
    if (out->rung) {
      const int* rung = b->hout<int>(L.rung);
      for (int m = 0; m < nmol; ++m) out->rung[m] = status[m] == GFN1_OK ? rung[m] : -1;
    }
  }
  int worst = GFN1_OK, first = -1;
  for (int m = 0; m < b->nmol; ++m) {
    if (status[m] > worst) worst = status[m];
    if (status[m] != GFN1_OK && first < 0) first = m;
  }
  if (worst != GFN1_OK && first == b->host_err_mol && !b->host_err.empty()) {
    return fail(eng, worst, b->host_err);  // the host validation's own message
  } else if (worst != GFN1_OK) {
    std::string msg = "molecule " + std::to_string(first) + ": ";
    switch (status[first]) {
      case GFN1_E_SCC_NOT_CONVERGED: msg += "GFN1 SCC did not converge"; break;
      case GFN1_E_INVALID_INPUT: msg += "invalid input (empty molecule, electron count or non-positive-definite overlap)"; break;
      case GFN1_E_UNSUPPORTED: msg += "element outside the device path (no parameters or f shells)"; break;
      case GFN1_E_MISSING_ELEMENT: msg += "missing GFN1 parameter block"; break;
      default: msg += "error " + std::to_string(status[first]);
    }
    return fail(eng, worst, msg);
  }
  return GFN1_OK;
}

bool finite_all(const double* x, long long n) {
  for (long long i = 0; i < n; ++i)
    if (!std::isfinite(x[i])) return false;
  return true;
}

bool finite_all_f(const float* x, long long n) {
  for (long long i = 0; i < n; ++i)
    if (!std::isfinite(x[i])) return false;
  return true;
}

bool same_bits(double x, double y) { return std::memcmp(&x, &y, sizeof(double)) == 0; }

bool same_options(const gfn1_options& a, const gfn1_options& b) {
  return a.max_scc == b.max_scc && same_bits(a.energy_tolerance, b.energy_tolerance) &&
         same_bits(a.charge_tolerance, b.charge_tolerance) && same_bits(a.mixing, b.mixing) &&
         a.scc_broyden == b.scc_broyden && a.scc_broyden_size == b.scc_broyden_size &&
         same_bits(a.electronic_temperature, b.electronic_temperature) &&
         a.enable_dispersion == b.enable_dispersion && a.compute_gradient == b.compute_gradient &&
         a.spin_multiplicity == b.spin_multiplicity && same_bits(a.level_shift, b.level_shift);
}

// Whether a call's topology, charges and options equal those of the last
// prepare() on the one-shot batch (and the large-molecule threshold and the
// engine's learned guess are unchanged), so that its layout, processing order,
// size classes and validated statuses still hold.  Values compare bitwise.
bool same_topology(const gfn1_batch* b, int nmol, const int32_t* atom_offsets, const uint8_t* z, const double* charge,
                   const gfn1_options* opt) {
  const gfn1_batch::TopologyKey& k = b->last_topology;
  if (!k.valid || nmol != b->nmol || (int)k.atom_offsets.size() != nmol + 1) return false;
  if (std::memcmp(k.atom_offsets.data(), atom_offsets, sizeof(int32_t) * (nmol + 1)) != 0) return false;
  const size_t natoms = (size_t)atom_offsets[nmol];
  if (k.z.size() != natoms || (natoms && std::memcmp(k.z.data(), z, natoms) != 0)) return false;
  if (charge ? (k.charge.size() != (size_t)nmol || std::memcmp(k.charge.data(), charge, sizeof(double) * nmol) != 0)
             : !k.charge.empty())
    return false;
  gfn1_options o;
  if (opt) o = *opt;
  else fill_default(&o);
  return same_options(o, k.opt) && k.dense_n == dense_threshold() && k.guess == b->eng->guess;
}

void remember_topology(gfn1_batch* b, int nmol, const int32_t* atom_offsets, const uint8_t* z, const double* charge,
                       const gfn1_options* opt) {
  gfn1_batch::TopologyKey& k = b->last_topology;
  k.atom_offsets.assign(atom_offsets, atom_offsets + nmol + 1);
  k.z.assign(z, z + atom_offsets[nmol]);
  if (charge) k.charge.assign(charge, charge + nmol);
  else k.charge.clear();
  if (opt) k.opt = *opt;
  else fill_default(&k.opt);
  k.dense_n = dense_threshold();
  k.guess = b->eng->guess;
  k.valid = true;
}

}  // namespace

// ============================================================== C ABI
extern "C" {

void gfn1_default_options(gfn1_options* opt) {
  if (opt) fill_default(opt);
}

const char* gfn1_last_error(const gfn1_engine* eng) {
  (void)eng;
  return t_error.c_str();
}

int gfn1_engine_create(const char* param_spec, int device, gfn1_engine** out) {
  if (!out) return fail(nullptr, GFN1_E_INVALID_INPUT, "null output handle");
  *out = nullptr;
  std::string path;
  if (!param_spec || !*param_spec || std::strcmp(param_spec, "builtin") == 0 || std::strcmp(param_spec, "builtin:gfn1") == 0)
    path = default_tables_path();
  else
    path = param_spec;
  Tables t;
  std::string err;
  if (!load_tables(path.c_str(), t, err)) return fail(nullptr, GFN1_E_IO, err);
  gfn1_engine* eng = new gfn1_engine();
  eng->device = device;
  if (!build_elements(eng, t, err)) {
    delete eng;
    return fail(nullptr, GFN1_E_MISSING_GLOBAL, err);
  }
  DeviceGuard dg(device);
  cudaError_t e = dg.status;
  if (e != cudaSuccess) {
    delete eng;
    return cuda_fail(nullptr, e, "cudaSetDevice");
  }
  cudaDeviceGetAttribute(&eng->num_sms, cudaDevAttrMultiProcessorCount, device);
  if ((e = cudaMalloc(&eng->d_elem, sizeof(ElemTable) * kNZ)) != cudaSuccess ||
      (e = cudaMalloc(&eng->d_pair, sizeof(double) * eng->pair_scaling.size())) != cudaSuccess ||
      (e = cudaMalloc(&eng->d_c6, sizeof(double) * eng->c6ref.size())) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&eng->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    gfn1_engine_destroy(eng);
    return cuda_fail(nullptr, e, "engine allocation");
  }
  cudaMemcpy(eng->d_elem, eng->elem, sizeof(ElemTable) * kNZ, cudaMemcpyHostToDevice);
  cudaMemcpy(eng->d_pair, eng->pair_scaling.data(), sizeof(double) * eng->pair_scaling.size(), cudaMemcpyHostToDevice);
  e = cudaMemcpy(eng->d_c6, eng->c6ref.data(), sizeof(double) * eng->c6ref.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    gfn1_engine_destroy(eng);
    return cuda_fail(nullptr, e, "engine table upload");
  }
  *out = eng;
  return GFN1_OK;
}

void gfn1_engine_destroy(gfn1_engine* eng) {
  if (!eng) return;
  if (eng->oneshot) gfn1_batch_destroy(eng->oneshot);
  if (eng->guess) eng->guess->eng = nullptr;
  if (eng->d_elem) cudaFree(eng->d_elem);
  if (eng->d_pair) cudaFree(eng->d_pair);
  if (eng->d_c6) cudaFree(eng->d_c6);
  if (eng->stream) cudaStreamDestroy(eng->stream);
  delete eng;
}

int gfn1_basis_size(const gfn1_engine* eng, int nat, const uint8_t* z, int32_t* nao, int32_t* nshells) {
  if (!eng || nat < 0 || (nat > 0 && !z)) return fail(eng, GFN1_E_INVALID_INPUT, "invalid arguments");
  int n = 0, s = 0;
  for (int a = 0; a < nat; ++a) {
    const int zz = z[a];
    if (zz < 1 || zz > kMaxZ) return fail(eng, GFN1_E_MISSING_ELEMENT, "missing GFN1 parameter block for Z=" + std::to_string(zz));
    if (!eng->device_ok[zz])
      return fail(eng, GFN1_E_UNSUPPORTED, "element Z=" + std::to_string(zz) + " is outside the device path");
    n += eng->elem[zz].nao;
    s += eng->elem[zz].nsh;
  }
  if (nao) *nao = n;
  if (nshells) *nshells = s;
  return GFN1_OK;
}

int gfn1_batch_create(gfn1_engine* eng, int nmol, const int32_t* atom_offsets, const uint8_t* z, const double* charge,
                      const gfn1_options* opt, gfn1_batch** out) {
  if (!eng || !out || nmol < 1 || !atom_offsets || !z) return fail(eng, GFN1_E_INVALID_INPUT, "invalid batch arguments");
  *out = nullptr;
  DeviceGuard dg(eng->device);
  gfn1_batch* b = new gfn1_batch();
  b->eng = eng;
  const char* prof = std::getenv("GFN1_PROFILE");
  b->profiling = prof && *prof && *prof != '0';
  std::string first_err;
  int worst = GFN1_OK;
  int rc = prepare(b, nmol, atom_offsets, z, charge, opt, first_err, worst);
  if (rc == GFN1_OK) rc = upload_inputs(b, eng->stream);
  if (rc == GFN1_OK) {
    cudaError_t e = cudaStreamSynchronize(eng->stream);
    if (e != cudaSuccess) rc = cuda_fail(eng, e, "batch upload");
  }
  if (rc != GFN1_OK) {
    gfn1_batch_destroy(b);
    return rc;
  }
  *out = b;
  if (worst != GFN1_OK) fail(eng, worst, first_err);
  return GFN1_OK;
}

void gfn1_batch_destroy(gfn1_batch* b) {
  if (!b) return;
  b->release();
  delete b;
}

int gfn1_batch_set_positions(gfn1_batch* b, const double* xyz, int on_device) {
  if (!b || !xyz) return fail(b ? b->eng : nullptr, GFN1_E_INVALID_INPUT, "invalid arguments");
  cudaError_t e = cudaMemcpyAsync(b->din<double>(b->lay.xyz), xyz, sizeof(double) * 3 * b->natoms,
                                  on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, b->eng->stream);
  if (e != cudaSuccess) return cuda_fail(b->eng, e, "set positions");
  if (!on_device) e = cudaStreamSynchronize(b->eng->stream);  // the caller may reuse its buffer
  if (e != cudaSuccess) return cuda_fail(b->eng, e, "set positions");
  return GFN1_OK;
}

int gfn1_batch_set_initial_charges(gfn1_batch* b, const double* q, int on_device) {
  if (!b) return fail(nullptr, GFN1_E_INVALID_INPUT, "invalid arguments");
  if (!q) {
    b->has_init_q = false;
    return GFN1_OK;
  }
  cudaError_t e = cudaMemcpyAsync(b->din<double>(b->lay.init_q), q, sizeof(double) * b->nshells,
                                  on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, b->eng->stream);
  if (e == cudaSuccess && !on_device) e = cudaStreamSynchronize(b->eng->stream);
  if (e != cudaSuccess) return cuda_fail(b->eng, e, "set initial charges");
  b->has_init_q = true;
  return GFN1_OK;
}

int gfn1_batch_launch_stage(gfn1_batch* b, int stage, void* stream) {
  if (!b) return fail(nullptr, GFN1_E_INVALID_INPUT, "null batch");
  cudaStream_t st = stream ? (cudaStream_t)stream : b->eng->stream;
  if (stream && stage <= 0) {  // order earlier engine-stream copies before the caller's stream
    cudaEvent_t ev;
    cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    cudaEventRecord(ev, b->eng->stream);
    cudaStreamWaitEvent(st, ev, 0);
    cudaEventDestroy(ev);
  }
  if (stage < 0) {
    for (int s = 0; s < 3; ++s) {
      int rc = launch_stage(b, s, st);
      if (rc != GFN1_OK) return rc;
    }
  } else {
    int rc = launch_stage(b, stage, st);
    if (rc != GFN1_OK) return rc;
  }
  if (stream && (stage < 0 || stage == 2)) {  // later engine-stream copies wait for the caller's stream
    cudaEvent_t ev;
    cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    cudaEventRecord(ev, st);
    cudaStreamWaitEvent(b->eng->stream, ev, 0);
    cudaEventDestroy(ev);
  }
  return GFN1_OK;
}

int gfn1_batch_launch(gfn1_batch* b, void* stream) { return gfn1_batch_launch_stage(b, -1, stream); }

int gfn1_batch_info(const gfn1_batch* b, int64_t* natoms, int64_t* nshells, int64_t* naos, int32_t* launches) {
  if (!b) return fail(nullptr, GFN1_E_INVALID_INPUT, "null batch");
  if (natoms) *natoms = b->natoms;
  if (nshells) *nshells = b->nshells;
  if (naos) *naos = b->naos;
  if (launches) {  // setup, one SCC launch per non-empty size class, the fallback ladder, gradient, learned guess
    const int nd = b->n_dense, ns = b->nmol - nd;  // (the large-molecule SCC launches vary with its iterations)
    *launches = (ns > 0) + (nd > 0) + (b->cls[0].n_cta > 0) + (b->cls[1].n_cta > 0) + (b->robust.n_cta > 0) +
                (b->opt.compute_gradient ? (ns > 0) + 2 * (nd > 0) : 0) + (b->guess && !b->has_init_q ? 3 : 0);
  }
  return GFN1_OK;
}

int gfn1_batch_outputs_device(gfn1_batch* b, gfn1_outputs* out) {
  if (!b || !out) return fail(nullptr, GFN1_E_INVALID_INPUT, "invalid arguments");
  const BlobLayout& L = b->lay;
  out->energy = nullptr;  // total_free is terms[m*15 + 0]
  out->terms = b->dout<double>(L.terms);
  out->gradient = b->dout<double>(L.grad);
  out->shell_charges = b->dout<double>(L.shell_q);
  out->atomic_charges = b->dout<double>(L.atom_q);
  out->dipole = b->dout<double>(L.dipole);
  out->fermi_level = b->dout<double>(L.fermi);
  out->iterations = b->dout<int>(L.iterations);
  out->status = b->dout<int>(L.status);
  out->rung = b->dout<int>(L.rung);
  return GFN1_OK;
}

int gfn1_batch_download(gfn1_batch* b, const gfn1_outputs* out) {
  if (!b) return fail(nullptr, GFN1_E_INVALID_INPUT, "null batch");
  return finish(b, out, b->eng->stream);
}

int gfn1_last_wide_plan(gfn1_engine* eng, int32_t* panel, int32_t* min_rows, int32_t* ctas_per_molecule,
                        double* reduction_ms, int32_t* tuned) {
  if (!eng) return fail(eng, GFN1_E_INVALID_INPUT, "invalid arguments");
  int nb = 0, mr = 0, g = 0, tu = 0;
  float ms = 0.f;
  const gfn1_batch* b = eng->oneshot;
  if (b && b->wide && !b->wide_ids.empty()) wide_plan_info(b->wide, &nb, &mr, &g, &ms, &tu);
  if (panel) *panel = nb;
  if (min_rows) *min_rows = mr;
  if (ctas_per_molecule) *ctas_per_molecule = g;
  if (reduction_ms) *reduction_ms = ms;
  if (tuned) *tuned = tu;
  return GFN1_OK;
}

int gfn1_batch_stage_cycles(const gfn1_batch* b, uint64_t* cycles, int n) {
  if (!b || !cycles) return fail(nullptr, GFN1_E_INVALID_INPUT, "invalid arguments");
  if (!b->profiling) return fail(b->eng, GFN1_E_INVALID_INPUT, "stage profiling is off (set GFN1_PROFILE=1)");
  const int k = std::min(n, (int)kStages);
  cudaError_t e = cudaMemcpy(cycles, b->stage.p, sizeof(uint64_t) * k, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? GFN1_OK : cuda_fail(b->eng, e, "stage cycles");
}

int gfn1_batch_io_bytes(const gfn1_batch* b, int64_t* h2d, int64_t* d2h) {
  if (!b) return fail(nullptr, GFN1_E_INVALID_INPUT, "null batch");
  if (h2d) *h2d = (int64_t)b->lay.in_bytes;
  if (d2h) *d2h = (int64_t)b->lay.out_bytes;
  return GFN1_OK;
}

int gfn1_batch_energy_gradient(gfn1_engine* eng, int nmol, const int32_t* atom_offsets, const uint8_t* z,
                               const double* xyz_bohr, const double* charge, const double* init_shell_q,
                               const gfn1_options* opt, const gfn1_outputs* out) {
  if (!eng || nmol < 1 || !atom_offsets || !z || !xyz_bohr) return fail(eng, GFN1_E_INVALID_INPUT, "invalid arguments");
  DeviceGuard dg(eng->device);
  if (!eng->oneshot) {
    eng->oneshot = new gfn1_batch();
    eng->oneshot->eng = eng;
  }
  gfn1_batch* b = eng->oneshot;
  const char* prof = std::getenv("GFN1_PROFILE");
  b->profiling = prof && *prof && *prof != '0';
  int rc = GFN1_OK;
  if (same_topology(b, nmol, atom_offsets, z, charge, opt)) {
    b->has_init_q = false;  // everything else prepare() sets depends only on the key
  } else {
    std::string first_err;
    int worst = GFN1_OK;
    rc = prepare(b, nmol, atom_offsets, z, charge, opt, first_err, worst);
    if (rc != GFN1_OK) return rc;
    remember_topology(b, nmol, atom_offsets, z, charge, opt);
  }
  if (!finite_all(xyz_bohr, 3 * b->natoms)) return fail(eng, GFN1_E_NAN, "non-finite coordinate");
  std::memcpy(b->hin<double>(b->lay.xyz), xyz_bohr, sizeof(double) * 3 * b->natoms);
  if (init_shell_q) {
    std::memcpy(b->hin<double>(b->lay.init_q), init_shell_q, sizeof(double) * b->nshells);
    b->has_init_q = true;
  }
  cudaStream_t st = eng->stream;
  if ((rc = upload_inputs(b, st)) != GFN1_OK) return rc;
  for (int s = 0; s < 3; ++s)
    if ((rc = launch_stage(b, s, st)) != GFN1_OK) return rc;
  return finish(b, out, st);
}

// S, H0, P, W (N x N, row-major) and the orbital energies / occupations (N)
// of molecule m from the batch's device buffers; every pointer may be null.
static int copy_molecule_matrices(gfn1_batch* b, int m, double* S, double* H0, double* P, double* W, double* eps,
                                  double* occ) {
  gfn1_engine* eng = b->eng;
  if (m < 0 || m >= b->nmol) return fail(eng, GFN1_E_INVALID_INPUT, "molecule index out of range");
  const int* h_ao = b->hin<int>(b->lay.ao_off);
  const long long* h_mat = b->hin<long long>(b->lay.mat_off);
  const size_t n = (size_t)(h_ao[m + 1] - h_ao[m]);
  struct Part {
    double* dst;
    const double* src;
    size_t count;
  } parts[6] = {{S, b->S.p + h_mat[m], n * n},       {H0, b->H0.p + h_mat[m], n * n},
                {P, b->P.p + h_mat[m], n * n},       {W, b->W.p + h_mat[m], n * n},
                {eps, b->orb_eps.p + h_ao[m], n},    {occ, b->orb_occ.p + h_ao[m], n}};
  for (const Part& q : parts) {
    if (!q.dst || q.count == 0) continue;
    cudaError_t e = cudaMemcpy(q.dst, q.src, sizeof(double) * q.count, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(eng, e, "matrix copy");
  }
  return GFN1_OK;
}

// Fock matrix of the last diagonalisation, F = H0 - 1/2 S_mu,nu (v_mu + v_nu)
// with v the AO potential of that diagonalisation's input charges
// (fock_from_shell_potential, src/electronic.rs:3133-3158), the final shell
// potential of the output charges (ElectronicResult::shell_scc_potential,
// src/electronic.rs:1980, 2031) and the atoms' coordination numbers
// (ElectronicResult::coordination_numbers, src/hamiltonian.rs:41, 87).
static int copy_molecule_fock(gfn1_batch* b, int m, double* F, double* shell_potential, double* cn) {
  gfn1_engine* eng = b->eng;
  if (m < 0 || m >= b->nmol) return fail(eng, GFN1_E_INVALID_INPUT, "molecule index out of range");
  const int* h_atom = b->hin<int>(b->lay.atom_off);
  const int* h_shell = b->hin<int>(b->lay.shell_off);
  const int* h_ao = b->hin<int>(b->lay.ao_off);
  const long long* h_mat = b->hin<long long>(b->lay.mat_off);
  const int* h_z = b->hin<int>(b->lay.z);
  const int a0 = h_atom[m], nat = h_atom[m + 1] - a0, sh0 = h_shell[m], nsh = h_shell[m + 1] - sh0;
  const size_t n = (size_t)(h_ao[m + 1] - h_ao[m]);
  cudaError_t e = cudaSuccess;
  if (shell_potential && nsh > 0)
    e = cudaMemcpy(shell_potential, b->shell_pot.p + sh0, sizeof(double) * nsh, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && cn && nat > 0) e = cudaMemcpy(cn, b->cn.p + a0, sizeof(double) * nat, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && F && n > 0) {
    std::vector<double> S(n * n), vin(nsh), vao(n);
    e = cudaMemcpy(F, b->H0.p + h_mat[m], sizeof(double) * n * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(S.data(), b->S.p + h_mat[m], sizeof(double) * n * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(vin.data(), b->shell_pot_in.p + sh0, sizeof(double) * nsh, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) {
      size_t o = 0;
      int s = 0;
      for (int a = 0; a < nat; ++a) {
        const ElemTable& el = eng->elem[h_z[a0 + a]];
        for (int k = 0; k < el.nsh; ++k)
          for (int q = 0; q < 2 * el.l[k] + 1; ++q) vao[o + el.ao_first[k] + q] = vin[s + k];
        s += el.nsh;
        o += el.nao;
      }
      for (size_t i = 0; i < n; ++i)
        for (size_t j = 0; j < n; ++j) F[i * n + j] -= 0.5 * S[i * n + j] * (vao[i] + vao[j]);
    }
  }
  return e == cudaSuccess ? GFN1_OK : cuda_fail(eng, e, "Fock copy");
}

int gfn1_last_molecule_fock(gfn1_engine* eng, int m, double* F, double* shell_potential, double* cn) {
  if (!eng) return fail(nullptr, GFN1_E_INVALID_INPUT, "null engine");
  if (!eng->oneshot || eng->oneshot->nmol < 1) return fail(eng, GFN1_E_INVALID_INPUT, "no calculation on this engine");
  DeviceGuard dg(eng->device);
  cudaError_t e = cudaStreamSynchronize(eng->stream);
  if (e != cudaSuccess) return cuda_fail(eng, e, "stream synchronise");
  return copy_molecule_fock(eng->oneshot, m, F, shell_potential, cn);
}

int gfn1_batch_molecule_fock(gfn1_batch* b, int m, double* F, double* shell_potential, double* cn) {
  if (!b) return fail(nullptr, GFN1_E_INVALID_INPUT, "null batch");
  DeviceGuard dg(b->eng->device);
  cudaError_t e = cudaDeviceSynchronize();  // launches may be on any of the caller's streams
  if (e != cudaSuccess) return cuda_fail(b->eng, e, "device synchronise");
  return copy_molecule_fock(b, m, F, shell_potential, cn);
}

int gfn1_last_molecule_matrices(gfn1_engine* eng, int m, double* S, double* H0, double* P, double* W, double* eps,
                                double* occ) {
  if (!eng) return fail(nullptr, GFN1_E_INVALID_INPUT, "null engine");
  if (!eng->oneshot || eng->oneshot->nmol < 1) return fail(eng, GFN1_E_INVALID_INPUT, "no calculation on this engine");
  DeviceGuard dg(eng->device);
  cudaError_t e = cudaStreamSynchronize(eng->stream);
  if (e != cudaSuccess) return cuda_fail(eng, e, "stream synchronise");
  return copy_molecule_matrices(eng->oneshot, m, S, H0, P, W, eps, occ);
}

int gfn1_batch_molecule_matrices(gfn1_batch* b, int m, double* S, double* H0, double* P, double* W, double* eps,
                                 double* occ) {
  if (!b) return fail(nullptr, GFN1_E_INVALID_INPUT, "null batch");
  DeviceGuard dg(b->eng->device);
  cudaError_t e = cudaDeviceSynchronize();  // launches may be on any of the caller's streams
  if (e != cudaSuccess) return cuda_fail(b->eng, e, "device synchronise");
  return copy_molecule_matrices(b, m, S, H0, P, W, eps, occ);
}

int gfn1_run(gfn1_engine* eng, int nat, const uint8_t* z, const double* xyz_bohr, double charge,
             const double* init_shell_q, const gfn1_options* opt, const gfn1_outputs* out) {
  int32_t off[2] = {0, nat};
  return gfn1_batch_energy_gradient(eng, 1, off, z, xyz_bohr, &charge, init_shell_q, opt, out);
}

int gfn1_guess_create(gfn1_engine* eng, const float* params, int64_t nparams, gfn1_guess** out) {
  if (!eng || !params || !out) return fail(eng, GFN1_E_INVALID_INPUT, "invalid arguments");
  *out = nullptr;
  if (nparams != kGuessParams)
    return fail(eng, GFN1_E_INVALID_INPUT,
                "guess parameter vector has " + std::to_string(nparams) + " values, expected " +
                    std::to_string(kGuessParams));
  if (!finite_all_f(params, nparams)) return fail(eng, GFN1_E_NAN, "non-finite guess parameter");
  for (int f = 0; f < kGuessDesc; ++f)
    if (!(params[kGuessDesc + f] > 0.0f)) return fail(eng, GFN1_E_INVALID_INPUT, "guess feature scale must be positive");
  cudaSetDevice(eng->device);
  gfn1_guess* g = new gfn1_guess();
  g->eng = eng;
  cudaError_t e = guess_model_upload(params, g->model);
  if (e != cudaSuccess) {
    delete g;
    return cuda_fail(eng, e, "guess upload");
  }
  *out = g;
  return GFN1_OK;
}

void gfn1_guess_destroy(gfn1_guess* g) {
  if (!g) return;
  if (g->eng && g->eng->guess == g) g->eng->guess = nullptr;
  if (g->eng && g->eng->oneshot && g->eng->oneshot->guess == g) g->eng->oneshot->guess = nullptr;
  guess_model_free(g->model);
  delete g;
}

int gfn1_engine_set_guess(gfn1_engine* eng, gfn1_guess* g) {
  if (!eng) return fail(nullptr, GFN1_E_INVALID_INPUT, "null engine");
  if (g && g->eng != eng) return fail(eng, GFN1_E_INVALID_INPUT, "guess belongs to another engine");
  eng->guess = g;
  return GFN1_OK;
}

int gfn1_batch_set_guess(gfn1_batch* b, gfn1_guess* g) {
  if (!b) return fail(nullptr, GFN1_E_INVALID_INPUT, "null batch");
  if (g && g->eng != b->eng) return fail(b->eng, GFN1_E_INVALID_INPUT, "guess belongs to another engine");
  b->guess = g;
  if (g && !(b->gx.ensure((size_t)kGuessIn * std::max<long long>(b->natoms, 1)) &&
             b->gy.ensure((size_t)kGuessOut * std::max<long long>(b->natoms, 1)) &&
             b->gq.ensure((size_t)std::max<long long>(b->nshells, 1)))) {
    b->guess = nullptr;
    return fail(b->eng, GFN1_E_DEVICE, "device allocation failed for the learned guess");
  }
  return GFN1_OK;
}

int gfn1_guess_infer_device(gfn1_guess* g, int64_t natoms, const float* x, float* y, void* stream) {
  if (!g || natoms < 0 || (natoms > 0 && (!x || !y))) return fail(g ? g->eng : nullptr, GFN1_E_INVALID_INPUT, "invalid arguments");
  cudaError_t e = launch_guess_infer(g->model, natoms, x, y, (cudaStream_t)stream);
  return e == cudaSuccess ? GFN1_OK : cuda_fail(g->eng, e, "guess inference");
}

int gfn1_guess_predict_device(gfn1_guess* g, int nmol, const int32_t* atom_off, const int32_t* shell_off,
                              const int32_t* z, const double* xyz, const double* charge, float* x_scratch,
                              float* y_scratch, double* init_q, void* stream) {
  if (!g || nmol < 0 || (nmol > 0 && (!atom_off || !shell_off || !z || !xyz || !x_scratch || !y_scratch || !init_q)))
    return fail(g ? g->eng : nullptr, GFN1_E_INVALID_INPUT, "invalid arguments");
  if (nmol == 0) return GFN1_OK;
  cudaStream_t st = (cudaStream_t)stream;
  int32_t n32 = 0;  // total atom count, read back once from the device offsets
  cudaError_t e = cudaMemcpyAsync(&n32, atom_off + nmol, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  const int64_t natoms = n32;
  const GuessModel& m = g->model;
  if (e == cudaSuccess) e = launch_guess_features(nmol, atom_off, z, xyz, m.params, m.params + kGuessDesc, x_scratch, st);
  if (e == cudaSuccess) e = launch_guess_infer(m, natoms, x_scratch, y_scratch, st);
  if (e == cudaSuccess) e = launch_guess_project(nmol, atom_off, shell_off, z, y_scratch, charge, init_q, st);
  return e == cudaSuccess ? GFN1_OK : cuda_fail(g->eng, e, "guess prediction");
}

}  // extern "C"

// ============================================================== no-allocation entry point
//
// gfn1_run_noalloc evaluates one molecule without allocating anything: no
// cudaMalloc, cudaHostAlloc or cudaFree, and no allocating library routine.
// Every device buffer the three kernels need lives in g_noalloc_scratch below,
// a fixed 4.25 MiB array that exists on every GPU that loads this library for
// as long as the process runs.  The host side stages its few kilobytes on the
// stack.  Sizes beyond kNa* are rejected.
namespace {
constexpr int kNaMaxAtoms = 64;
constexpr int kNaMaxAo = 128;
constexpr int kNaMaxShells = 128;
constexpr int kNaMaxHist = 250;
constexpr size_t kNoallocBytes = 4456448;  // 4.25 MiB
constexpr int kNaMaxDevices = 64;
// Device address of the array, per device.  Host threads making their first
// call on a device at the same time store the same value; the atomics keep
// that well defined.
std::atomic<unsigned char*> g_noalloc_dev_ptr[kNaMaxDevices];
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

extern "C" int gfn1_run_noalloc(gfn1_engine* eng, int nat, const uint8_t* z, const double* xyz_bohr, double charge,
                                const double* init_shell_q, const gfn1_options* opt, const gfn1_outputs* out,
                                void* stream) {
  if (!eng || nat < 1 || !z || !xyz_bohr) return fail(eng, GFN1_E_INVALID_INPUT, "invalid arguments");
  gfn1_options o;
  if (opt) o = *opt;
  else fill_default(&o);
  if (o.max_scc < 1) return fail(eng, GFN1_E_INVALID_INPUT, "max_scc must be at least 1");
  if (nat > kNaMaxAtoms)
    return fail(eng, GFN1_E_INVALID_INPUT, "gfn1_run_noalloc handles at most " + std::to_string(kNaMaxAtoms) +
                                               " atoms; got " + std::to_string(nat) + " (use gfn1_run)");
  int n = 0, nsh = 0;
  double nref = 0.0;
  for (int a = 0; a < nat; ++a) {
    const int zz = z[a];
    if (zz < 1 || zz > kMaxZ) return fail(eng, GFN1_E_MISSING_ELEMENT, "missing GFN1 parameter block for Z=" + std::to_string(zz));
    if (!eng->device_ok[zz])
      return fail(eng, GFN1_E_UNSUPPORTED, "element Z=" + std::to_string(zz) + " is outside the device path");
    n += eng->elem[zz].nao;
    nsh += eng->elem[zz].nsh;
    nref += eng->refocc_total[zz];
  }
  const int cap = std::max(1, std::min(std::max(o.scc_broyden_size, 2), o.max_scc));
  if (n > kNaMaxAo || nsh > kNaMaxShells)
    return fail(eng, GFN1_E_INVALID_INPUT, "gfn1_run_noalloc handles at most " + std::to_string(kNaMaxAo) +
                                               " AOs and shells; got " + std::to_string(n) + " AOs, " +
                                               std::to_string(nsh) + " shells (use gfn1_run)");
  if (cap > kNaMaxHist)
    return fail(eng, GFN1_E_INVALID_INPUT, "gfn1_run_noalloc keeps at most " + std::to_string(kNaMaxHist) +
                                               " Broyden history vectors (min(scc_broyden_size, max_scc))");
  if (!finite_all(xyz_bohr, 3LL * nat)) return fail(eng, GFN1_E_NAN, "non-finite coordinate");
  const double nelec = nref - charge;
  if (!std::isfinite(nelec) || nelec < -1e-8 || nelec > 2.0 * n + 1e-8)
    return fail(eng, GFN1_E_INVALID_INPUT, "invalid electron count");
  {
    const std::string se = spin_multiplicity_error(o.spin_multiplicity, nelec, n);
    if (!se.empty()) return fail(eng, GFN1_E_INVALID_INPUT, se);
  }
  if (o.level_shift != 0.0)
    return fail(eng, GFN1_E_INVALID_INPUT, "gfn1_run_noalloc runs without a level shift (use gfn1_run)");
  const int dev = eng->device;
  if (dev < 0 || dev >= kNaMaxDevices) return fail(eng, GFN1_E_INVALID_INPUT, "device ordinal out of range");
  DeviceGuard dg(dev);  // the caller's current device comes back on return
  cudaError_t e = dg.status;
  if (e != cudaSuccess) return cuda_fail(eng, e, "cudaSetDevice");
  unsigned char* base = g_noalloc_dev_ptr[dev].load(std::memory_order_acquire);
  if (!base) {  // once per device, with that device current
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(eng, e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    base = (unsigned char*)p;
    g_noalloc_dev_ptr[dev].store(base, std::memory_order_release);
  }
  cudaStream_t st = stream ? (cudaStream_t)stream : eng->stream;

  // ---- layout inside the scratch array (byte offsets, 256-aligned)
  const long long n2 = (((long long)n * n + 31) / 32) * 32;
  const long long npair = (long long)nat * (nat - 1) / 2;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t at = off;
    off = align256(off + bytes);
    return at;
  };
  // input region, mirrored by the stack staging buffer
  const size_t i_atom = take(2 * sizeof(int)), i_shell = take(2 * sizeof(int)), i_ao = take(2 * sizeof(int));
  const size_t i_mat = take(2 * sizeof(long long)), i_gam = take(2 * sizeof(long long)),
               i_pair = take(2 * sizeof(long long));
  const size_t i_order = take(sizeof(int)), i_st0 = take(sizeof(int)), i_z = take(sizeof(int) * nat);
  const size_t i_charge = take(sizeof(double)), i_xyz = take(sizeof(double) * 3 * nat),
               i_q0 = take(sizeof(double) * nsh);
  const size_t in_bytes = off;
  // output region
  const size_t o_terms = take(sizeof(double) * kTerms), o_grad = take(sizeof(double) * 3 * nat),
               o_shq = take(sizeof(double) * nsh), o_atq = take(sizeof(double) * nat),
               o_dip = take(sizeof(double) * 3), o_fermi = take(sizeof(double)), o_iter = take(sizeof(int)),
               o_status = take(sizeof(int));
  const size_t out_end = off;
  // work region
  const size_t w_S = take(sizeof(double) * n2), w_H0 = take(sizeof(double) * n2), w_P = take(sizeof(double) * n2),
               w_W = take(sizeof(double) * n2);
  const long long ws_doubles = scc_workspace_doubles(n, nsh, cap, nat);
  const size_t w_ws = take(sizeof(double) * ws_doubles), w_gam = take(sizeof(double) * (size_t)nsh * nsh),
               w_pair = take(sizeof(double) * 8 * std::max<long long>(npair, 1)), w_cn = take(sizeof(double) * nat),
               w_pot = take(sizeof(double) * nsh), w_se = take(sizeof(double) * nsh),
               w_gcl = take(sizeof(double) * 3 * nat), w_queue = take(4 * sizeof(int));
  // the engine's learned guess (as gfn1_run uses it) when the caller gives no
  // initial charges: descriptors and network outputs of the molecule's atoms
  const bool use_guess = eng->guess != nullptr && init_shell_q == nullptr;
  const size_t w_gx = use_guess ? take(sizeof(float) * kGuessIn * nat) : 0,
               w_gy = use_guess ? take(sizeof(float) * kGuessOut * nat) : 0;
  if (off > kNoallocBytes) return fail(eng, GFN1_E_INVALID_INPUT, "molecule exceeds the no-allocation scratch");

  // ---- stage inputs on the stack and copy them into the scratch array
  alignas(256) unsigned char hin[12288];
  alignas(256) unsigned char hout[8192];
  if (in_bytes > sizeof hin || out_end - o_terms > sizeof hout)
    return fail(eng, GFN1_E_INVALID_INPUT, "molecule exceeds the no-allocation staging buffers");
  std::memset(hin, 0, in_bytes);
  ((int*)(hin + i_atom))[1] = nat;
  ((int*)(hin + i_shell))[1] = nsh;
  ((int*)(hin + i_ao))[1] = n;
  ((long long*)(hin + i_mat))[1] = n2;
  ((long long*)(hin + i_gam))[1] = (long long)nsh * nsh;
  ((long long*)(hin + i_pair))[1] = npair;
  for (int a = 0; a < nat; ++a) ((int*)(hin + i_z))[a] = z[a];
  *(double*)(hin + i_charge) = charge;
  std::memcpy(hin + i_xyz, xyz_bohr, sizeof(double) * 3 * nat);
  if (init_shell_q) std::memcpy(hin + i_q0, init_shell_q, sizeof(double) * nsh);
  if ((e = cudaMemcpyAsync(base, hin, in_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return cuda_fail(eng, e, "host to device copy");
  // every call reuses the array: clear what the kernels expect to start at zero
  if ((e = cudaMemsetAsync(base + o_status, 0, sizeof(int), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(base + w_queue, 0, 4 * sizeof(int), st)) != cudaSuccess)
    return cuda_fail(eng, e, "scratch reset");

  Batch B;
  std::memset(&B, 0, sizeof B);
  B.nmol = 1;
  B.max_nat = nat;
  B.atom_off = (const int*)(base + i_atom);
  B.shell_off = (const int*)(base + i_shell);
  B.ao_off = (const int*)(base + i_ao);
  B.mat_off = (const long long*)(base + i_mat);
  B.gam_off = (const long long*)(base + i_gam);
  B.pair_off = (const long long*)(base + i_pair);
  B.order = (const int*)(base + i_order);
  B.z = (const int*)(base + i_z);
  B.xyz = (const double*)(base + i_xyz);
  B.charge = (const double*)(base + i_charge);
  B.init_q = (init_shell_q || use_guess) ? (const double*)(base + i_q0) : nullptr;
  B.S = (double*)(base + w_S);
  B.H0 = (double*)(base + w_H0);
  B.P = (double*)(base + w_P);
  B.W = (double*)(base + w_W);
  B.ws = (double*)(base + w_ws);
  B.ws_stride = ws_doubles;
  B.ws_maxn = n;
  B.ws_maxnsh = nsh;
  B.ws_cap = cap;
  B.gam = (double*)(base + w_gam);
  B.pairbuf = (double*)(base + w_pair);
  B.cn = (double*)(base + w_cn);
  B.shell_q = (double*)(base + o_shq);
  B.shell_pot = (double*)(base + w_pot);
  B.atom_q = (double*)(base + o_atq);
  B.se = (double*)(base + w_se);
  B.terms = (double*)(base + o_terms);
  B.grad = (double*)(base + o_grad);
  B.grad_classic = (double*)(base + w_gcl);
  B.dipole = (double*)(base + o_dip);
  B.fermi = (double*)(base + o_fermi);
  B.iterations = (int*)(base + o_iter);
  B.status = (int*)(base + o_status);
  B.queue = (int*)(base + w_queue);
  B.stage_cycles = nullptr;
  const Model M = eng->model();
  SccOptions so;
  so.max_scc = o.max_scc;
  so.broyden = o.scc_broyden;
  so.broyden_size = o.scc_broyden_size;
  so.enable_dispersion = o.enable_dispersion;
  so.energy_tol = o.energy_tolerance;
  so.charge_tol = o.charge_tolerance;
  so.mixing = o.mixing;
  so.etemp = o.electronic_temperature;
  so.spin_mult = o.spin_multiplicity;
  so.level_shift = 0.0;
  const size_t sm_setup = sizeof(double) * (16 * (size_t)nat + 32) + sizeof(int) * (3 * (size_t)nat + 2 + 2 * (size_t)nsh);
  const size_t sm_scc = std::max(scc_smem_bytes(nsh, n, nat, 0),
                                 std::min(scc_smem_bytes(nsh, n, nat, n), scc_max_dynamic_smem(n > 96 ? 512 : 256)));
  const size_t sm_grad = sizeof(double) * 7 * (size_t)nat + sizeof(int) * (3 * (size_t)nat + 2);
  if (use_guess) {  // predicted shell charges into the initial-charge slot of the input region
    const GuessModel& g = eng->guess->model;
    float* gx = (float*)(base + w_gx);
    float* gy = (float*)(base + w_gy);
    if ((e = launch_guess_features(1, B.atom_off, B.z, B.xyz, g.params, g.params + kGuessDesc, gx, st)) !=
            cudaSuccess ||
        (e = launch_guess_infer(g, nat, gx, gy, st)) != cudaSuccess ||
        (e = launch_guess_project(1, B.atom_off, B.shell_off, B.z, gy, B.charge, (double*)(base + i_q0), st)) !=
            cudaSuccess)
      return cuda_fail(eng, e, "learned guess");
  }
  if ((e = launch_setup(2, dim3(1), 128, sm_setup, st, B, M, o.enable_dispersion, nsh, nullptr)) != cudaSuccess)
    return cuda_fail(eng, e, "setup launch");
  SccLaunch SL;
  SL.q_begin = 0;
  SL.q_end = 1;
  SL.counter = B.queue;
  SL.ws = B.ws;
  SL.ws_stride = ws_doubles;
  SL.maxn = n;
  SL.maxnsh = nsh;
  SL.maxnat = nat;
  SL.cap = cap;
  SL.smem_bytes = (int)sm_scc;
  if ((e = launch_scc(n > 96 ? 512 : 256, 1, sm_scc, st, B, M, so, SL)) != cudaSuccess)
    return cuda_fail(eng, e, "scc launch");
  if (o.compute_gradient && (e = launch_grad(2, dim3(1), sm_grad, st, B, M, nullptr, 3)) != cudaSuccess)
    return cuda_fail(eng, e, "gradient launch");
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(eng, e, "kernel launch");
  if ((e = cudaMemcpyAsync(hout, base + o_terms, out_end - o_terms, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return cuda_fail(eng, e, "device to host copy");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(eng, e, "no-allocation run");
  auto hp = [&](size_t o_) { return hout + (o_ - o_terms); };
  const int status = *(const int*)hp(o_status);
  const double* terms = (const double*)hp(o_terms);
  if (out) {
    if (out->energy) out->energy[0] = terms[0];
    if (out->terms) std::memcpy(out->terms, terms, sizeof(double) * kTerms);
    if (out->gradient && o.compute_gradient) std::memcpy(out->gradient, hp(o_grad), sizeof(double) * 3 * nat);
    if (out->shell_charges) std::memcpy(out->shell_charges, hp(o_shq), sizeof(double) * nsh);
    if (out->atomic_charges) std::memcpy(out->atomic_charges, hp(o_atq), sizeof(double) * nat);
    if (out->dipole) std::memcpy(out->dipole, hp(o_dip), sizeof(double) * 3);
    if (out->fermi_level) std::memcpy(out->fermi_level, hp(o_fermi), sizeof(double));
    if (out->iterations) std::memcpy(out->iterations, hp(o_iter), sizeof(int));
    if (out->status) out->status[0] = status;
    if (out->rung) out->rung[0] = status == GFN1_OK ? 0 : -1;  // this entry point runs rung 0 only
  }
  if (status != GFN1_OK)
    return fail(eng, status, status == GFN1_E_SCC_NOT_CONVERGED ? "GFN1 SCC did not converge"
                                                                 : "molecule failed with status " + std::to_string(status));
  return GFN1_OK;
}

// ============================================================== geometry optimisation
extern "C" void gfn1_default_opt_options(gfn1_opt_options* o) {
  if (!o) return;
  o->max_iterations = 250;  // GeometryOptimizationOptions defaults (src/optimizer.rs:27-50)
  o->gradient_tolerance = 1.0e-4;
  o->step_tolerance = 1.0e-7;
  o->history = 12;
  o->initial_step = 1.0;
  o->max_atom_step = 0.30;
  o->max_rounds = 100000;
}

extern "C" int gfn1_batch_optimize(gfn1_batch* b, const gfn1_opt_options* opt, double* xyz_out, double* energy,
                                   double* max_gradient, int32_t* iterations, int32_t* converged, int32_t* status,
                                   int32_t* rounds) {
  if (!b) return fail(nullptr, GFN1_E_INVALID_INPUT, "null batch");
  gfn1_engine* eng = b->eng;
  if (!b->opt.compute_gradient) return fail(eng, GFN1_E_INVALID_INPUT, "the batch was created without gradients");
  gfn1_opt_options o;
  if (opt) o = *opt;
  else gfn1_default_opt_options(&o);
  if (o.history < 1 || o.history > 12 || o.max_iterations < 0 || o.max_rounds < 1)
    return fail(eng, GFN1_E_INVALID_INPUT, "optimiser options out of range (history 1..12)");
  DeviceGuard dg(eng->device);
  cudaStream_t st = eng->stream;
  const int nmol = b->nmol;
  const long long n3 = 3 * b->natoms;
  const int H = o.history;
  if (!b->opt_mol.ensure(opt_mol_bytes() * nmol) || !b->opt_x.ensure(n3) || !b->opt_g.ensure(n3) ||
      !b->opt_d.ensure(n3) || !b->opt_S.ensure((size_t)H * n3) || !b->opt_Y.ensure((size_t)H * n3) ||
      !b->opt_q.ensure((size_t)std::max<long long>(b->nshells, 1)) || !b->opt_flags.ensure((size_t)nmol + 1))
    return fail(eng, GFN1_E_DEVICE, "device allocation failed for the optimiser");
  OptArrays A;
  A.mol = (OptMol*)b->opt_mol.p;
  A.x = b->opt_x.p;
  A.g = b->opt_g.p;
  A.d = b->opt_d.p;
  A.S = b->opt_S.p;
  A.Y = b->opt_Y.p;
  A.q = b->opt_q.p;
  A.x_in = b->din<double>(b->lay.xyz);
  A.q_in = b->din<double>(b->lay.init_q);
  A.skip = b->opt_flags.p;
  A.active = b->opt_flags.p + nmol;
  A.n3 = n3;
  OptParams P;
  P.max_iterations = o.max_iterations;
  P.history = H;
  P.gradient_tolerance = o.gradient_tolerance;
  P.step_tolerance = o.step_tolerance;
  P.initial_step = o.initial_step;
  P.max_atom_step = o.max_atom_step;
  const bool had_init_q = b->has_init_q;
  b->opt_skip = nullptr;
  int rc = GFN1_OK;
  int nround = 0;
  cudaError_t e = cudaSuccess;
  auto run_engine = [&]() {
    for (int s = 0; s < 3 && rc == GFN1_OK; ++s) rc = launch_stage(b, s, st);
  };
  // the starting geometries
  run_engine();
  if (rc == GFN1_OK && (e = cudaMemsetAsync(A.active, 0, sizeof(int), st)) != cudaSuccess) rc = cuda_fail(eng, e, "optimiser");
  if (rc == GFN1_OK && (e = launch_opt_round(b->dev(), A, P, nmol, 1, st)) != cudaSuccess) rc = cuda_fail(eng, e, "optimiser");
  // rounds: every pending trial geometry of every molecule in one engine pass
  while (rc == GFN1_OK) {
    int act = 0;
    if ((e = cudaMemcpyAsync(&act, A.active, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
      rc = cuda_fail(eng, e, "optimiser round");
      break;
    }
    if (act == 0 || nround >= o.max_rounds) break;
    ++nround;
    b->has_init_q = true;  // trials start from the current geometries' converged charges
    b->opt_skip = A.skip;
    run_engine();
    if (rc != GFN1_OK) break;
    if ((e = cudaMemsetAsync(A.active, 0, sizeof(int), st)) != cudaSuccess ||
        (e = launch_opt_round(b->dev(), A, P, nmol, 0, st)) != cudaSuccess)
      rc = cuda_fail(eng, e, "optimiser round");
  }
  b->opt_skip = nullptr;
  b->has_init_q = had_init_q;
  if (rc != GFN1_OK) return rc;
  if ((e = launch_opt_final(b->dev(), A, nmol, st)) != cudaSuccess) return cuda_fail(eng, e, "optimiser results");
  std::vector<unsigned char> hm(opt_mol_bytes() * nmol);
  if ((e = cudaMemcpyAsync(hm.data(), A.mol, hm.size(), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (xyz_out && (e = cudaMemcpyAsync(xyz_out, A.x, sizeof(double) * n3, cudaMemcpyDeviceToHost, st)) != cudaSuccess) ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cuda_fail(eng, e, "optimiser results");
  int worst = GFN1_OK;
  for (int m = 0; m < nmol; ++m) {
    const OptMol& mm = *(const OptMol*)(hm.data() + opt_mol_bytes() * m);
    if (energy) energy[m] = mm.error == kOk ? mm.energy : NAN;
    if (max_gradient) max_gradient[m] = mm.error == kOk ? mm.maxg : NAN;
    if (iterations) iterations[m] = mm.iterations;
    if (converged) converged[m] = mm.converged;
    if (status) status[m] = mm.error;
    worst = std::max(worst, mm.error);
  }
  if (rounds) *rounds = nround;
  if (worst != GFN1_OK) return fail(eng, worst, "geometry optimisation failed for at least one molecule (see status)");
  return GFN1_OK;
}

