// CPU FP64 oracle for the GFN1-xTB non-periodic SCC energy + analytic gradient.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain C++, the algorithm of
// gfn1-rs v0.5.1 (`run_electronic` src/electronic.rs:800 -> `analytic_gradient`
// src/gradient.rs:56) so that the CUDA engine's results can be checked against it.
// Nothing in the product library links, calls or loads this code; only tests/,
// __graft_entry__.smoke() and bench.py's CPU baseline do.
//
// Every function names the reference file:line it follows.  The data tables
// (parameters, STO-nG, D3 reference) are read from gfn1_tables.txt, generated from
// the reference tree by gfn1-rs_b200/data/gen_tables.py.
//
// Deliberate equivalences (not copies): the reference's faer eigensolver
// (`symmetric_eigen`, src/linalg.rs:153) is replaced by a Householder
// tridiagonalisation + implicit-shift QL solver (Golub & Van Loan, Matrix
// Computations, 4th ed., Alg. 8.3.1 / 8.3.3).  Eigenvector signs and rotations
// inside degenerate subspaces may differ; P, W, E and g do not depend on them.

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>
#include <atomic>
#include <thread>

namespace {

// ---------------------------------------------------------------- constants
// src/basis.rs:18 (legacy eV->Eh used for the parameter file)
const double EV_TO_HARTREE_MODEL = 1.0 / 27.21138505;
// src/constants.rs:26-27
const double KB_HARTREE_PER_K = 3.1668115634556e-6;
const double ANGSTROM_TO_BOHR = 1.8897261246257702;
// src/integrals.rs:17
const double PRIMITIVE_SCREEN_EPS = 1.0e-13;
// src/model.rs:24-32, src/dispersion.rs:30-32
const double CUTOFF_REPULSION = 25.0;
const double CUTOFF_CN = 30.0;
const double CUTOFF_INTEGRAL = 30.0;
const double D3_CN_CUTOFF = 25.0;
const double D3_PAIR_CUTOFF = 50.0;
const double D3_WF = 4.0;
const double PI = 3.14159265358979323846;

enum Status {
  OK = 0,
  E_IO = 1,
  E_PARSE = 2,
  E_INVALID_INPUT = 3,
  E_MISSING_ELEMENT = 4,
  E_MISSING_GLOBAL = 5,
  E_LINEAR_ALGEBRA = 6,
  E_SINGULAR_CELL = 7,
  E_SCC_NOT_CONVERGED = 8,
};

struct OracleError : std::runtime_error {
  int code;
  OracleError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

struct Vec3 {
  double x = 0, y = 0, z = 0;
  Vec3() {}
  Vec3(double a, double b, double c) : x(a), y(b), z(c) {}
  Vec3 operator+(const Vec3& o) const { return {x + o.x, y + o.y, z + o.z}; }
  Vec3 operator-(const Vec3& o) const { return {x - o.x, y - o.y, z - o.z}; }
  Vec3 operator*(double s) const { return {x * s, y * s, z * s}; }
  Vec3& operator+=(const Vec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
  Vec3& operator-=(const Vec3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  double norm2() const { return x * x + y * y + z * z; }
  double norm() const { return std::sqrt(norm2()); }
  double operator[](int k) const { return k == 0 ? x : (k == 1 ? y : z); }
};

// ---------------------------------------------------------------- tables
struct Tables {
  std::map<std::string, std::vector<double>> kv;
  bool loaded = false;
  const std::vector<double>& get(const std::string& k) const {
    auto it = kv.find(k);
    if (it == kv.end()) throw OracleError(E_MISSING_GLOBAL, "missing table entry `" + k + "`");
    return it->second;
  }
  bool has(const std::string& k) const { return kv.count(k) != 0; }
  double scalar(const std::string& k, double dflt) const {
    auto it = kv.find(k);
    return it == kv.end() ? dflt : it->second.at(0);
  }
};

Tables g_tables;

// C stdio on purpose: iostreams pull in locale state that clashes with a second
// libstdc++ already loaded into the host process.
void load_tables(const char* path) {
  FILE* fp = std::fopen(path, "rb");
  if (!fp) throw OracleError(E_IO, std::string("cannot open tables file ") + path);
  std::string text;
  char buf[1 << 16];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof buf, fp)) > 0) text.append(buf, got);
  std::fclose(fp);
  Tables t;
  size_t pos = 0;
  while (pos < text.size()) {
    size_t eol = text.find('\n', pos);
    if (eol == std::string::npos) eol = text.size();
    std::string line = text.substr(pos, eol - pos);
    pos = eol + 1;
    if (line.empty() || line[0] == '#') continue;
    const char* c = line.c_str();
    char* end = nullptr;
    while (*c == ' ') ++c;
    const char* ks = c;
    while (*c && *c != ' ') ++c;
    std::string key(ks, c - ks);
    long n = std::strtol(c, &end, 10);
    if (end == c || n < 0) throw OracleError(E_PARSE, "bad table line for `" + key + "`");
    c = end;
    std::vector<double> v((size_t)n);
    for (long i = 0; i < n; ++i) {
      v[i] = std::strtod(c, &end);
      if (end == c) throw OracleError(E_PARSE, "bad table value for `" + key + "`");
      c = end;
    }
    t.kv[key] = std::move(v);
  }
  t.loaded = true;
  g_tables = std::move(t);
}

// ---------------------------------------------------------------- parameters
// src/params.rs:119-162 (ShellParam, ElementParam), :361-376 (k_shell/pair_scaling)
struct ShellParam {
  int n, l;
  double level_ev, slater, poly_raw, lpar_raw;
};
struct ElementParam {
  int z = 0;
  std::vector<ShellParam> shells;
  double gam = 0, gam3_raw = 0, repa = 0, repb = 0;
  double lpar[3] = {0, 0, 0}, poly[3] = {0, 0, 0};
  bool present = false;
  double gam3_model() const { return 0.1 * gam3_raw; }  // src/params.rs:148-150
  // src/params.rs:152-161: hardness uses the LPAR of the first shell with that l
  double shell_hardness(int l) const {
    double lp = 0.0;
    for (auto& s : shells)
      if (s.l == l) { lp = s.lpar_raw; break; }
    return gam * (1.0 + 0.1 * lp);
  }
};

struct Params {
  ElementParam elem[87];
  double glob(const char* k, double dflt) const { return g_tables.scalar(std::string("glob.") + k, dflt); }
  double req(const char* k) const {
    std::string key = std::string("glob.") + k;
    if (!g_tables.has(key)) throw OracleError(E_MISSING_GLOBAL, std::string("missing required $globpar entry `") + k + "`");
    return g_tables.get(key)[0];
  }
  const ElementParam& element(int z) const {
    if (z < 1 || z > 86 || !elem[z].present)
      throw OracleError(E_MISSING_ELEMENT, "missing GFN1 parameter block for Z=" + std::to_string(z));
    return elem[z];
  }
  // src/params.rs:694-710
  static double default_pair_scaling(int za, int zb) {
    auto drow = [](int z) -> double {
      if (z >= 21 && z < 30) return 1.1;
      if (z >= 39 && z < 48) return 1.2;
      if (z >= 57 && z < 80) return 1.2;
      return -1.0;
    };
    double a = drow(za), b = drow(zb);
    if (a > 0 && b > 0) return 0.5 * (a + b);
    return 1.0;
  }
  double pair_scaling(int za, int zb) const {  // src/params.rs:361-367
    int a = std::min(za, zb), b = std::max(za, zb);
    std::string key = "pair." + std::to_string(a) + "." + std::to_string(b);
    if (g_tables.has(key)) return g_tables.get(key)[0];
    return default_pair_scaling(za, zb);
  }
  double k_shell(int l) const {  // src/params.rs:369-376
    if (l == 0) return glob("ks", 1.85);
    if (l == 1) return glob("kp", 2.25);
    return glob("kd", 2.00);
  }
};

Params g_params;

void build_params() {
  for (int z = 1; z <= 86; ++z) {
    std::string p = "elem." + std::to_string(z) + ".";
    if (!g_tables.has(p + "ao")) continue;
    ElementParam& e = g_params.elem[z];
    e.z = z;
    auto ao = g_tables.get(p + "ao");
    auto lev = g_tables.get(p + "lev");
    auto ex = g_tables.get(p + "exp");
    e.gam = g_tables.get(p + "gam")[0];
    e.gam3_raw = g_tables.get(p + "gam3")[0];
    e.repa = g_tables.get(p + "repa")[0];
    e.repb = g_tables.get(p + "repb")[0];
    const char* sfx[3] = {"s", "p", "d"};
    for (int l = 0; l < 3; ++l) {
      e.poly[l] = g_tables.get(p + "poly" + sfx[l])[0];
      e.lpar[l] = g_tables.get(p + "lpar" + sfx[l])[0];
    }
    for (size_t i = 0; i < ao.size() / 2; ++i) {
      ShellParam s;
      s.n = (int)ao[2 * i];
      s.l = (int)ao[2 * i + 1];
      s.level_ev = lev[i];
      s.slater = ex[i];
      s.poly_raw = s.l < 3 ? e.poly[s.l] : 0.0;
      s.lpar_raw = s.l < 3 ? e.lpar[s.l] : 0.0;
      e.shells.push_back(s);
    }
    e.present = true;
  }
}

// ---------------------------------------------------------------- data tables
// src/data_tables.rs:195-219
double atomic_radius_bohr(int z) {
  double v = g_tables.get("atomic_radius_ang").at(z);
  if (v <= 0) throw OracleError(E_INVALID_INPUT, "no xTB atomic radius for Z=" + std::to_string(z));
  return v * ANGSTROM_TO_BOHR;
}
double covalent_radius_d3_bohr(int z) {
  double v = g_tables.get("covrad_ang").at(z);
  if (v <= 0) throw OracleError(E_INVALID_INPUT, "no mctc covalent radius for Z=" + std::to_string(z));
  return (4.0 / 3.0) * v * ANGSTROM_TO_BOHR;
}
double pauling_en(int z) {  // src/data_tables.rs:176-193
  if (z > 86) throw OracleError(E_INVALID_INPUT, "no Pauling electronegativity for Z=" + std::to_string(z));
  return g_tables.get("pauling_en").at(z);
}
double reference_occupation(int z, int l) {  // src/basis.rs:296-309
  if (l > 2) return 0.0;
  return g_tables.get("refocc").at(3 * z + l);
}

// ---------------------------------------------------------------- STO-nG
// src/sto.rs:790-881 (slater_to_gauss), :891-897 (primitive normalisation)
struct Prim {
  double a, c;
};

std::vector<Prim> slater_to_gauss(int ng, int n, int l, double zeta) {
  if (ng < 1 || ng > 6) throw OracleError(E_INVALID_INPUT, "STO-nG size out of range");
  bool special = (n == 6 && ng == 6 && l <= 1);
  if ((n > 5 || n <= l) && !special) throw OracleError(E_INVALID_INPUT, "unsupported STO-nG shell");
  if (zeta <= 0) throw OracleError(E_INVALID_INPUT, "Slater exponent must be positive");
  std::vector<double> alpha(ng), coeff(ng);
  if (special) {
    auto& a = g_tables.get(l == 0 ? "sto.alpha6s" : "sto.alpha6p");
    auto& c = g_tables.get(l == 0 ? "sto.coeff6s" : "sto.coeff6p");
    for (int i = 0; i < 6; ++i) { alpha[i] = a[i]; coeff[i] = c[i]; }
  } else {
    int ityp1 = (l == 0) ? n : (l == 1 ? 4 + n : (l == 2 ? 7 + n : (l == 3 ? 9 + n : 10 + n)));
    if (ityp1 < 1 || ityp1 > 15) throw OracleError(E_INVALID_INPUT, "no STO table entry");
    auto& a = g_tables.get("sto.alpha." + std::to_string(ng));
    auto& c = g_tables.get("sto.coeff." + std::to_string(ng));
    for (int i = 0; i < ng; ++i) {
      alpha[i] = a[(ityp1 - 1) * ng + i];
      coeff[i] = c[(ityp1 - 1) * ng + i];
    }
  }
  static const double dfact[8] = {1.0, 1.0, 3.0, 15.0, 105.0, 945.0, 10395.0, 135135.0};
  const double top = 2.0 / PI;
  std::vector<Prim> out(ng);
  double z2 = zeta * zeta;
  for (int i = 0; i < ng; ++i) {
    double al = alpha[i] * z2;
    double c = coeff[i] * std::pow(top * al, 0.75) * std::pow(std::sqrt(4.0 * al), l) / std::sqrt(dfact[l]);
    out[i] = {al, c};
  }
  return out;
}

// src/basis.rs:251-279
int gfn1_number_of_primitives(int z, int n, int l) {
  int np;
  if (z <= 2) np = (l == 0) ? (n == 1 ? 4 : 3) : (l == 1 ? 3 : 4);
  else np = (l <= 1) ? 6 : 4;
  return np;
}

// src/basis.rs:281-293 (kcn shift) and :295-302 (kind)
int gfn1_kind(int z) {
  if (z == 1 || z == 2 || (z >= 6 && z <= 10) || (z >= 14 && z <= 18) || (z >= 32 && z <= 36) ||
      (z >= 50 && z <= 54) || (z >= 82 && z <= 86))
    return 1;
  if (z >= 21 && z <= 24) return 2;
  return 0;
}
double gfn1_kcn_shift(double level_ev, int l, int z) {
  int kind = gfn1_kind(z);
  if (kind == 0) return 0.0;
  double f = 0.0;
  if (l == 0) f = g_params.glob("cns", 0.6);
  else if (l == 1) f = g_params.glob("cnp", -0.3);
  else if (l == 2) f = (kind == 1) ? g_params.glob("cnd1", -0.5) : g_params.glob("cnd2", 0.5);
  return -level_ev * EV_TO_HARTREE_MODEL * f * 0.01;
}

// src/basis.rs:318-344
void orthogonalize_same_center(const std::vector<Prim>& ref, std::vector<Prim>& shell) {
  double ov = 0.0;
  for (auto& a : ref)
    for (auto& b : shell) {
      double eab = a.a + b.a;
      double k = std::pow(std::sqrt(PI / eab), 3);
      ov += a.c * b.c * k;
    }
  for (auto& a : ref) shell.push_back({a.a, -ov * a.c});
  double nrm = 0.0;
  for (auto& a : shell)
    for (auto& b : shell) {
      double eab = a.a + b.a;
      nrm += a.c * b.c * std::pow(std::sqrt(PI / eab), 3);
    }
  double sc = 1.0 / std::sqrt(nrm);
  for (auto& p : shell) p.c *= sc;
}

// ---------------------------------------------------------------- basis
struct CartComp {
  int px, py, pz;
  double coef;
};
struct AO {
  int atom, shell, l;
  std::vector<CartComp> comps;
  std::vector<Prim> prims;
};
struct Shell {
  int atom, z, l, first_ao, nao;
  bool is_valence;
  double hdiag_ha, kcn, poly, ref_occ, hardness, gam3;
};
struct Basis {
  std::vector<AO> aos;
  std::vector<Shell> shells;
  std::vector<int> atom_shell_first, atom_shell_count, atom_ao_first, atom_ao_count;
  double total_ref = 0.0;
};

// src/basis.rs:382-441
std::vector<std::vector<CartComp>> spherical_components(int l) {
  const double s3 = std::sqrt(3.0), s32 = s3 / 2.0;
  if (l == 0) return {{{0, 0, 0, 1.0}}};
  if (l == 1) return {{{1, 0, 0, 1.0}}, {{0, 1, 0, 1.0}}, {{0, 0, 1, 1.0}}};
  if (l == 2)
    return {{{2, 0, 0, s32}, {0, 2, 0, -s32}},
            {{2, 0, 0, 0.5}, {0, 2, 0, 0.5}, {0, 0, 2, -1.0}},
            {{1, 1, 0, s3}},
            {{1, 0, 1, s3}},
            {{0, 1, 1, s3}}};
  throw OracleError(E_INVALID_INPUT, "integral engine implements s, p, d shells only");
}

// src/basis.rs:121-233
Basis build_basis(const std::vector<int>& zs) {
  Basis b;
  int nat = (int)zs.size();
  b.atom_shell_first.resize(nat);
  b.atom_shell_count.resize(nat);
  b.atom_ao_first.resize(nat);
  b.atom_ao_count.resize(nat);
  for (int a = 0; a < nat; ++a) {
    const ElementParam& e = g_params.element(zs[a]);
    b.atom_shell_first[a] = (int)b.shells.size();
    b.atom_ao_first[a] = (int)b.aos.size();
    bool seen[5] = {false, false, false, false, false};
    std::vector<Prim> same_l_ref[5];
    bool has_ref[5] = {false, false, false, false, false};
    for (auto& sp : e.shells) {
      int l = sp.l;
      bool valence = !seen[l];
      seen[l] = true;
      auto comps = spherical_components(l);
      int np = gfn1_number_of_primitives(zs[a], sp.n, l);
      auto prims = slater_to_gauss(np, sp.n, l, sp.slater);
      if (has_ref[l]) orthogonalize_same_center(same_l_ref[l], prims);
      else { same_l_ref[l] = prims; has_ref[l] = true; }
      double shell_ref = valence ? reference_occupation(zs[a], l) : 0.0;
      Shell sh;
      sh.atom = a;
      sh.z = zs[a];
      sh.l = l;
      sh.first_ao = (int)b.aos.size();
      sh.nao = (int)comps.size();
      sh.is_valence = valence;
      sh.hdiag_ha = sp.level_ev * EV_TO_HARTREE_MODEL;
      sh.kcn = gfn1_kcn_shift(sp.level_ev, l, zs[a]);
      sh.poly = sp.poly_raw * 0.01;
      sh.ref_occ = shell_ref;
      sh.hardness = e.shell_hardness(l);  // src/coulomb.rs:58-62
      sh.gam3 = e.gam3_model();
      int shell_index = (int)b.shells.size();
      for (auto& c : comps) {
        AO ao;
        ao.atom = a;
        ao.shell = shell_index;
        ao.l = l;
        ao.comps = c;
        ao.prims = prims;
        b.aos.push_back(ao);
      }
      b.shells.push_back(sh);
      b.total_ref += shell_ref;
    }
    b.atom_shell_count[a] = (int)b.shells.size() - b.atom_shell_first[a];
    b.atom_ao_count[a] = (int)b.aos.size() - b.atom_ao_first[a];
  }
  return b;
}

// ---------------------------------------------------------------- overlap integrals
// src/integrals.rs:895-920
double moment_1d(int ia, int jb, double alpha, double beta, double a, double b, double p, const double* g) {
  static const double binom[8][8] = {{1, 0, 0, 0, 0, 0, 0, 0},  {1, 1, 0, 0, 0, 0, 0, 0},
                                     {1, 2, 1, 0, 0, 0, 0, 0},  {1, 3, 3, 1, 0, 0, 0, 0},
                                     {1, 4, 6, 4, 1, 0, 0, 0},  {1, 5, 10, 10, 5, 1, 0, 0},
                                     {1, 6, 15, 20, 15, 6, 1, 0}, {1, 7, 21, 35, 35, 21, 7, 1}};
  double pc = (alpha * a + beta * b) / p;
  double pa = pc - a, pb = pc - b;
  double sum = 0.0;
  for (int u = 0; u <= ia; ++u) {
    double ca = binom[ia][u] * std::pow(pa, ia - u);
    for (int v = 0; v <= jb; ++v) {
      double cb = binom[jb][v] * std::pow(pb, jb - v);
      int uv = u + v;
      if (uv % 2 == 0) sum += ca * cb * g[uv / 2];
    }
  }
  return sum;
}

double comp_abs_sum(const AO& a) {
  double s = 0;
  for (auto& c : a.comps) s += std::fabs(c.coef);
  return s;
}

// src/integrals.rs:30-45
double primitive_pair_bound(double pref, double cscale, double alpha, double beta, double r, double r2, int order) {
  double p = alpha + beta;
  double kab = std::exp(-alpha * beta / p * r2);
  double spread = std::sqrt(1.0 / p);
  double gpref = (PI / p) * std::sqrt(PI / p);
  double poly = std::pow(1.0 + r + spread, order);
  return std::fabs(pref) * cscale * kab * gpref * poly;
}

// src/integrals.rs:290-360 restricted to the overlap (index 0 of the 10 moments)
double contracted_overlap(const AO& a, const AO& b, const Vec3& ca, const Vec3& cb) {
  Vec3 d = ca - cb;
  double r2 = d.norm2(), r = std::sqrt(r2);
  double cscale = comp_abs_sum(a) * comp_abs_sum(b);
  int order = a.l + b.l + 2;
  double s = 0.0;
  for (auto& pa : a.prims)
    for (auto& pb : b.prims) {
      double pref = pa.c * pb.c;
      double al = pa.a, be = pb.a, p = al + be;
      if (primitive_pair_bound(pref, cscale, al, be, r, r2, order) < PRIMITIVE_SCREEN_EPS) continue;
      double kab = std::exp(-al * be / p * r2);
      double g[7];
      g[0] = std::sqrt(PI / p);
      for (int m = 1; m <= 6; ++m) g[m] = g[m - 1] * (m - 0.5) / p;
      for (auto& x : a.comps)
        for (auto& y : b.comps) {
          double cf = pref * x.coef * y.coef * kab;
          double sx = moment_1d(x.px, y.px, al, be, ca.x, cb.x, p, g);
          double sy = moment_1d(x.py, y.py, al, be, ca.y, cb.y, p, g);
          double sz = moment_1d(x.pz, y.pz, al, be, ca.z, cb.z, p, g);
          s += cf * sx * sy * sz;
        }
    }
  return s;
}

// src/integrals.rs:481-537 + :782-868 restricted to the overlap: returns S and
// the bra/ket centre derivatives of S.
void contracted_overlap_deriv(const AO& a, const AO& b, const Vec3& ca, const Vec3& cb, double& s, Vec3& dbra,
                              Vec3& dket) {
  Vec3 d = ca - cb;
  double r2 = d.norm2(), r = std::sqrt(r2);
  double cscale = comp_abs_sum(a) * comp_abs_sum(b);
  int order = a.l + b.l + 3;
  s = 0.0;
  dbra = Vec3();
  dket = Vec3();
  for (auto& pa : a.prims)
    for (auto& pb : b.prims) {
      double pref = pa.c * pb.c;
      double al = pa.a, be = pb.a, p = al + be;
      if (primitive_pair_bound(pref, cscale, al, be, r, r2, order) < PRIMITIVE_SCREEN_EPS) continue;
      double kab = std::exp(-al * be / p * r2);
      double g[8];
      g[0] = std::sqrt(PI / p);
      for (int m = 1; m <= 7; ++m) g[m] = g[m - 1] * (m - 0.5) / p;
      for (auto& x : a.comps)
        for (auto& y : b.comps) {
          double cf = pref * x.coef * y.coef * kab;
          int ia[3] = {x.px, x.py, x.pz}, jb[3] = {y.px, y.py, y.pz};
          double cA[3] = {ca.x, ca.y, ca.z}, cB[3] = {cb.x, cb.y, cb.z};
          double m0[3], mAp[3], mAm[3], mBp[3], mBm[3];
          for (int k = 0; k < 3; ++k) {
            m0[k] = moment_1d(ia[k], jb[k], al, be, cA[k], cB[k], p, g);
            mAp[k] = moment_1d(ia[k] + 1, jb[k], al, be, cA[k], cB[k], p, g);
            mAm[k] = ia[k] > 0 ? moment_1d(ia[k] - 1, jb[k], al, be, cA[k], cB[k], p, g) : 0.0;
            mBp[k] = moment_1d(ia[k], jb[k] + 1, al, be, cA[k], cB[k], p, g);
            mBm[k] = jb[k] > 0 ? moment_1d(ia[k], jb[k] - 1, al, be, cA[k], cB[k], p, g) : 0.0;
          }
          s += cf * m0[0] * m0[1] * m0[2];
          double da[3], db[3];
          for (int k = 0; k < 3; ++k) {
            double o1 = m0[(k + 1) % 3] * m0[(k + 2) % 3];
            da[k] = (2.0 * al * mAp[k] - ia[k] * mAm[k]) * o1;
            db[k] = (2.0 * be * mBp[k] - jb[k] * mBm[k]) * o1;
          }
          dbra += Vec3(da[0], da[1], da[2]) * cf;
          dket += Vec3(db[0], db[1], db[2]) * cf;
        }
    }
}

// ---------------------------------------------------------------- dense helpers
struct Mat {
  int n = 0, m = 0;
  std::vector<double> a;
  Mat() {}
  Mat(int r, int c) : n(r), m(c), a((size_t)r * c, 0.0) {}
  double& operator()(int i, int j) { return a[(size_t)i * m + j]; }
  double operator()(int i, int j) const { return a[(size_t)i * m + j]; }
};

Mat matmul(const Mat& A, const Mat& B) {
  Mat C(A.n, B.m);
  for (int i = 0; i < A.n; ++i)
    for (int k = 0; k < A.m; ++k) {
      double aik = A(i, k);
      if (aik == 0.0) continue;
      const double* brow = &B.a[(size_t)k * B.m];
      double* crow = &C.a[(size_t)i * C.m];
      for (int j = 0; j < B.m; ++j) crow[j] += aik * brow[j];
    }
  return C;
}
Mat transpose(const Mat& A) {
  Mat T(A.m, A.n);
  for (int i = 0; i < A.n; ++i)
    for (int j = 0; j < A.m; ++j) T(j, i) = A(i, j);
  return T;
}

// Symmetric eigensolver: Householder reduction to tridiagonal form followed by
// the implicit-shift QL iteration with accumulated transformations (Golub & Van
// Loan Alg. 8.3.1 and the QL variant of Alg. 8.3.3).  Eigenvalues ascending,
// eigenvectors in the columns of V.  Replaces faer's self_adjoint_eigen used by
// src/linalg.rs:153-191.
void sym_eig(const Mat& Ain, std::vector<double>& w, Mat& V) {
  int n = Ain.n;
  w.assign(n, 0.0);
  V = Mat(n, n);
  for (int i = 0; i < n; ++i) V(i, i) = 1.0;
  if (n == 1) {
    w[0] = Ain(0, 0);
    return;
  }
  Mat A = Ain;
  std::vector<double> e(n, 0.0), v(n), p(n), wv(n);
  // Householder reduction A = Q T Q^T (Golub & Van Loan Alg. 8.3.1); Q kept in V
  for (int k = 0; k < n - 2; ++k) {
    int m = n - k - 1;  // length of the column below the diagonal
    double xn2 = 0.0;
    for (int i = 0; i < m; ++i) {
      v[i] = A(k + 1 + i, k);
      xn2 += v[i] * v[i];
    }
    double tail = xn2 - v[0] * v[0];
    if (tail == 0.0) continue;  // already tridiagonal in this column
    double xn = std::sqrt(xn2);
    double alpha = v[0] >= 0.0 ? -xn : xn;
    v[0] -= alpha;
    double vn2 = v[0] * v[0] + tail;
    double beta = 2.0 / vn2;
    // p = beta * B v, B = A[k+1:, k+1:]
    for (int i = 0; i < m; ++i) {
      double s = 0.0;
      for (int j = 0; j < m; ++j) s += A(k + 1 + i, k + 1 + j) * v[j];
      p[i] = beta * s;
    }
    double pv = 0.0;
    for (int i = 0; i < m; ++i) pv += p[i] * v[i];
    double K = 0.5 * beta * pv;
    for (int i = 0; i < m; ++i) wv[i] = p[i] - K * v[i];
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) A(k + 1 + i, k + 1 + j) -= v[i] * wv[j] + wv[i] * v[j];
    A(k + 1, k) = A(k, k + 1) = alpha;
    for (int i = 1; i < m; ++i) A(k + 1 + i, k) = A(k, k + 1 + i) = 0.0;
    // V := V H, H = I - beta v v^T on indices k+1..n-1
    for (int r = 0; r < n; ++r) {
      double t = 0.0;
      for (int i = 0; i < m; ++i) t += V(r, k + 1 + i) * v[i];
      t *= beta;
      for (int i = 0; i < m; ++i) V(r, k + 1 + i) -= t * v[i];
    }
  }
  for (int i = 0; i < n; ++i) w[i] = A(i, i);
  for (int i = 0; i < n - 1; ++i) e[i] = A(i + 1, i);
  e[n - 1] = 0.0;
  // implicit-shift QL on the tridiagonal (d = w, e[i] couples i and i+1)
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    int m;
    do {
      for (m = l; m < n - 1; ++m) {
        double dd = std::fabs(w[m]) + std::fabs(w[m + 1]);
        if (std::fabs(e[m]) <= 1e-300 || std::fabs(e[m]) <= std::numeric_limits<double>::epsilon() * dd) break;
      }
      if (m != l) {
        if (iter++ == 200) throw OracleError(E_LINEAR_ALGEBRA, "QL iteration did not converge");
        double g = (w[l + 1] - w[l]) / (2.0 * e[l]);
        double r = std::hypot(g, 1.0);
        g = w[m] - w[l] + e[l] / (g + (g >= 0 ? std::fabs(r) : -std::fabs(r)));
        double s = 1.0, c = 1.0, p = 0.0;
        int i;
        for (i = m - 1; i >= l; --i) {
          double f = s * e[i];
          double b = c * e[i];
          r = std::hypot(f, g);
          e[i + 1] = r;
          if (r == 0.0) {
            w[i + 1] -= p;
            e[m] = 0.0;
            break;
          }
          s = f / r;
          c = g / r;
          g = w[i + 1] - p;
          r = (w[i] - g) * s + 2.0 * c * b;
          p = s * r;
          w[i + 1] = g + p;
          g = c * r - b;
          for (int k = 0; k < n; ++k) {
            double t = V(k, i + 1);
            V(k, i + 1) = s * V(k, i) + c * t;
            V(k, i) = c * V(k, i) - s * t;
          }
        }
        if (r == 0.0 && i >= l) continue;
        w[l] -= p;
        e[l] = g;
        e[m] = 0.0;
      }
    } while (m != l);
  }
  // sort ascending
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return w[a] < w[b]; });
  std::vector<double> w2(n);
  Mat V2(n, n);
  for (int j = 0; j < n; ++j) {
    w2[j] = w[idx[j]];
    for (int i = 0; i < n; ++i) V2(i, j) = V(i, idx[j]);
  }
  w = w2;
  V = V2;
}

// ---------------------------------------------------------------- system / pairs
struct System {
  std::vector<int> z;
  std::vector<Vec3> pos;
  double charge = 0.0;
  int nat() const { return (int)z.size(); }
};

struct Pair {
  int i, j;
  Vec3 dr;  // pos[j] - pos[i]
  double r2, r;
};

// src/pairlist.rs:164-235 for a molecule: i<j, DIST_EPS^2 < r2 <= cutoff^2,
// sorted by (r2, i, j)
std::vector<Pair> unique_pairs(const System& s, double cutoff, bool sorted) {
  std::vector<Pair> out;
  double c2 = cutoff * cutoff;
  for (int i = 0; i < s.nat(); ++i)
    for (int j = i + 1; j < s.nat(); ++j) {
      Vec3 dr = s.pos[j] - s.pos[i];
      double r2 = dr.norm2();
      if (r2 <= 1e-24 || r2 > c2) continue;
      out.push_back({i, j, dr, r2, std::sqrt(r2)});
    }
  if (sorted)
    std::stable_sort(out.begin(), out.end(), [](const Pair& a, const Pair& b) {
      if (a.r2 != b.r2) return a.r2 < b.r2;
      if (a.i != b.i) return a.i < b.i;
      return a.j < b.j;
    });
  return out;
}

// ---------------------------------------------------------------- coordination
// src/coordination.rs:51-106
struct CnPair {
  int i, j;
  Vec3 rij;  // pos[i] - pos[j]
  double dcn_dr;
};
void exp_count(double kcn, double r, double rc, double& value, double& dvalue) {
  double raw = -kcn * (rc / r - 1.0);
  double arg = std::min(80.0, std::max(-80.0, raw));
  double e = std::exp(arg);
  value = 1.0 / (1.0 + e);
  dvalue = (raw < -80.0 || raw > 80.0) ? 0.0 : -kcn * rc * e / (r * r * (1.0 + e) * (1.0 + e));
}
std::vector<double> coordination(const System& s, double cutoff, std::vector<CnPair>* pairs) {
  std::vector<double> rad(s.nat());
  for (int a = 0; a < s.nat(); ++a) rad[a] = covalent_radius_d3_bohr(s.z[a]);
  std::vector<double> cn(s.nat(), 0.0);
  for (auto& p : unique_pairs(s, cutoff, false)) {
    double rc = rad[p.i] + rad[p.j];
    if (rc <= 1e-12) continue;
    double v, dv;
    exp_count(16.0, p.r, rc, v, dv);
    cn[p.i] += v;
    cn[p.j] += v;
    if (pairs) pairs->push_back({p.i, p.j, p.dr * -1.0, dv});
  }
  return cn;
}

// ---------------------------------------------------------------- H0
// src/hamiltonian.rs:136-165
double shell_polynomial(const Shell& a, const Shell& b, double rr) {
  return (1.0 + a.poly * rr) * (1.0 + b.poly * rr);
}
double kshell_pair(int li, int lj) {
  if ((li == 0 && lj == 1) || (li == 1 && lj == 0)) return g_params.glob("ksp", 2.08);
  return 0.5 * (g_params.k_shell(li) + g_params.k_shell(lj));
}
double hscale(const Shell& a, const Shell& b) {
  double kdiff = g_params.glob("kdiff", 2.85);
  if (a.is_valence && b.is_valence) {
    double den = std::pow(pauling_en(a.z) - pauling_en(b.z), 2);
    double ens = g_params.glob("enscale", -0.7) * 0.01;
    return g_params.pair_scaling(a.z, b.z) * kshell_pair(a.l, b.l) * (1.0 + ens * den);
  } else if (a.is_valence) {
    return 0.5 * (kshell_pair(a.l, a.l) + kdiff);
  } else if (b.is_valence) {
    return 0.5 * (kshell_pair(b.l, b.l) + kdiff);
  }
  return kdiff;
}

// ---------------------------------------------------------------- options / results
struct Options {
  int max_scc = 250;
  double energy_tolerance = 1e-6;
  double charge_tolerance = 2e-5;
  double mixing = 0.4;
  int scc_broyden = 1;
  int scc_broyden_size = 250;
  double electronic_temperature = 300.0;
  int enable_dispersion = 1;
  double level_shift = 0.0;
  double eigen_tolerance = 1e-12;
  int spin_multiplicity = 0;  // 0: None
};

// ---------------------------------------------------------------- Broyden
// src/electronic.rs:3203-3316, :3759-3806
double dotv(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0;
  for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}
std::vector<double> damped_step(const std::vector<double>& q, const std::vector<double>& r, double mix) {
  std::vector<double> o(q.size());
  for (size_t i = 0; i < q.size(); ++i) o[i] = q[i] + mix * r[i];
  return o;
}
bool solve_linear(std::vector<std::vector<double>> a, std::vector<double>& b) {
  int n = (int)b.size();
  for (int col = 0; col < n; ++col) {
    int piv = col;
    double pabs = std::fabs(a[col][col]);
    for (int row = col + 1; row < n; ++row)
      if (std::fabs(a[row][col]) > pabs) { piv = row; pabs = std::fabs(a[row][col]); }
    if (pabs < 1e-18) return false;
    if (piv != col) { std::swap(a[piv], a[col]); std::swap(b[piv], b[col]); }
    double dg = a[col][col];
    for (int j = col; j < n; ++j) a[col][j] /= dg;
    b[col] /= dg;
    for (int row = 0; row < n; ++row) {
      if (row == col) continue;
      double f = a[row][col];
      if (f == 0.0) continue;
      for (int j = col; j < n; ++j) a[row][j] -= f * a[col][j];
      b[row] -= f * b[col];
    }
  }
  return true;
}
bool trusted(const std::vector<double>& v) {
  for (double x : v)
    if (!std::isfinite(x) || std::fabs(x) >= 10.0) return false;
  return true;
}

struct Broyden {
  int memory;
  double damp;
  int iter = 0;
  std::vector<std::vector<double>> df, u;
  std::vector<double> omega, qlast, dqlast;
  Broyden(int ndim, int mem, double d) : memory(mem), damp(d), df(mem, std::vector<double>(ndim, 0.0)),
                                         u(mem, std::vector<double>(ndim, 0.0)), omega(mem, 0.0),
                                         qlast(ndim, 0.0), dqlast(ndim, 0.0) {}
  bool next(const std::vector<double>& q, const std::vector<double>& dq, std::vector<double>& out) {
    iter += 1;
    if (iter == 1) {
      dqlast = dq;
      qlast = q;
      out = damped_step(q, dq, damp);
      return true;
    }
    int itn = iter - 1;
    int it1 = (itn - 1) % memory;
    const double omega0 = 0.01, minw = 1.0, maxw = 100000.0, wfac = 0.01;
    double dqn = std::sqrt(dotv(dq, dq));
    omega[it1] = dqn > wfac / maxw ? wfac / dqn : maxw;
    if (omega[it1] < minw) omega[it1] = minw;
    std::vector<double> dfc(dq.size());
    for (size_t i = 0; i < dq.size(); ++i) dfc[i] = dq[i] - dqlast[i];
    double inv = 1.0 / std::max(std::sqrt(dotv(dfc, dfc)), std::numeric_limits<double>::epsilon());
    for (auto& v : dfc) v *= inv;
    df[it1] = dfc;
    for (size_t i = 0; i < dq.size(); ++i) u[it1][i] = damp * df[it1][i] + inv * (q[i] - qlast[i]);
    int start = itn > memory ? itn - memory + 1 : 1;
    std::vector<int> active;
    for (int j = start; j <= itn; ++j) active.push_back((j - 1) % memory);
    int m = (int)active.size();
    std::vector<std::vector<double>> beta(m, std::vector<double>(m, 0.0));
    std::vector<double> c(m, 0.0);
    for (int r = 0; r < m; ++r) {
      int i = active[r];
      c[r] = omega[i] * dotv(df[i], dq);
      for (int cc = 0; cc < m; ++cc) {
        int j = active[cc];
        beta[r][cc] = omega[i] * omega[j] * dotv(df[i], df[j]);
      }
      beta[r][r] += omega0 * omega0;
    }
    if (!solve_linear(beta, c)) return false;
    dqlast = dq;
    qlast = q;
    out = damped_step(q, dq, damp);
    for (int r = 0; r < m; ++r) {
      int i = active[r];
      double sc = omega[i] * c[r];
      for (size_t k = 0; k < out.size(); ++k) out[k] -= sc * u[i][k];
    }
    return true;
  }
};

// ---------------------------------------------------------------- occupations
// src/electronic.rs:3853-3921 (cap = 2, both spins in one orbital) and the
// one-spin channels of :3958-4045 (cap = 1): occupation cap / (1 + e^x),
// aufbau fills of at most cap, entropy cap kT [n ln n + (1-n) ln(1-n)] with
// n = f / cap.
struct Occ {
  std::vector<double> f;
  double mu = 0, ts = 0;
};
double fermi_occ(double eps, double mu, double kt, double cap = 2.0) {
  double x = std::min(80.0, std::max(-80.0, (eps - mu) / kt));
  return cap / (1.0 + std::exp(x));
}
Occ occupations(const std::vector<double>& eps, double nelec, double kt, double cap = 2.0) {
  Occ o;
  int n = (int)eps.size();
  o.f.assign(n, 0.0);
  if (kt <= 0.0) {  // aufbau, src/electronic.rs:3830-3851
    double rem = std::max(0.0, nelec);
    for (int i = 0; i < n; ++i) {
      double fill = std::min(rem, cap);
      o.f[i] = fill;
      rem -= fill;
      if (rem <= 0.0) break;
    }
    int homo = 0;
    for (int i = n - 1; i >= 0; --i)
      if (o.f[i] > 1e-12) { homo = i; break; }
    o.mu = n ? eps[homo] : 0.0;
    return o;
  }
  if (nelec <= 0.0) { o.mu = n ? eps[0] : 0.0; return o; }
  if (nelec >= cap * n) { o.f.assign(n, cap); o.mu = n ? eps[n - 1] : 0.0; return o; }
  double mn = *std::min_element(eps.begin(), eps.end());
  double mx = *std::max_element(eps.begin(), eps.end());
  double lo = mn - 100.0 * kt - 10.0, hi = mx + 100.0 * kt + 10.0;
  for (int it = 0; it < 200; ++it) {
    double mu = 0.5 * (lo + hi);
    double sum = 0.0;
    for (double e : eps) sum += fermi_occ(e, mu, kt, cap);
    double nlo = lo, nhi = hi;
    if (sum < nelec) nlo = mu; else nhi = mu;
    if (nlo == lo && nhi == hi) break;
    lo = nlo;
    hi = nhi;
  }
  o.mu = 0.5 * (lo + hi);
  o.ts = 0.0;
  for (int i = 0; i < n; ++i) {
    o.f[i] = fermi_occ(eps[i], o.mu, kt, cap);
    double nn = std::min(1.0 - 1e-16, std::max(1e-16, o.f[i] / cap));
    o.ts += cap * kt * (nn * std::log(nn) + (1.0 - nn) * std::log(1.0 - nn));
  }
  return o;
}

// src/electronic.rs:545-598: alpha and beta electron counts of a requested
// spin multiplicity (0 = none), with the reference's checks.
struct SpinChannels {
  bool on = false;
  double alpha = 0, beta = 0;
};
SpinChannels resolve_spin_channels(double nelec, int mult, int norb) {
  SpinChannels c;
  if (mult == 0) return c;
  if (mult < 1) throw OracleError(E_INVALID_INPUT, "spin multiplicity must be at least 1");
  const double rounded = std::round(nelec);
  if (std::fabs(nelec - rounded) > 1e-8)
    throw OracleError(E_INVALID_INPUT, "spin multiplicity requires an integer electron count");
  const long long ne = (long long)rounded, unpaired = mult - 1;
  if (unpaired > ne) throw OracleError(E_INVALID_INPUT, "spin multiplicity needs more unpaired electrons than the system has");
  if ((ne - unpaired) % 2 != 0) throw OracleError(E_INVALID_INPUT, "spin multiplicity is incompatible with the electron count");
  const long long a = (ne + unpaired) / 2, b = (ne - unpaired) / 2;
  if (a > norb || b > norb) throw OracleError(E_INVALID_INPUT, "spin multiplicity needs more orbitals than the basis has");
  c.on = true;
  c.alpha = (double)a;
  c.beta = (double)b;
  return c;
}

// src/electronic.rs:3930-3956: each spin channel filled on its own.
Occ spin_constrained_occupations(const std::vector<double>& eps, const SpinChannels& c, double kt) {
  Occ a = occupations(eps, c.alpha, kt, 1.0), b = occupations(eps, c.beta, kt, 1.0);
  Occ o;
  o.f.resize(eps.size());
  for (size_t i = 0; i < eps.size(); ++i) o.f[i] = a.f[i] + b.f[i];
  o.mu = 0.5 * (a.mu + b.mu);
  o.ts = a.ts + b.ts;
  return o;
}

// ---------------------------------------------------------------- electrostatics
// src/coulomb.rs:82-107, :140-193
Mat coulomb_matrix(const System& s, const Basis& b) {
  int nsh = (int)b.shells.size();
  Mat A(nsh, nsh);
  for (int i = 0; i < nsh; ++i) {
    int ai = b.shells[i].atom;
    for (int j = 0; j <= i; ++j) {
      int aj = b.shells[j].atom;
      double g = 2.0 / (1.0 / b.shells[i].hardness + 1.0 / b.shells[j].hardness);
      double v;
      if (ai == aj) v = g;
      else {
        double r = (s.pos[aj] - s.pos[ai]).norm();
        v = 1.0 / std::sqrt(r * r + 1.0 / (g * g));
      }
      A(i, j) = v;
      A(j, i) = v;
    }
  }
  return A;
}
struct Coul {
  double e2 = 0, e3 = 0;
  std::vector<double> pot, qat;
};
Coul coulomb(const Basis& b, const Mat& A, const std::vector<double>& q, int nat) {
  int nsh = (int)q.size();
  Coul c;
  c.pot.assign(nsh, 0.0);
  for (int i = 0; i < nsh; ++i) {
    double s = 0;
    for (int j = 0; j < nsh; ++j) s += A(i, j) * q[j];
    c.pot[i] = s;
  }
  for (int i = 0; i < nsh; ++i) c.e2 += q[i] * c.pot[i];
  c.e2 *= 0.5;
  c.qat.assign(nat, 0.0);
  for (int i = 0; i < nsh; ++i) c.qat[b.shells[i].atom] += q[i];
  for (int a = 0; a < nat; ++a) {
    if (b.atom_shell_count[a] == 0) continue;
    int off = b.atom_shell_first[a];
    double g3 = b.shells[off].gam3;
    double qa = c.qat[a];
    c.e3 += qa * qa * qa * g3 / 3.0;
    double pot = qa * qa * g3;
    for (int k = 0; k < b.atom_shell_count[a]; ++k) c.pot[off + k] += pot;
  }
  return c;
}

// ---------------------------------------------------------------- repulsion
// src/repulsion.rs:39-59, :139-159
double repulsion(const System& s, std::vector<Vec3>* grad) {
  double e = 0.0;
  double kexp = g_params.glob("kexp", 1.5);
  double kexpl = g_params.glob("kexplight", kexp);
  for (auto& p : unique_pairs(s, CUTOFF_REPULSION, false)) {
    const ElementParam& a = g_params.element(s.z[p.i]);
    const ElementParam& b = g_params.element(s.z[p.j]);
    double alpha = std::sqrt(a.repa * b.repa);
    double zeff = a.repb * b.repb;
    double k = (s.z[p.i] <= 2 && s.z[p.j] <= 2) ? kexpl : kexp;
    double rk = std::pow(p.r, k);
    double en = zeff * std::exp(-alpha * rk) / p.r;
    double pref = (alpha * rk * k + 1.0) * en / (p.r * p.r);
    e += en;
    if (grad) {
      Vec3 dg = p.dr * pref;
      (*grad)[p.i] += dg;
      (*grad)[p.j] -= dg;
    }
  }
  return e;
}

// ---------------------------------------------------------------- D3(BJ)
// src/dispersion.rs:1232-1360 (two-body; GFN1 has s9 = 0 so ATM is skipped),
// :1629-1692 (reference weights), :1753-1787 (atomic C6), :3136-3170 (lookups)
int d3_nref(int z) {
  int n = (int)g_tables.get("d3.nref").at(z - 1);
  if (n <= 0) throw OracleError(E_INVALID_INPUT, "no D3 reference count for Z=" + std::to_string(z));
  return n;
}
double d3_r4r2(int z) {
  double raw = g_tables.get("d3.r4r2").at(z - 1);
  double v = std::sqrt(0.5 * raw * std::sqrt((double)z));
  return v;
}
double d3_c6ref(int zi, int iref, int zj, int jref) {
  int a, b, ia, ib;
  if (zi > zj) { a = zi; b = zj; ia = iref; ib = jref; }
  else { a = zj; b = zi; ia = jref; ib = iref; }
  auto& blk = g_tables.get("d3.c6." + std::to_string(a) + "." + std::to_string(b));
  return blk.at(ia * d3_nref(b) + ib);
}
double dispersion(const System& s, std::vector<Vec3>* grad) {
  double s6 = g_params.glob("s6", 1.0);
  double s8 = g_params.req("s8");
  double s9 = g_params.req("s9");
  double a1 = g_params.req("a1");
  double a2 = g_params.req("a2");
  if (std::fabs(s9) > 1e-15) throw OracleError(E_INVALID_INPUT, "D3 ATM term (s9 != 0) is not supported");
  int nat = s.nat();
  std::vector<CnPair> cnp;
  std::vector<double> cn = coordination(s, D3_CN_CUTOFF, &cnp);
  std::vector<std::vector<double>> gw(nat), dgw(nat);
  for (int i = 0; i < nat; ++i) {
    int nr = d3_nref(s.z[i]);
    auto& cref = g_tables.get("d3.cnref." + std::to_string(s.z[i]));
    std::vector<double> logit(nr);
    double mx = -INFINITY;
    for (int k = 0; k < nr; ++k) {
      logit[k] = -D3_WF * std::pow(cn[i] - cref[k], 2);
      mx = std::max(mx, logit[k]);
    }
    std::vector<double> raw(nr);
    double norm = 0, dnorm = 0;
    for (int k = 0; k < nr; ++k) {
      raw[k] = std::exp(logit[k] - mx);
      norm += raw[k];
      dnorm += 2.0 * D3_WF * (cref[k] - cn[i]) * raw[k];
    }
    double ninv = 1.0 / norm;
    gw[i].resize(nr);
    dgw[i].resize(nr);
    for (int k = 0; k < nr; ++k) {
      double expd = 2.0 * D3_WF * (cref[k] - cn[i]) * raw[k];
      gw[i][k] = raw[k] * ninv;
      dgw[i][k] = expd * ninv - raw[k] * dnorm * ninv * ninv;
      if (!std::isfinite(gw[i][k])) gw[i][k] = 0;
      if (!std::isfinite(dgw[i][k])) dgw[i][k] = 0;
    }
  }
  Mat c6(nat, nat), dc6(nat, nat);
  for (int i = 0; i < nat; ++i)
    for (int j = 0; j <= i; ++j) {
      double cij = 0, di = 0, dj = 0;
      for (size_t a = 0; a < gw[i].size(); ++a)
        for (size_t b = 0; b < gw[j].size(); ++b) {
          double r = d3_c6ref(s.z[i], (int)a, s.z[j], (int)b);
          cij += gw[i][a] * gw[j][b] * r;
          di += dgw[i][a] * gw[j][b] * r;
          dj += gw[i][a] * dgw[j][b] * r;
        }
      c6(i, j) = c6(j, i) = cij;
      if (i == j) dc6(i, i) = di + dj;
      else { dc6(i, j) = di; dc6(j, i) = dj; }
    }
  double e = 0.0;
  std::vector<double> dedcn(nat, 0.0);
  for (auto& p : unique_pairs(s, D3_PAIR_CUTOFF, true)) {
    int i = p.i, j = p.j;
    if (p.r2 <= 1e-14) continue;
    double r4r2ij = 3.0 * d3_r4r2(s.z[i]) * d3_r4r2(s.z[j]);
    double r0 = a1 * std::sqrt(r4r2ij) + a2;
    double r02 = r0 * r0, r06 = r02 * r02 * r02, r08 = r06 * r02;
    double r2 = p.r2, r4 = r2 * r2;
    double t6 = 1.0 / (r4 * r2 + r06);
    double t8 = 1.0 / (r4 * r4 + r08);
    double d6 = -6.0 * r4 * t6 * t6;
    double d8 = -8.0 * r4 * r2 * t8 * t8;
    double ed = s6 * t6 + s8 * r4r2ij * t8;
    double gd = s6 * d6 + s8 * r4r2ij * d8;
    double cij = c6(i, j);
    e -= cij * ed;
    if (grad) {
      Vec3 rij = p.dr * -1.0;
      Vec3 dg = rij * (-cij * gd);
      (*grad)[i] += dg;
      (*grad)[j] -= dg;
    }
    dedcn[i] -= dc6(i, j) * ed;
    dedcn[j] -= dc6(j, i) * ed;
  }
  if (grad) {
    for (auto& p : cnp) {
      if (p.i == p.j) continue;
      double r = p.rij.norm();
      if (r <= 1e-14) continue;
      double pref = (dedcn[p.i] + dedcn[p.j]) * p.dcn_dr / r;
      Vec3 gi = p.rij * pref;
      (*grad)[p.i] += gi;
      (*grad)[p.j] -= gi;
    }
  }
  return e;
}

// ---------------------------------------------------------------- halogen bonds
// src/halogen.rs:64-160 (energy and gradient) with the triples of :716-786.
// Each donor X (Cl, Br, I, At) whose strength c = 0.1 CXB is non-zero pairs
// with its nearest other atom K and with every acceptor J (N, O, P, S) within
// 20 bohr (r^2 > 1e-24 and r^2 <= 400).  With T = (r_KX^2 + r_JX^2 - r_JK^2) /
// (r_KX r_JX) (twice the cosine of the K-X-J angle), b = 1/2 - T/4 and
// u = (r0 / r_JX)^6, r0 = xbrad (R_X + R_J) in the xTB atomic radii,
//   E_XJ = c b^6 (u^2 - xbdamp u) / (1 + u^2),
// where r_JX carries the reference's +1e-18.  The gradient is written as the
// derivatives of E_XJ with respect to the three squared distances.
bool is_halogen_donor(int z) { return z == 17 || z == 35 || z == 53 || z == 85; }
bool is_halogen_acceptor(int z) { return z == 7 || z == 8 || z == 15 || z == 16; }

double halogen(const System& s, std::vector<Vec3>* grad) {
  const double cutoff2 = 20.0 * 20.0, eps = 1e-18;
  double e = 0.0;
  for (int x = 0; x < s.nat(); ++x) {
    if (!is_halogen_donor(s.z[x])) continue;
    const std::string key = "elem." + std::to_string(s.z[x]) + ".cxb";
    const double c = 0.1 * (g_tables.has(key) ? g_tables.get(key)[0] : 0.0);
    int k = -1;
    double kr2 = 0.0;
    for (int j = 0; j < s.nat(); ++j) {  // nearest other atom inside the cutoff
      if (j == x) continue;
      const double r2 = (s.pos[j] - s.pos[x]).norm2();
      if (r2 <= 1e-24 || r2 > cutoff2) continue;
      if (k < 0 || r2 < kr2) { k = j; kr2 = r2; }
    }
    if (k < 0 || c == 0.0) continue;
    const double damp = g_params.req("xbdamp"), rscale = g_params.req("xbrad");
    for (int j = 0; j < s.nat(); ++j) {
      if (j == x || !is_halogen_acceptor(s.z[j])) continue;
      const Vec3 vjx = s.pos[j] - s.pos[x], vkx = s.pos[k] - s.pos[x], vjk = s.pos[j] - s.pos[k];
      const double djx = vjx.norm2(), dkx = vkx.norm2(), djk = vjk.norm2();
      if (djx <= 1e-24 || djx > cutoff2) continue;  // outside the donor's neighbour list
      if (djx <= eps || dkx <= eps) continue;
      const double rjx = std::sqrt(djx) + eps, rkx = std::sqrt(dkx) + eps;
      const double xy = std::sqrt(dkx * djx);
      if (xy <= eps) continue;
      const double T = (dkx + djx - djk) / xy;
      const double b = 0.5 - 0.25 * T;
      const double b5 = std::pow(b, 5.0), b6 = b5 * b;
      const double r0 = rscale * (atomic_radius_bohr(s.z[x]) + atomic_radius_bohr(s.z[j]));
      const double u = std::pow(r0 / rjx, 6.0);
      const double num = u * u - damp * u, den = 1.0 + u * u;
      const double L = num / den;
      e += c * b6 * L;
      if (!grad) continue;
      // dL/dr_JX and dE/dT
      const double dL = (6.0 * u * (damp - 2.0 * u) / den + 12.0 * u * u * num / (den * den)) / rjx;
      const double dET = -1.5 * c * b5 * L;
      // dE/d(r^2) for the three squared distances
      const double gjx = dET * (1.0 / (rkx * rjx) - 0.5 * T / (rjx * rjx)) + 0.5 * c * b6 * dL / rjx;
      const double gkx = dET * (1.0 / (rkx * rjx) - 0.5 * T / (rkx * rkx));
      const double gjk = -dET / xy;
      (*grad)[j] += vjx * (2.0 * gjx) + vjk * (2.0 * gjk);
      (*grad)[x] -= vjx * (2.0 * gjx) + vkx * (2.0 * gkx);
      (*grad)[k] += vkx * (2.0 * gkx) - vjk * (2.0 * gjk);
    }
  }
  return e;
}

// ---------------------------------------------------------------- SCC
struct Step {
  Mat P, W, F;
  std::vector<double> eps, f, q;
  double mu = 0, ts = 0;
};

struct Result {
  double terms[15] = {0};
  std::vector<Vec3> grad;
  std::vector<double> shell_q, atom_q, eps, cn, occ;
  Vec3 dipole;
  int iterations = 0;
  bool converged = false;
  int rung = -1;       // fallback-ladder attempt that converged (src/electronic.rs:1420)
  double etemp = 0.0;  // electronic temperature of that attempt (src/electronic.rs:2024-2026)
  double fermi = 0, nelec = 0, rms = 0;
  Mat S, H0, P, W, F;            // F: Fock matrix of the last step (SccStep::fock)
  std::vector<double> shell_pot;  // potential of the final output charges (shell_scc_potential)
  int nao = 0, nsh = 0;
};

// src/electronic.rs:800-847 + :849-2054 (plain charge-vector SCC branch) and
// src/gradient.rs:122-531 (analytic gradient, stock terms only)
Result run(const System& sys, const Options& opt, const double* init_q, bool want_grad) {
  Result res;
  int nat = sys.nat();
  if (nat == 0) throw OracleError(E_INVALID_INPUT, "cannot run GFN1 SCC for an empty basis");
  for (int a = 0; a < nat; ++a) {
    if (!(std::isfinite(sys.pos[a].x) && std::isfinite(sys.pos[a].y) && std::isfinite(sys.pos[a].z)))
      throw OracleError(E_INVALID_INPUT, "non-finite coordinate");
  }
  Basis b = build_basis(sys.z);
  int n = (int)b.aos.size(), nsh = (int)b.shells.size();
  res.nao = n;
  res.nsh = nsh;
  // --- H0 (src/hamiltonian.rs:44-134)
  std::vector<CnPair> cn_pairs;
  std::vector<double> cn = coordination(sys, CUTOFF_CN, &cn_pairs);
  Mat S(n, n);
  for (int a = 0; a < nat; ++a) {  // src/integrals.rs:166-186 (on-site blocks)
    int f = b.atom_ao_first[a], c = b.atom_ao_count[a];
    for (int i = f; i < f + c; ++i)
      for (int j = f; j < f + c; ++j) S(i, j) = contracted_overlap(b.aos[i], b.aos[j], sys.pos[a], sys.pos[a]);
  }
  for (int a = 0; a < nat; ++a)  // src/integrals.rs:188-220 (directed atom pairs)
    for (int bb = 0; bb < nat; ++bb) {
      if (a == bb) continue;
      Vec3 dr = sys.pos[bb] - sys.pos[a];
      double r2 = dr.norm2();
      if (r2 <= 1e-24 || r2 > CUTOFF_INTEGRAL * CUTOFF_INTEGRAL) continue;
      int fa = b.atom_ao_first[a], na = b.atom_ao_count[a];
      int fb = b.atom_ao_first[bb], nb = b.atom_ao_count[bb];
      for (int i = fa; i < fa + na; ++i)
        for (int j = fb; j < fb + nb; ++j)
          S(i, j) += contracted_overlap(b.aos[i], b.aos[j], sys.pos[a], sys.pos[bb]);
    }
  std::vector<double> se(nsh), dsedcn(nsh);
  for (int i = 0; i < nsh; ++i) {
    dsedcn[i] = -b.shells[i].kcn;
    se[i] = b.shells[i].hdiag_ha - b.shells[i].kcn * cn[b.shells[i].atom];
  }
  Mat H0(n, n);
  for (int i = 0; i < n; ++i) {
    const Shell& si = b.shells[b.aos[i].shell];
    for (int j = 0; j <= i; ++j) {
      const Shell& sj = b.shells[b.aos[j].shell];
      double hij;
      if (si.atom == sj.atom) hij = 0.5 * (se[b.aos[i].shell] + se[b.aos[j].shell]);
      else {
        double r2 = (sys.pos[si.atom] - sys.pos[sj.atom]).norm2();
        double rad = atomic_radius_bohr(si.z) + atomic_radius_bohr(sj.z);
        double rr = std::sqrt(std::sqrt(r2) / rad);
        hij = 0.5 * (se[b.aos[i].shell] + se[b.aos[j].shell]) * hscale(si, sj) * shell_polynomial(si, sj, rr);
      }
      double v = S(i, j) * hij;
      H0(i, j) = v;
      H0(j, i) = v;
    }
  }
  // --- SCC setup (src/electronic.rs:861-927)
  double nelec = b.total_ref - sys.charge;
  if (!std::isfinite(nelec)) throw OracleError(E_INVALID_INPUT, "electron count is not finite");
  if (nelec < -1e-8) throw OracleError(E_INVALID_INPUT, "electron count is negative");
  if (nelec > 2.0 * n + 1e-8) throw OracleError(E_INVALID_INPUT, "electron count exceeds basis capacity");
  res.nelec = nelec;
  const SpinChannels spin = resolve_spin_channels(nelec, opt.spin_multiplicity, n);
  Mat A = coulomb_matrix(sys, b);
  // Lowdin orthogonaliser (src/linalg.rs:193-217)
  std::vector<double> sw;
  Mat U;
  sym_eig(S, sw, U);
  Mat Us(n, n);
  for (int k = 0; k < n; ++k) {
    if (sw[k] <= opt.eigen_tolerance) {
      char buf[128];
      snprintf(buf, sizeof buf, "overlap matrix is not positive definite; eigenvalue %d = %.3e", k, sw[k]);
      throw OracleError(E_INVALID_INPUT, buf);
    }
    double fac = 1.0 / std::sqrt(sw[k]);
    for (int i = 0; i < n; ++i) Us(i, k) = U(i, k) * fac;
  }
  Mat X = matmul(Us, transpose(U));
  Mat XT = transpose(X);
  double erep = repulsion(sys, nullptr);
  double edisp = opt.enable_dispersion ? dispersion(sys, nullptr) : 0.0;
  // --- SCC loop (src/electronic.rs:1231-1955)
  double base_mixing = std::min(1.0, std::max(0.01, opt.mixing));
  bool base_broyden = opt.scc_broyden != 0;
  struct Rung { bool broyden; double mix, lshift, etemp; int maxit; };
  int robust = std::max(opt.max_scc, 800);
  Rung ladder[4] = {{base_broyden, base_mixing, opt.level_shift, opt.electronic_temperature, opt.max_scc},
                    {false, 0.20, std::max(opt.level_shift, 0.20), opt.electronic_temperature, robust},
                    {false, 0.10, std::max(opt.level_shift, 0.10), opt.electronic_temperature, robust},
                    {true, base_mixing, 0.0, std::max(opt.electronic_temperature, 3000.0), std::max(opt.max_scc, 250)}};
  bool converged = false;
  int iterations = 0;
  double final_rms = INFINITY;
  Step last;
  bool have_last = false;
  auto scc_step = [&](const std::vector<double>& qin, double etemp, double lshift, const Mat* prevP) {
    Step st;
    Coul c = coulomb(b, A, qin, nat);  // src/electronic.rs:2089-2092
    std::vector<double> vao(n);
    for (int sh = 0; sh < nsh; ++sh)
      for (int k = 0; k < b.shells[sh].nao; ++k) vao[b.shells[sh].first_ao + k] = c.pot[sh];
    Mat F = H0;  // src/electronic.rs:3133-3158
    for (int i = 0; i < n; ++i)
      for (int j = 0; j <= i; ++j) {
        double v = -S(i, j) * 0.5 * (vao[i] + vao[j]);
        F(i, j) += v;
        if (i != j) F(j, i) += v;
      }
    if (lshift != 0.0 && prevP) {  // src/electronic.rs:2125-2137
      Mat SP = matmul(S, *prevP);
      Mat SPS = matmul(SP, S);
      for (size_t k = 0; k < F.a.size(); ++k) F.a[k] += lshift * (S.a[k] - 0.5 * SPS.a[k]);
    }
    Mat Fo = matmul(XT, matmul(F, X));  // src/linalg.rs:219-241
    Mat V;
    sym_eig(Fo, st.eps, V);
    Mat C = matmul(X, V);
    double kt = std::max(0.0, etemp) * KB_HARTREE_PER_K;
    Occ o = spin.on ? spin_constrained_occupations(st.eps, spin, kt) : occupations(st.eps, nelec, kt);
    st.f = o.f;
    st.mu = o.mu;
    st.ts = o.ts;
    // column_weighted_gram (src/linalg.rs:243-273)
    auto gram = [&](const std::vector<double>& wgt) {
      Mat Cs(n, n);
      for (int col = 0; col < n; ++col) {
        if (wgt[col] == 0.0) continue;
        for (int row = 0; row < n; ++row) Cs(row, col) = C(row, col) * wgt[col];
      }
      Mat out = matmul(Cs, transpose(C));
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < i; ++j) {
          double avg = 0.5 * (out(i, j) + out(j, i));
          out(i, j) = avg;
          out(j, i) = avg;
        }
      return out;
    };
    st.P = gram(st.f);
    std::vector<double> ef(n);
    for (int i = 0; i < n; ++i) ef[i] = st.eps[i] * st.f[i];
    st.W = gram(ef);
    st.F = F;
    st.q.assign(nsh, 0.0);  // src/electronic.rs:3160-3180
    for (int sh = 0; sh < nsh; ++sh) {
      double pop = 0.0;
      for (int k = 0; k < b.shells[sh].nao; ++k) {
        int mu = b.shells[sh].first_ao + k;
        for (int nu = 0; nu < n; ++nu) pop += S(mu, nu) * st.P(mu, nu);
      }
      st.q[sh] = b.shells[sh].ref_occ - pop;
    }
    return st;
  };
  auto e_el = [&](const Mat& P) {
    double s = 0;
    for (size_t k = 0; k < P.a.size(); ++k) s += H0.a[k] * P.a[k];
    return s;
  };
  int rung_used = -1;
  for (int attempt = 0; attempt < 4 && !converged; ++attempt) {
    const Rung& rg = ladder[attempt];
    rung_used = attempt;
    std::vector<double> vmix(nsh, 0.0);
    if (init_q) for (int i = 0; i < nsh; ++i) vmix[i] = init_q[i];
    Broyden br(nsh, std::max(opt.scc_broyden_size, 2), rg.mix);
    Mat prevP;
    bool have_prev = false;
    bool have_e = false;
    double last_e = 0.0;
    have_last = false;
    final_rms = INFINITY;
    for (int it = 1; it <= rg.maxit; ++it) {
      iterations = it;
      Step st = scc_step(vmix, rg.etemp, rg.lshift, have_prev ? &prevP : nullptr);
      double ss = 0;
      for (int i = 0; i < nsh; ++i) ss += (st.q[i] - vmix[i]) * (st.q[i] - vmix[i]);
      final_rms = nsh ? std::sqrt(ss / nsh) : 0.0;
      Coul co = coulomb(b, A, st.q, nat);  // src/electronic.rs:2173-2191
      double escc = e_el(st.P) + co.e2 + co.e3 + st.ts;
      double err = have_e ? std::fabs(escc - last_e) : INFINITY;
      if (err < opt.energy_tolerance && final_rms < opt.charge_tolerance) {
        converged = true;
        last = st;
        have_last = true;
        break;
      }
      std::vector<double> resid(nsh);
      for (int i = 0; i < nsh; ++i) resid[i] = st.q[i] - vmix[i];
      std::vector<double> qn;
      if (!rg.broyden) qn = damped_step(vmix, resid, rg.mix);
      else {
        std::vector<double> cand;
        if (br.next(vmix, resid, cand) && trusted(cand)) qn = cand;
        else qn = damped_step(vmix, resid, rg.mix);
      }
      if (rg.lshift != 0.0) { prevP = st.P; have_prev = true; }
      else have_prev = false;
      vmix = qn;
      last_e = escc;
      have_e = true;
      last = st;
      have_last = true;
    }
  }
  res.iterations = iterations;
  res.rms = final_rms;
  if (!converged) {
    char buf[160];
    snprintf(buf, sizeof buf, "GFN1 SCC did not converge after %d iterations (rms=%.6e)", iterations, final_rms);
    throw OracleError(E_SCC_NOT_CONVERGED, buf);
  }
  (void)have_last;
  // --- final assembly (src/electronic.rs:1957-2053)
  double eel = e_el(last.P);
  Coul sc = coulomb(b, A, last.q, nat);
  double ehal = halogen(sys, nullptr);
  double total_internal = eel + sc.e2 + sc.e3 + erep + edisp + ehal;
  double total_free = total_internal + last.ts;
  // named_values order, src/electronic.rs:681-699
  double t[15] = {total_free, total_internal, erep, eel, sc.e2, sc.e3, 0.0, edisp, ehal, 0.0, 0.0, 0.0, 0.0, 0.0, last.ts};
  std::memcpy(res.terms, t, sizeof t);
  res.converged = true;
  res.rung = rung_used;
  res.etemp = ladder[rung_used].etemp;
  res.shell_q = last.q;
  res.atom_q = sc.qat;
  res.eps = last.eps;
  res.occ = last.f;
  res.fermi = last.mu;
  res.cn = cn;
  res.dipole = Vec3();
  for (int a = 0; a < nat; ++a) res.dipole += sys.pos[a] * sc.qat[a];  // src/field.rs:89-95
  res.S = S;
  res.H0 = H0;
  res.P = last.P;
  res.W = last.W;
  res.F = last.F;          // src/electronic.rs:2019
  res.shell_pot = sc.pot;  // src/electronic.rs:1980, 2031
  if (!want_grad) return res;

  // --- analytic gradient (src/gradient.rs:122-242, :244-531)
  std::vector<Vec3> g(nat), gel(nat);
  std::vector<double> dedcn(nat, 0.0);
  std::vector<double> vao(n);
  for (int sh = 0; sh < nsh; ++sh)
    for (int k = 0; k < b.shells[sh].nao; ++k) vao[b.shells[sh].first_ao + k] = sc.pot[sh];
  std::vector<double> srad(nsh);
  for (int i = 0; i < nsh; ++i) srad[i] = atomic_radius_bohr(b.shells[i].z);
  for (auto& pr : unique_pairs(sys, CUTOFF_INTEGRAL, true)) {
    int anu = pr.i, amu = pr.j;
    Vec3 rmu = sys.pos[amu], rnu = sys.pos[anu];
    Vec3 rvec = rmu - rnu;
    double r2 = rvec.norm2();
    Vec3 gmu, gnu;
    double dcmu = 0, dcnu = 0;
    if (r2 > 1e-12) {
      for (int smu = b.atom_shell_first[amu]; smu < b.atom_shell_first[amu] + b.atom_shell_count[amu]; ++smu) {
        const Shell& Smu = b.shells[smu];
        for (int snu = b.atom_shell_first[anu]; snu < b.atom_shell_first[anu] + b.atom_shell_count[anu]; ++snu) {
          const Shell& Snu = b.shells[snu];
          double radsum = srad[smu] + srad[snu];
          double rr = std::sqrt(std::sqrt(r2) / radsum);
          double hs = hscale(Smu, Snu) * shell_polynomial(Smu, Snu, rr);
          double hij = 0.5 * (se[smu] + se[snu]) * hs;
          // src/gradient.rs:1157-1175
          Vec3 dlog;
          {
            double fi = 1.0 + Smu.poly * rr, fj = 1.0 + Snu.poly * rr;
            double poly = fi * fj;
            if (std::fabs(poly) > 1e-18) {
              double dpoly = (fi * Snu.poly + fj * Smu.poly) * 0.5 * rr / r2;
              dlog = rvec * (dpoly / poly);
            }
          }
          for (int mu = Smu.first_ao; mu < Smu.first_ao + Smu.nao; ++mu)
            for (int nu = Snu.first_ao; nu < Snu.first_ao + Snu.nao; ++nu) {
              double ov;
              Vec3 dbra, dket;
              contracted_overlap_deriv(b.aos[mu], b.aos[nu], rmu, rnu, ov, dbra, dket);
              double p = last.P(mu, nu), w = last.W(mu, nu);
              double coeff = p * (2.0 * hij - (vao[mu] + vao[nu])) - 2.0 * w;
              gmu += dbra * coeff;
              gnu += dket * coeff;
              Vec3 pg = dlog * (2.0 * p * hij * ov);
              gmu += pg;
              gnu -= pg;
              dcmu += dsedcn[smu] * hs * p * ov;
              dcnu += dsedcn[snu] * hs * p * ov;
            }
        }
      }
    }
    gel[amu] += gmu;
    gel[anu] += gnu;
    dedcn[amu] += dcmu;
    dedcn[anu] += dcnu;
  }
  for (int sh = 0; sh < nsh; ++sh)  // src/gradient.rs:464-469
    for (int k = 0; k < b.shells[sh].nao; ++k) {
      int mu = b.shells[sh].first_ao + k;
      dedcn[b.shells[sh].atom] += dsedcn[sh] * last.P(mu, mu);
    }
  for (auto& p : cn_pairs) {  // src/gradient.rs:470-490
    if (p.i == p.j) continue;
    double r = p.rij.norm();
    if (r <= 1e-12) continue;
    double pref = (dedcn[p.i] + dedcn[p.j]) * p.dcn_dr / r;
    Vec3 gi = p.rij * pref;
    gel[p.i] += gi;
    gel[p.j] -= gi;
  }
  for (int i = 0; i < nsh; ++i) {  // src/gradient.rs:493-516
    int ai = b.shells[i].atom;
    for (int j = 0; j < i; ++j) {
      int aj = b.shells[j].atom;
      if (ai == aj) continue;
      Vec3 rv = sys.pos[ai] - sys.pos[aj];
      double r = rv.norm();
      if (r <= 1e-12) continue;
      double gm = 2.0 / (1.0 / b.shells[i].hardness + 1.0 / b.shells[j].hardness);
      double den = r * r + 1.0 / (gm * gm);
      Vec3 dk = rv * (-1.0 / (den * std::sqrt(den)));
      double scale = last.q[i] * last.q[j];
      gel[ai] += dk * scale;
      gel[aj] -= dk * scale;
    }
  }
  for (int a = 0; a < nat; ++a) g[a] += gel[a];
  std::vector<Vec3> grep(nat), gdisp(nat);
  std::vector<Vec3> ghal(nat);
  repulsion(sys, &grep);
  if (opt.enable_dispersion) dispersion(sys, &gdisp);
  halogen(sys, &ghal);
  for (int a = 0; a < nat; ++a) g[a] += grep[a] + gdisp[a] + ghal[a];
  res.grad = g;
  return res;
}

thread_local std::string t_err;

}  // namespace

// ============================================================== C API
extern "C" {

struct oracle_options {
  int max_scc;
  double energy_tolerance;
  double charge_tolerance;
  double mixing;
  int scc_broyden;
  int scc_broyden_size;
  double electronic_temperature;
  int enable_dispersion;
  double charge;
  double level_shift;
  int spin_multiplicity;  // 0: none
};

const char* oracle_last_error() { return t_err.c_str(); }

int oracle_init(const char* tables_path) {
  try {
    load_tables(tables_path);
    build_params();
    return OK;
  } catch (const OracleError& e) {
    t_err = e.what();
    return e.code;
  }
}

static Options to_opts(const oracle_options* o) {
  Options opt;
  if (o) {
    opt.max_scc = o->max_scc;
    opt.energy_tolerance = o->energy_tolerance;
    opt.charge_tolerance = o->charge_tolerance;
    opt.mixing = o->mixing;
    opt.scc_broyden = o->scc_broyden;
    opt.scc_broyden_size = o->scc_broyden_size;
    opt.electronic_temperature = o->electronic_temperature;
    opt.enable_dispersion = o->enable_dispersion;
    opt.level_shift = o->level_shift;
    opt.spin_multiplicity = o->spin_multiplicity;
  }
  return opt;
}

int oracle_sizes(int nat, const int* z, int* nao, int* nsh) {
  try {
    std::vector<int> zs(z, z + nat);
    Basis b = build_basis(zs);
    *nao = (int)b.aos.size();
    *nsh = (int)b.shells.size();
    return OK;
  } catch (const OracleError& e) {
    t_err = e.what();
    return e.code;
  }
}

// The halogen-bond term alone (src/halogen.rs:64-160): energy and, when grad
// is not null, its gradient [nat*3].
int oracle_halogen(int nat, const int* z, const double* xyz_bohr, double* energy, double* grad) {
  try {
    System s;
    s.z.assign(z, z + nat);
    for (int a = 0; a < nat; ++a) s.pos.push_back(Vec3(xyz_bohr[3 * a], xyz_bohr[3 * a + 1], xyz_bohr[3 * a + 2]));
    std::vector<Vec3> g(nat);
    *energy = halogen(s, grad ? &g : nullptr);
    if (grad)
      for (int a = 0; a < nat; ++a) { grad[3 * a] = g[a].x; grad[3 * a + 1] = g[a].y; grad[3 * a + 2] = g[a].z; }
    return OK;
  } catch (const OracleError& e) {
    t_err = e.what();
    return e.code;
  }
}

// One classical term alone, energy and (grad not null) gradient [nat*3]:
// which = 0 repulsion (src/repulsion.rs:24-59, 139-159), 1 D3(BJ) dispersion
// (src/dispersion.rs:1232-1360), 2 halogen bonds (src/halogen.rs:64-160).
// The per-term split of the reference's gradient probe
// (tests/gradient_fd_probe.rs:41-120).
int oracle_classical_term(int which, int nat, const int* z, const double* xyz_bohr, double* energy, double* grad) {
  try {
    if (which < 0 || which > 2) throw OracleError(E_INVALID_INPUT, "unknown classical term");
    System s;
    s.z.assign(z, z + nat);
    for (int a = 0; a < nat; ++a) s.pos.push_back(Vec3(xyz_bohr[3 * a], xyz_bohr[3 * a + 1], xyz_bohr[3 * a + 2]));
    std::vector<Vec3> g(nat);
    std::vector<Vec3>* gp = grad ? &g : nullptr;
    *energy = which == 0 ? repulsion(s, gp) : which == 1 ? dispersion(s, gp) : halogen(s, gp);
    if (grad)
      for (int a = 0; a < nat; ++a) { grad[3 * a] = g[a].x; grad[3 * a + 1] = g[a].y; grad[3 * a + 2] = g[a].z; }
    return OK;
  } catch (const OracleError& e) {
    t_err = e.what();
    return e.code;
  }
}

// One molecule.  Output pointers may be null.  terms[15] in the order of
// EnergyTerms::named_values (src/electronic.rs:681-699).
int oracle_run(int nat, const int* z, const double* xyz_bohr, const oracle_options* o, const double* init_shell_q,
               int want_grad, double* terms, double* grad, double* shell_q, double* atom_q, double* eps,
               double* occ, double* dipole, double* cn, int* iterations, int* converged, double* fermi, double* S,
               double* H0, double* P, double* W, int* rung, double* etemp_used, double* F, double* shell_pot) {
  try {
    System s;
    s.z.assign(z, z + nat);
    for (int a = 0; a < nat; ++a) s.pos.push_back(Vec3(xyz_bohr[3 * a], xyz_bohr[3 * a + 1], xyz_bohr[3 * a + 2]));
    s.charge = o ? o->charge : 0.0;
    Options opt = to_opts(o);
    Result r = run(s, opt, init_shell_q, want_grad != 0);
    if (terms) std::memcpy(terms, r.terms, sizeof r.terms);
    if (grad && want_grad)
      for (int a = 0; a < nat; ++a) { grad[3 * a] = r.grad[a].x; grad[3 * a + 1] = r.grad[a].y; grad[3 * a + 2] = r.grad[a].z; }
    if (shell_q) std::copy(r.shell_q.begin(), r.shell_q.end(), shell_q);
    if (atom_q) std::copy(r.atom_q.begin(), r.atom_q.end(), atom_q);
    if (eps) std::copy(r.eps.begin(), r.eps.end(), eps);
    if (occ) std::copy(r.occ.begin(), r.occ.end(), occ);
    if (dipole) { dipole[0] = r.dipole.x; dipole[1] = r.dipole.y; dipole[2] = r.dipole.z; }
    if (cn) std::copy(r.cn.begin(), r.cn.end(), cn);
    if (iterations) *iterations = r.iterations;
    if (converged) *converged = r.converged ? 1 : 0;
    if (fermi) *fermi = r.fermi;
    if (S) std::copy(r.S.a.begin(), r.S.a.end(), S);
    if (H0) std::copy(r.H0.a.begin(), r.H0.a.end(), H0);
    if (P) std::copy(r.P.a.begin(), r.P.a.end(), P);
    if (W) std::copy(r.W.a.begin(), r.W.a.end(), W);
    if (rung) *rung = r.rung;
    if (etemp_used) *etemp_used = r.etemp;
    if (F) std::copy(r.F.a.begin(), r.F.a.end(), F);
    if (shell_pot) std::copy(r.shell_pot.begin(), r.shell_pot.end(), shell_pot);
    return OK;
  } catch (const OracleError& e) {
    t_err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    t_err = e.what();
    return E_INVALID_INPUT;
  }
}

// Batch of independent molecules, parallel over molecules on `nthreads` host
// threads (one molecule per thread at a time; 0 = all hardware threads).  atom_offsets has nmol+1 entries.  shell_offsets (nmol+1, may be
// null) places each molecule's shell charges in shell_q.
int oracle_run_batch(int nmol, const int* atom_offsets, const int* z, const double* xyz_bohr, const double* charge,
                     const oracle_options* o, int want_grad, int nthreads, double* energy, double* grad,
                     const int* shell_offsets, double* shell_q, int* iterations, int* status, int* rungs) {
  std::atomic<int> next(0), worst(OK);
  auto worker = [&]() {
    for (;;) {
      int m = next.fetch_add(1);
      if (m >= nmol) break;
      int a0 = atom_offsets[m], nat = atom_offsets[m + 1] - atom_offsets[m];
      int code = OK;
      try {
        System s;
        s.z.assign(z + a0, z + a0 + nat);
        for (int a = 0; a < nat; ++a)
          s.pos.push_back(Vec3(xyz_bohr[3 * (a0 + a)], xyz_bohr[3 * (a0 + a) + 1], xyz_bohr[3 * (a0 + a) + 2]));
        s.charge = charge ? charge[m] : 0.0;
        Options opt = to_opts(o);
        Result r = run(s, opt, nullptr, want_grad != 0);
        if (energy) energy[m] = r.terms[0];
        if (grad && want_grad)
          for (int a = 0; a < nat; ++a) {
            grad[3 * (a0 + a)] = r.grad[a].x;
            grad[3 * (a0 + a) + 1] = r.grad[a].y;
            grad[3 * (a0 + a) + 2] = r.grad[a].z;
          }
        if (shell_q && shell_offsets) std::copy(r.shell_q.begin(), r.shell_q.end(), shell_q + shell_offsets[m]);
        if (iterations) iterations[m] = r.iterations;
        if (rungs) rungs[m] = r.rung;
      } catch (const OracleError& e) {
        code = e.code;
      } catch (const std::exception&) {
        code = E_INVALID_INPUT;
      }
      if (status) status[m] = code;
      if (rungs && code != OK) rungs[m] = -1;
      int w = worst.load();
      while (code > w && !worst.compare_exchange_weak(w, code)) {
      }
    }
  };
  int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  nt = std::min(nt, std::max(1, nmol));
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
  return worst.load();
}

}  // extern "C"
