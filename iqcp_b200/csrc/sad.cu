// SAD initial density: superposition of spherically averaged atomic RHF
// densities (build_sad_density, crates/qc-core/src/scf/sad.rs:698-760, which
// follows PySCF's AtomSphAverageRHF, atom_hf.py:89-188).
//
// Host code.  Per element of the basis, a one-atom context gives the atomic
// S, T, V and the 8-fold compressed ERIs from this library's kernels; the
// atomic SCF itself is a few dozen iterations on matrices of at most ~20
// functions, solved here with a cyclic Jacobi eigensolver on the radial
// blocks (at most 5 x 5 for the bases of the tables).  Steps:
//   - basis functions grouped by l in order of first appearance, each shell
//     contributing its n_comp Cartesian components (1, 3, 6): sad.rs:145-198;
//   - eigenproblem per l on the component-averaged radial blocks
//     F_avg[i][j] = sum_m F[(i,m),(j,m)] / n_comp (same for S), solved by
//     symmetric orthogonalisation (S eigenvalues below 1e-10 dropped), the
//     radial vectors copied to every component: sad.rs:207-356;
//   - occupations per l from the configuration (s, p, d electron counts):
//     full radial shells 2 per component, the next one fractional
//     remaining / n_comp per component: sad.rs:362-520;
//   - SCF from the core Hamiltonian, F = H + sum_ls D_ls [(mn|ls) - 1/2 (ml|ns)],
//     E = 1/2 Tr D (H + F), stop when |dE| < 1e-10 or after 40 Fock builds
//     (the density that produced the converged F is returned): sad.rs:525-640;
//     one-electron atoms take the core-Hamiltonian density;
//   - the atomic block of each element is computed once and copied to every
//     atom of that element (sad.rs:740-756); blocks are also kept for the
//     process, keyed by element and shells, for the next geometry.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/iqcp.h"

namespace {

// (n_s, n_p, n_d) electrons of the ground configuration, H..Ar (sad.rs:67-90)
void electron_config(int z, int cfg[3]) {
  static const int t[19][3] = {{0, 0, 0}, {1, 0, 0},  {2, 0, 0}, {3, 0, 0}, {4, 0, 0}, {4, 1, 0},  {4, 2, 0},
                               {4, 3, 0}, {4, 4, 0},  {4, 5, 0}, {4, 6, 0}, {5, 6, 0}, {6, 6, 0},  {6, 7, 0},
                               {6, 8, 0}, {6, 9, 0},  {6, 10, 0}, {6, 11, 0}, {6, 12, 0}};
  for (int k = 0; k < 3; ++k) cfg[k] = (z >= 0 && z <= 18) ? t[z][k] : 0;
}

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// Cyclic Jacobi: a (n x n, row-major, symmetric) is destroyed; w ascending,
// v[:, k] the eigenvector of w[k].
void jacobi_eig(int n, std::vector<double> a, std::vector<double>& w, std::vector<double>& v) {
  v.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) v[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        tot += a[(size_t)i * n + j] * a[(size_t)i * n + j];
        if (i != j) off += a[(size_t)i * n + j] * a[(size_t)i * n + j];
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a[(size_t)p * n + q];
        if (apq == 0.0) continue;
        const double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q];
        const double theta = 0.5 * (aqq - app) / apq;
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {  // rotate rows/columns p, q
          const double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
          a[(size_t)k * n + p] = c * akp - s * akq;
          a[(size_t)k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = a[(size_t)p * n + k], aqk = a[(size_t)q * n + k];
          a[(size_t)p * n + k] = c * apk - s * aqk;
          a[(size_t)q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = v[(size_t)k * n + p], vkq = v[(size_t)k * n + q];
          v[(size_t)k * n + p] = c * vkp - s * vkq;
          v[(size_t)k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return a[(size_t)x * n + x] < a[(size_t)y * n + y]; });
  std::vector<double> vs((size_t)n * n);
  w.resize(n);
  for (int k = 0; k < n; ++k) {
    w[k] = a[(size_t)ord[k] * n + ord[k]];
    for (int i = 0; i < n; ++i) vs[(size_t)i * n + k] = v[(size_t)i * n + ord[k]];
  }
  v.swap(vs);
}

// F c = S c e on a small radial block by symmetric orthogonalisation
// (sad.rs:289-356): returns eigenvalues ascending and C (n x n, column k).
void gen_eig(int n, const std::vector<double>& f, const std::vector<double>& s, std::vector<double>& e,
             std::vector<double>& c) {
  e.assign(n, 0.0);
  c.assign((size_t)n * n, 0.0);
  if (n == 1) {
    e[0] = f[0] / s[0];
    c[0] = 1.0 / std::sqrt(s[0]);
    return;
  }
  std::vector<double> sw, sv;
  jacobi_eig(n, s, sw, sv);
  std::vector<double> x((size_t)n * n, 0.0);
  for (int k = 0; k < n; ++k) {
    if (sw[k] < 1e-10) continue;  // linear dependence
    const double is = 1.0 / std::sqrt(sw[k]);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) x[(size_t)i * n + j] += sv[(size_t)i * n + k] * is * sv[(size_t)j * n + k];
  }
  std::vector<double> fx((size_t)n * n, 0.0), fp((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double t = 0.0;
      for (int k = 0; k < n; ++k) t += f[(size_t)i * n + k] * x[(size_t)k * n + j];
      fx[(size_t)i * n + j] = t;
    }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double t = 0.0;
      for (int k = 0; k < n; ++k) t += x[(size_t)k * n + i] * fx[(size_t)k * n + j];
      fp[(size_t)i * n + j] = t;
    }
  std::vector<double> cp;
  jacobi_eig(n, fp, e, cp);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < n; ++k) {
      double t = 0.0;
      for (int j = 0; j < n; ++j) t += x[(size_t)i * n + j] * cp[(size_t)j * n + k];
      c[(size_t)i * n + k] = t;
    }
}

struct LGroup {
  int l, n_comp, n_rad;
  std::vector<int> bf;  // [radial shell][component] -> atomic basis function
};

std::vector<LGroup> l_groups(const std::vector<int>& shell_l) {
  std::vector<LGroup> g;
  int off = 0;
  for (int l : shell_l) {
    auto it = std::find_if(g.begin(), g.end(), [&](const LGroup& x) { return x.l == l; });
    if (it == g.end()) {
      g.push_back({l, ncart(l), 0, {}});
      it = g.end() - 1;
    }
    for (int c = 0; c < it->n_comp; ++c) it->bf.push_back(off + c);
    ++it->n_rad;
    off += ncart(l);
  }
  return g;
}

// Density from the spherically averaged eigenproblem of F with the
// fractional occupations of configuration cfg.  Per l the radial shells are
// occupied lowest first (the reference picks each l's columns in ascending
// energy order, sad.rs:431-518).
std::vector<double> sph_avg_density(int n, const std::vector<double>& F, const std::vector<double>& S,
                                    const std::vector<LGroup>& groups, const int cfg[3]) {
  std::vector<double> D((size_t)n * n, 0.0);
  for (const LGroup& g : groups) {
    const int nr = g.n_rad, nc = g.n_comp;
    std::vector<double> fa((size_t)nr * nr), sa((size_t)nr * nr);
    for (int i = 0; i < nr; ++i)
      for (int j = 0; j < nr; ++j) {
        double fs = 0.0, ss = 0.0;
        for (int m = 0; m < nc; ++m) {
          const int r = g.bf[(size_t)i * nc + m], c = g.bf[(size_t)j * nc + m];
          fs += F[(size_t)r * n + c];
          ss += S[(size_t)r * n + c];
        }
        fa[(size_t)i * nr + j] = fs / nc;
        sa[(size_t)i * nr + j] = ss / nc;
      }
    if (g.l >= 3) continue;
    const int ne = cfg[g.l];
    if (ne == 0) continue;
    std::vector<double> e, C;
    gen_eig(nr, fa, sa, e, C);
    const int per = 2 * nc, ndocc = ne / per, rem = ne - ndocc * per;
    for (int i = 0; i < nr; ++i) {
      const double occ = i < ndocc ? 2.0 : (i == ndocc && rem > 0 ? double(rem) / nc : 0.0);
      if (occ == 0.0) continue;
      for (int m = 0; m < nc; ++m)
        for (int a = 0; a < nr; ++a)
          for (int b = 0; b < nr; ++b)
            D[(size_t)g.bf[(size_t)a * nc + m] * n + g.bf[(size_t)b * nc + m]] +=
                occ * C[(size_t)a * nr + i] * C[(size_t)b * nr + i];
    }
  }
  return D;
}

inline long long pidx(long long i, long long j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

// Atomic block of element z from its shells (one-atom basis at the origin of
// its own centre): nbf_a x nbf_a, row-major.
int atomic_density(int z, const iqcp_basis_desc& one, const iqcp_options* opts, std::vector<double>& Da) {
  std::vector<int> sl(one.l, one.l + one.n_shells);
  int n = 0;
  for (int l : sl) n += ncart(l);
  iqcp_ctx* ctx = nullptr;
  int rc = iqcp_create(&one, opts, &ctx);
  if (rc) return rc;
  std::vector<double> S((size_t)n * n), T((size_t)n * n), V((size_t)n * n), H((size_t)n * n);
  rc = iqcp_one_electron(ctx, S.data(), T.data(), V.data());
  std::vector<double> eri;
  if (!rc && z >= 2) {
    const long long np = (long long)n * (n + 1) / 2;
    eri.resize((size_t)(np * (np + 1) / 2));
    rc = iqcp_eri_compressed(ctx, eri.data(), (long long)eri.size());
  }
  iqcp_destroy(ctx);
  if (rc) return rc;
  for (size_t i = 0; i < H.size(); ++i) H[i] = T[i] + V[i];
  const std::vector<LGroup> groups = l_groups(sl);
  int cfg[3];
  electron_config(z, cfg);
  Da = sph_avg_density(n, H, S, groups, cfg);
  if (z <= 1) return 0;
  double e_old = HUGE_VAL;
  for (int it = 0; it < 40; ++it) {
    std::vector<double> F = H;
    for (int m = 0; m < n; ++m)
      for (int v = 0; v <= m; ++v) {
        double g = 0.0;
        for (int l = 0; l < n; ++l)
          for (int s = 0; s < n; ++s) {
            const double d = Da[(size_t)l * n + s];
            if (std::fabs(d) < 1e-15) continue;
            const double jv = eri[(size_t)pidx(pidx(m, v), pidx(l, s))];
            const double kv = eri[(size_t)pidx(pidx(m, l), pidx(v, s))];
            g += d * (jv - 0.5 * kv);
          }
        F[(size_t)m * n + v] += g;
        if (m != v) F[(size_t)v * n + m] += g;
      }
    double e = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) e += Da[(size_t)i * n + j] * (H[(size_t)j * n + i] + F[(size_t)j * n + i]);
    e *= 0.5;
    if (std::fabs(e - e_old) < 1e-10) break;
    e_old = e;
    Da = sph_avg_density(n, F, S, groups, cfg);
  }
  return 0;
}

// Atomic blocks already computed in this process, keyed by the element and
// its shells (l, primitive count, exponents, coefficients): a batch of
// geometries in one basis computes each element once.
struct AtomKey {
  int z;
  std::vector<int> shape;
  std::vector<double> prims;
  bool operator<(const AtomKey& o) const {
    if (z != o.z) return z < o.z;
    if (shape != o.shape) return shape < o.shape;
    return prims < o.prims;
  }
};
std::mutex g_atom_mu;
std::map<AtomKey, std::vector<double>> g_atom_cache;

}  // namespace

extern "C" int iqcp_sad_density(const iqcp_basis_desc* basis, const iqcp_options* opts, double* D) {
  if (!basis || !D || basis->n_shells <= 0 || basis->n_atoms <= 0) return IQCP_ERR_ARG;
  const int ns = basis->n_shells, na = basis->n_atoms;
  std::vector<int> off(ns + 1, 0), pstart(ns + 1, 0);
  for (int s = 0; s < ns; ++s) {
    if (basis->l[s] < 0 || basis->l[s] > 2 || basis->atom_of_shell[s] < 0 || basis->atom_of_shell[s] >= na)
      return IQCP_ERR_ARG;
    off[s + 1] = off[s] + ncart(basis->l[s]);
    pstart[s + 1] = pstart[s] + basis->nprim[s];
  }
  const int nbf = off[ns];
  std::memset(D, 0, sizeof(double) * (size_t)nbf * nbf);
  iqcp_options o;
  if (opts) o = *opts;
  else iqcp_default_options(&o);
  o.precision = IQCP_FP64;
  std::map<int, std::vector<double>> cache;  // per element (sad.rs:722-737)
  for (int a = 0; a < na; ++a) {
    std::vector<int> sh;
    for (int s = 0; s < ns; ++s)
      if (basis->atom_of_shell[s] == a) sh.push_back(s);
    if (sh.empty()) continue;
    const int z = basis->z[a];
    auto it = cache.find(z);
    if (it == cache.end()) {
      // one-atom basis: this atom's shells at its own position
      std::vector<int> l1, np1, at1;
      std::vector<double> c1, e1, k1;
      for (int s : sh) {
        l1.push_back(basis->l[s]);
        np1.push_back(basis->nprim[s]);
        at1.push_back(0);
        for (int x = 0; x < 3; ++x) c1.push_back(basis->atom_xyz[3 * a + x]);
        for (int p = pstart[s]; p < pstart[s + 1]; ++p) {
          e1.push_back(basis->exps[p]);
          k1.push_back(basis->coefs[p]);
        }
      }
      const int z1[1] = {z};
      iqcp_basis_desc one{(int)sh.size(), 1, l1.data(), np1.data(), at1.data(), c1.data(),
                          e1.data(),      k1.data(), basis->atom_xyz + 3 * a, z1};
      AtomKey key{z, {}, e1};
      key.prims.insert(key.prims.end(), k1.begin(), k1.end());
      for (size_t i = 0; i < l1.size(); ++i) {
        key.shape.push_back(l1[i]);
        key.shape.push_back(np1[i]);
      }
      std::vector<double> Da;
      {
        std::lock_guard<std::mutex> lock(g_atom_mu);
        auto hit = g_atom_cache.find(key);
        if (hit != g_atom_cache.end()) Da = hit->second;
      }
      if (Da.empty()) {
        const int rc = atomic_density(z, one, &o, Da);
        if (rc) return rc;
        std::lock_guard<std::mutex> lock(g_atom_mu);
        g_atom_cache.emplace(key, Da);
      }
      it = cache.emplace(z, std::move(Da)).first;
    }
    const std::vector<double>& Da = it->second;
    std::vector<int> gbf;  // atomic function -> molecular function
    for (int s : sh)
      for (int c = 0; c < ncart(basis->l[s]); ++c) gbf.push_back(off[s] + c);
    const int n = (int)gbf.size();
    if ((size_t)n * n != Da.size()) return IQCP_ERR_ARG;  // same element, different shells
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) D[(size_t)gbf[i] * nbf + gbf[j]] = Da[(size_t)i * n + j];
  }
  return IQCP_OK;
}
