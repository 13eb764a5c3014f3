// CPU oracle (TEST INFRASTRUCTURE ONLY): flat C entry points for ctypes.
// Matrices are row-major nbf x nbf; the basis is passed as plain shell arrays.
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle_internal.h"

namespace oracle {
void eri_compressed(const Basis& bs, double* eri, EriCounters* cnt);
void build_fock(int nbf, const double* H, const double* D, const double* eri, double* F);
void build_jk_stored(int nbf, const double* D, const double* eri, double* J, double* K);
void jk_direct(const Basis& bs, const double* D, double* J, double* K, int stride, int phase,
               EriCounters* cnt, long long* nq);
void eri_gradient(const Basis& bs, const double* D, double hf_frac, double* grad, int stride,
                  int phase, EriCounters* cnt);
void one_electron(const Basis& bs, int kind, double* out);
void one_electron_gradient(const Basis& bs, const double* D, const double* W, double* grad);
double nuclear_repulsion(const Basis& bs);
}  // namespace oracle

using namespace oracle;

#define BASIS_ARGS                                                                          \
  int n_shells, const int *l, const int *nprim, const int *atom_of_shell, const double *center, \
      const double *exps, const double *coefs, int natoms, const double *atom_xyz, const int *z
#define MAKE_BASIS \
  make_basis(n_shells, l, nprim, atom_of_shell, center, exps, coefs, natoms, atom_xyz, z)

extern "C" {

void or_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#endif
}

int or_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void or_boys_all(int m_max, double t, double* f) { boys_all(m_max, t, f); }

void or_set_root_precision(int extended) { set_root_precision(extended); }
int or_root_precision() { return root_precision(); }
int or_rys_roots(int n, double t, double* roots, double* weights) {
  return rys_roots(n, t, roots, weights);
}

double or_cart_norm(double alpha, int i, int j, int k) {
  const int pw[3] = {i, j, k};
  return cart_norm(alpha, pw);
}

// counters[3]: rys failures, T=0 fallbacks, surviving primitive quartets
void or_shell_eri(BASIS_ARGS, int si, int sj, int sk, int sl, double* out, long long* counters) {
  Basis bs = MAKE_BASIS;
  EriCounters c;
  shell_eri(bs.shells[si], bs.shells[sj], bs.shells[sk], bs.shells[sl], out, &c);
  if (counters) { counters[0] = c.rys_failures; counters[1] = c.t_zero_fallbacks; counters[2] = c.prim_quartets; }
}

void or_shell_eri_deriv(BASIS_ARGS, int si, int sj, int sk, int sl, double* out13) {
  Basis bs = MAKE_BASIS;
  shell_eri_deriv(bs.shells[si], bs.shells[sj], bs.shells[sk], bs.shells[sl], out13, nullptr);
}

void or_schwarz(BASIS_ARGS, double* q) {
  Basis bs = MAKE_BASIS;
  std::vector<double> v = schwarz_bounds(bs);
  std::memcpy(q, v.data(), sizeof(double) * v.size());
}

void or_eri_compressed(BASIS_ARGS, double* eri, long long* counters) {
  Basis bs = MAKE_BASIS;
  EriCounters c;
  eri_compressed(bs, eri, &c);
  if (counters) { counters[0] = c.rys_failures; counters[1] = c.t_zero_fallbacks; counters[2] = c.prim_quartets; }
}

void or_build_fock(int nbf, const double* H, const double* D, const double* eri, double* F) {
  build_fock(nbf, H, D, eri, F);
}

void or_build_jk_stored(int nbf, const double* D, const double* eri, double* J, double* K) {
  build_jk_stored(nbf, D, eri, J, K);
}

// counters[4]: rys failures, T=0 fallbacks, primitive quartets, shell quartets
void or_jk_direct(BASIS_ARGS, const double* D, double* J, double* K, int stride, int phase,
                  long long* counters) {
  Basis bs = MAKE_BASIS;
  EriCounters c;
  long long nq = 0;
  jk_direct(bs, D, J, K, stride, phase, &c, &nq);
  if (counters) { counters[0] = c.rys_failures; counters[1] = c.t_zero_fallbacks; counters[2] = c.prim_quartets; counters[3] = nq; }
}

void or_eri_gradient(BASIS_ARGS, const double* D, double hf_frac, double* grad, int stride,
                     int phase, long long* counters) {
  Basis bs = MAKE_BASIS;
  EriCounters c;
  std::memset(grad, 0, sizeof(double) * 3 * natoms);
  eri_gradient(bs, D, hf_frac, grad, stride, phase, &c);
  if (counters) { counters[0] = c.rys_failures; counters[1] = c.t_zero_fallbacks; counters[2] = c.prim_quartets; }
}

// kind: 0 overlap, 1 kinetic, 2 nuclear attraction
void or_one_electron(BASIS_ARGS, int kind, double* out) {
  Basis bs = MAKE_BASIS;
  one_electron(bs, kind, out);
}

void or_one_electron_gradient(BASIS_ARGS, const double* D, const double* W, double* grad) {
  Basis bs = MAKE_BASIS;
  one_electron_gradient(bs, D, W, grad);
}

double or_nuclear_repulsion(BASIS_ARGS) {
  Basis bs = MAKE_BASIS;
  return nuclear_repulsion(bs);
}

}  // extern "C"
