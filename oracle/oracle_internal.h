// CPU oracle: TEST INFRASTRUCTURE ONLY.
//
// A plain C++ restatement of the reference's FP64 Fock-build / ERI-gradient
// path (ExaPsi/IQCP, crates/qc-core).  Only the test-suite, the smoke check and
// the CPU-baseline leg of the benchmark load it, as the checker.  The product
// library (iqcp_b200/libiqcp_gpu.so) never links or calls anything here.
//
// Compiled with -ffp-contract=off so that every a*b+c is rounded twice, as
// rustc does by default; libm's exp/sqrt are the same glibc routines the
// reference's native build calls.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

namespace oracle {

constexpr int kMaxRoots = 10;       // rys/mod.rs:46 MAX_ROOTS

// ---- Boys / Rys (boys/mod.rs, rys/mod.rs) ---------------------------------
void boys_all(int m_max, double t, double* f);                   // boys/mod.rs:587
// Returns 0 on success, a negative code on RysError (rys/mod.rs:84-118).
int rys_roots(int nroots, double t, double* roots, double* weights);  // rys/mod.rs:253
// Working precision of rys_roots for the whole process: 0 = double, the
// reference's arithmetic (default); 1 = the same algorithm in long double,
// rounded to double at the end (a more accurate reading for diagnostics).
void set_root_precision(int extended);
int root_precision();

// ---- basis ------------------------------------------------------------------
struct Shell {
  int l;
  int atom;
  double center[3];
  std::vector<double> exps, coefs;
};

struct Basis {
  std::vector<Shell> shells;
  std::vector<int> offsets;   // first basis function of each shell
  int nbf = 0;
  int natoms = 0;
  std::vector<double> atom_xyz;
  std::vector<int> atom_z;
};

Basis make_basis(int n_shells, const int* l, const int* nprim, const int* atom_of_shell,
                 const double* center, const double* exps, const double* coefs,
                 int natoms, const double* atom_xyz, const int* z);

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }
// Cartesian powers in reference order (integrals/cartesian.rs:113-136)
void cart_powers(int l, int idx, int pw[3]);
double cart_norm(double alpha, const int pw[3]);                 // overlap.rs:343

// ---- ERI ----------------------------------------------------------------------
struct EriCounters {
  long long rys_failures = 0;        // primitive quartets dropped by a RysError
  long long t_zero_fallbacks = 0;    // ... of which re-done through the T=0 path
  long long prim_quartets = 0;       // surviving primitive quartets
};

// (ij|kl) block, row-major (i,j,k,l) -- eri/mod.rs:458-854
void shell_eri(const Shell& a, const Shell& b, const Shell& c, const Shell& d,
               double* out, EriCounters* cnt);
// 13 blocks: [0] integrals, [1 + 3*centre + dir] derivatives -- eri/mod.rs:2035-2548
void shell_eri_deriv(const Shell& a, const Shell& b, const Shell& c, const Shell& d,
                     double* out13, EriCounters* cnt);
// Q_ij = sqrt(max|(ij|ij)|) -- eri/mod.rs:1263
std::vector<double> schwarz_bounds(const Basis& bs);

constexpr double kSchwarzThreshold = 1e-12;  // eri/mod.rs:1258

}  // namespace oracle
