// Host runtime of libiqcp_gpu.so: basis construction from the built-in
// tables, per-geometry shell-pair tables and screened quartet work lists in
// HBM, and the extern "C" entry points declared in include/iqcp.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/iqcp.h"
#include "engine.cuh"
#include "internal.h"

#include "basis_tables.inc"

using namespace iqcp;

namespace {

struct ClassList {
  std::vector<int> pairs;   // ShellPair ids sorted by Q descending
};

struct TaskRange {
  int X, Y;
  int first, count;         // into the task array
  long long quartets;       // screened shell quartets in the range
  int mode[2];              // kernel variant for J/K [0] and gradient [1]
  int mode32[2];            // the same for the FP32 share of a mixed call
  int split[2];             // mixed form: 1 = FP64 + FP32 passes, 0 = the whole class in FP64
};

}  // namespace

struct iqcp_ctx {
  std::string err;
  int device = 0;
  iqcp_options opt;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  int nbf = 0, n_shells = 0, n_atoms = 0;   // totals over the molecules of the context
  // batched contexts: molecule m owns rows/cols [0, mol_nbf[m]) of the block at
  // mol_base[m] in every packed matrix (D, J, K, F, H, S) and atoms
  // [mol_atom0[m], mol_atom0[m+1]) of the gradient
  int n_mol = 1;
  std::vector<long long> mol_base;
  std::vector<int> mol_nbf, mol_bf0, mol_atom0, mol_shell0;
  long long packed = 0;
  long long* d_mol_base = nullptr;
  int* d_mol_n = nullptr;
  int* d_mol_bf0 = nullptr;
  Packing pack{};
  std::vector<int> shell_l, shell_off, shell_atom;
  // device tables
  ShellPair* d_pairs = nullptr;
  PrimPair* d_pp = nullptr;
  int* d_ket_list = nullptr;      // class lists concatenated
  QuartetTask* d_tasks = nullptr;
  double* d_ang = nullptr;        // per basis function angular factor
  double* d_Ds = nullptr;         // scaled density
  double* d_Jt = nullptr;
  double* d_Kt = nullptr;
  double* d_io[4] = {nullptr, nullptr, nullptr, nullptr};  // staging for host-buffer calls
  double* d_grad = nullptr;
  // mixed precision: per shell-block max |D| of every molecule (ns_m x ns_m
  // at d_dbase[m]), the FP32 quartet counter and the per-task FP32 masks
  double* d_dmax = nullptr;
  long long* d_dbase = nullptr;
  int* d_mol_shell0 = nullptr;
  int* d_mol_ns = nullptr;
  long long dmax_total = 0;
  unsigned long long* d_fp32 = nullptr;
  unsigned* d_mask = nullptr;
  int n_tasks = 0;
  int* d_counters = nullptr;      // one work counter per class range, kind and pass
  int* cur_counter = nullptr;
  bool mixed_call = false;
  bool in_capture = false;        // the last call was enqueued into a CUDA graph capture
  // basis copy for the one-electron kernel
  int* d_bint = nullptr;          // l | nprim | pstart | off | z | atom (per shell, molecule-local)
  double* d_bdbl = nullptr;       // center | exps | coefs | atom_xyz
  int n_prims = 0;
  // host copies
  std::vector<ShellPair> pairs;
  std::vector<int> list_offset;   // per class, into d_ket_list
  std::vector<ClassList> classes;
  std::vector<TaskRange> ranges;
  long long n_quartets = 0;
  double stats[4] = {0, 0, 0, 0};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // class launches run concurrently on the context stream and these side
  // streams (forked and joined with events), so one class's tail overlaps
  // the next class's start
  static constexpr int kSide = 3;
  cudaStream_t side[kSide] = {nullptr, nullptr, nullptr};
  cudaEvent_t fork_ev = nullptr, join_ev[kSide] = {nullptr, nullptr, nullptr};
  // per-launch timing of the quartet kernels (off unless requested)
  bool profile = false;
  std::vector<cudaEvent_t> pev;
  // kind: 0 J/K, 1 gradient, 2 / 3 their FP32 share in a mixed call
  struct LaunchRec { int kind, X, Y; float ms; long long quartets; int ev; };
  std::vector<LaunchRec> launch_log;
  int launches_total = 0;       // every kernel of the last call
  // surviving primitive quartets per task range (counted on first request)
  std::vector<long long> prim_quartets;
  // multi-density J/K: scaled densities and accumulators of nset densities
  // (grown on demand), and host-call staging of the inputs and outputs
  double* d_multi = nullptr;
  long long multi_cap = 0;      // doubles
  double* d_multi_io = nullptr;
  long long multi_io_cap = 0;   // doubles
  // spherical basis (single geometry): per Cartesian function {sph offset of
  // its shell, position in the shell, l}, per spherical function {Cartesian
  // offset of its shell, m index, l}; built on first use
  int nsph = 0;
  int* d_cart_info = nullptr;
  int* d_sph_info = nullptr;
  // batched SCF: per-molecule flags of the geometries still iterating (device,
  // owned by the SCF call; null = every molecule)
  const int* mol_active = nullptr;
  // host copies of the atoms (nuclear repulsion of the batched SCF)
  std::vector<int> atom_z;
  std::vector<double> atom_xyz;
};

namespace {

int fail(iqcp_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(ctx, IQCP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
  } while (0)

double rad_norm(double a, int l) {
  // (2a/pi)^{3/4} (4a)^{l/2}, the alpha-dependent part of overlap.rs:343
  const double tap = 2.0 * a / M_PI;
  double v = std::sqrt(std::sqrt(tap * tap * tap));
  const double fa = 4.0 * a;
  if (l == 1) v *= std::sqrt(fa);
  else if (l == 2) v *= fa;
  return v;
}

double ang_host(int l, int c) {
  return (l == 2 && (c == 0 || c == 3 || c == 5)) ? 1.0 / std::sqrt(3.0) : 1.0;
}

int basis_id(const char* name) {
  std::string s;
  for (const char* p = name; *p; ++p) {
    const char ch = (char)std::tolower((unsigned char)*p);
    if (ch != ' ' && ch != '_') s.push_back(ch);
  }
  if (s == "sto-3g" || s == "sto3g") return 0;
  if (s == "3-21g" || s == "321g") return 1;
  if (s == "6-31g" || s == "631g") return 2;
  if (s == "6-31g*" || s == "631g*" || s == "6-31gs" || s == "631gs" || s == "6-31g(d)" || s == "631g(d)") return 3;
  if (s == "6-31+g*" || s == "631+g*" || s == "6-31+gs" || s == "631+gs" || s == "6-31+g(d)" || s == "631+g(d)") return 4;
  if (s == "cc-pvdz" || s == "ccpvdz") return 5;
  return -1;
}

// Build class lists and quartet tasks from Schwarz bounds held in ctx->pairs.
// Per molecule, each class list is split into buckets of equal primitive-pair
// count (so the 32 kets of a warp share one primitive-loop length), each
// bucket sorted by Q descending so that the Schwarz test Q_bra * Q_ket >= thr
// keeps a prefix of it.  Unique quartets of a class with itself keep ket
// position <= bra position.  Tasks never mix molecules; the tasks of one class
// pair over all molecules form one range (one launch).
void build_tasks(iqcp_ctx* ctx, std::vector<int>& ket_list, std::vector<QuartetTask>& tasks) {
  const double thr = ctx->opt.schwarz_threshold;
  const int NC = kNumPairClasses;
  std::vector<std::vector<int>> lists((size_t)ctx->n_mol * NC);
  for (int i = 0; i < (int)ctx->pairs.size(); ++i) {
    const ShellPair& p = ctx->pairs[i];
    lists[(size_t)p.mol * NC + pair_class(ctx->shell_l[p.sa], ctx->shell_l[p.sb])].push_back(i);
  }
  std::vector<int> seg((size_t)ctx->n_mol * NC);
  std::vector<std::vector<std::pair<int, int>>> buckets((size_t)ctx->n_mol * NC);
  ket_list.clear();
  for (size_t li = 0; li < lists.size(); ++li) {
    auto& v = lists[li];
    std::stable_sort(v.begin(), v.end(), [&](int a, int b) {
      const ShellPair &pa = ctx->pairs[a], &pb = ctx->pairs[b];
      if (pa.np != pb.np) return pa.np > pb.np;
      return pa.Q > pb.Q;
    });
    for (size_t s0 = 0; s0 < v.size();) {
      size_t e0 = s0;
      while (e0 < v.size() && ctx->pairs[v[e0]].np == ctx->pairs[v[s0]].np) ++e0;
      buckets[li].push_back({(int)s0, (int)e0});
      s0 = e0;
    }
    seg[li] = (int)ket_list.size();
    ket_list.insert(ket_list.end(), v.begin(), v.end());
  }
  tasks.clear();
  ctx->ranges.clear();
  ctx->n_quartets = 0;
  for (int X = 0; X < NC; ++X)
    for (int Y = 0; Y <= X; ++Y) {
      TaskRange r{X, Y, (int)tasks.size(), 0, 0, {default_mode(X, Y, 0), default_mode(X, Y, 1)},
                  {default_mode(X, Y, 0), default_mode(X, Y, 1)}, {1, 1}};
      for (int m = 0; m < ctx->n_mol; ++m) {
        const size_t lx = (size_t)m * NC + X, ly = (size_t)m * NC + Y;
        const auto& LX = lists[lx];
        const auto& LY = lists[ly];
        for (int b = 0; b < (int)LX.size(); ++b) {
          const double qb = ctx->pairs[LX[b]].Q;
          for (const auto& bk : buckets[ly]) {
            if (X == Y && bk.first > b) break;
            const int hi_pos = (X == Y) ? std::min(bk.second, b + 1) : bk.second;
            int lo = bk.first, hi = hi_pos;   // prefix of the bucket with qb * qk >= thr
            while (lo < hi) {
              const int mid = (lo + hi) / 2;
              if (qb * ctx->pairs[LY[mid]].Q < thr) hi = mid; else lo = mid + 1;
            }
            const int nk = lo - bk.first;
            ctx->n_quartets += nk;
            r.quartets += nk;
            for (int k0 = 0; k0 < nk; k0 += 32) {
              QuartetTask t;
              t.bra = LX[b];
              t.ket0 = seg[ly] + bk.first + k0;
              t.nket = std::min(32, nk - k0);
              t.diag = (X == Y) ? 1 : 0;
              t.bra_pos = seg[lx] + b;
              t.flags = 0;
              tasks.push_back(t);
            }
          }
        }
      }
      r.count = (int)tasks.size() - r.first;
      ctx->ranges.push_back(r);
    }
}

int ensure_device(iqcp_ctx* ctx) {
  CK(cudaSetDevice(ctx->device));
  return IQCP_OK;
}

int ensure_profile_events(iqcp_ctx* ctx) {
  const size_t need = 4 * ctx->ranges.size();
  while (ctx->pev.size() < need) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    ctx->pev.push_back(e);
  }
  return IQCP_OK;
}

Mixed mixed_args(const iqcp_ctx* ctx, int pass) {
  Mixed m;
  m.dmax = ctx->d_dmax;
  m.dbase = ctx->d_dbase;
  m.shell0 = ctx->d_mol_shell0;
  m.ns = ctx->d_mol_ns;
  m.cutoff = ctx->opt.mixed_cutoff;
  m.pass = pass;
  m.fp32_count = pass == 2 ? ctx->d_fp32 : nullptr;
  m.mask = ctx->d_mask;
  return m;
}

JKArgs jk_args(const iqcp_ctx* ctx, const TaskRange& r, const double* Ds, double* Jt, double* Kt, int mode,
               int pass, int* counter) {
  JKArgs a;
  a.pairs = ctx->d_pairs;
  a.pp = ctx->d_pp;
  a.ket_list = ctx->d_ket_list;
  a.tasks = ctx->d_tasks + r.first;
  a.ntasks = r.count;
  a.D = Ds;
  a.nbf = ctx->nbf;
  a.J = Jt;
  a.K = Kt;
  a.prim_thr = ctx->opt.prim_threshold;
  a.mode = mode;
  a.mx = mixed_args(ctx, pass);
  a.mx.mask = ctx->d_mask + r.first;
  a.next_task = counter;
  a.mol_base = ctx->d_mol_base;
  a.mol_n = ctx->d_mol_n;
  a.nset = 1;
  a.set_stride = 0;
  a.mol_active = ctx->mol_active;
  return a;
}

GradArgs grad_args(const iqcp_ctx* ctx, const TaskRange& r, const double* Ds, double xscale, double* grad,
                   int mode, int pass, int* counter) {
  GradArgs a;
  a.pairs = ctx->d_pairs;
  a.pp = ctx->d_pp;
  a.ket_list = ctx->d_ket_list;
  a.tasks = ctx->d_tasks + r.first;
  a.ntasks = r.count;
  a.D = Ds;
  a.nbf = ctx->nbf;
  a.xscale = xscale;
  a.grad = grad;
  a.prim_thr = ctx->opt.prim_threshold;
  a.schwarz_thr = ctx->opt.schwarz_threshold;
  a.natoms = ctx->n_atoms;
  a.gsmem = ctx->n_atoms <= 2048 ? 1 : 0;
  a.mode = mode;
  a.mx = mixed_args(ctx, pass);
  a.mx.mask = ctx->d_mask + r.first;
  a.next_task = counter;
  a.mol_base = ctx->d_mol_base;
  a.mol_n = ctx->d_mol_n;
  return a;
}

// Mixed form for density dD (unscaled): per-shell-block density bound, then
// the FP32 mask of every task (kind 0 J/K, 1 gradient)
int prepare_mixed(iqcp_ctx* ctx, const double* dD, int kind) {
  CK(launch_shell_dmax(dD, ctx->pack, ctx->d_bint + 3 * ctx->n_shells, ctx->d_bint, mixed_args(ctx, 0),
                       ctx->dmax_total, ctx->d_dmax, ctx->stream));
  CK(launch_precision_masks(ctx->d_pairs, ctx->d_ket_list, ctx->d_tasks, ctx->n_tasks, mixed_args(ctx, 1),
                            kind == 1, ctx->d_mask, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_fp32, 0, sizeof(unsigned long long), ctx->stream));
  ctx->launches_total += 2;
  return IQCP_OK;
}

// True while the context stream is being captured into a CUDA graph: the
// device entry points then only enqueue work (no timing events, no stats read
// back, no host synchronisation).
bool capturing(const iqcp_ctx* ctx) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(ctx->stream, &st) != cudaSuccess) return false;
  return st != cudaStreamCaptureStatusNone;
}

// Launch the quartet kernels of every non-empty class range; kind 0 = J/K,
// 1 = gradient.  In a mixed call a class whose split flag is set launches
// twice, pass 1 (FP64 share) then pass 2 (FP32 share); launch(r, pass,
// counter, stream) issues one launch.  Launches go round-robin to the context
// stream and the side streams, forked after the counters' reset and joined
// before the end event: each launch has its own work counter and every
// kernel adds its results atomically, so they may overlap (a persistent
// kernel's blocks start on the SMs that the previous one's tail frees).
template <typename F>
int run_ranges(iqcp_ctx* ctx, int kind, F&& launch) {
  ctx->in_capture = capturing(ctx);
  const bool prof = ctx->profile && !ctx->in_capture;
  if (prof) {
    int rc = ensure_profile_events(ctx);
    if (rc) return rc;
  }
  const size_t nr = ctx->ranges.size();
  ctx->launch_log.clear();
  CK(cudaMemsetAsync(ctx->d_counters + 2 * kind * nr, 0, sizeof(int) * 2 * nr, ctx->stream));
  if (!ctx->in_capture) CK(cudaEventRecord(ctx->ev0, ctx->stream));
  // with per-launch profiling on, the launches stay on the context stream so
  // that each launch's events time it alone
  const int nst = prof ? 1 : 1 + iqcp_ctx::kSide;
  cudaStream_t streams[1 + iqcp_ctx::kSide] = {ctx->stream};
  if (nst > 1) {
    CK(cudaEventRecord(ctx->fork_ev, ctx->stream));
    for (int s = 0; s < iqcp_ctx::kSide; ++s) {
      streams[1 + s] = ctx->side[s];
      CK(cudaStreamWaitEvent(ctx->side[s], ctx->fork_ev, 0));
    }
  }
  int launches = 0;
  for (size_t i = 0; i < nr; ++i) {
    const TaskRange& r = ctx->ranges[i];
    if (r.count == 0) continue;
    const bool split = ctx->mixed_call && r.split[kind];
    for (int ps = 0; ps < (split ? 2 : 1); ++ps) {
      const int pass = split ? ps + 1 : 0;
      const int ev = int(2 * (2 * i + ps));
      cudaStream_t st = streams[launches % nst];
      if (prof) CK(cudaEventRecord(ctx->pev[ev], st));
      CK(launch(r, pass, ctx->d_counters + (2 * kind + ps) * nr + i, st));
      if (prof) CK(cudaEventRecord(ctx->pev[ev + 1], st));
      ++launches;
      ctx->launch_log.push_back({kind + (pass == 2 ? 2 : 0), r.X, r.Y, 0.f, pass == 2 ? 0 : r.quartets, ev});
    }
  }
  for (int s = 0; nst > 1 && s < iqcp_ctx::kSide; ++s) {
    CK(cudaEventRecord(ctx->join_ev[s], ctx->side[s]));
    CK(cudaStreamWaitEvent(ctx->stream, ctx->join_ev[s], 0));
  }
  if (!ctx->in_capture) CK(cudaEventRecord(ctx->ev1, ctx->stream));
  ctx->stats[0] = (double)ctx->n_quartets;
  ctx->stats[1] = launches;
  ctx->launches_total += launches;
  return IQCP_OK;
}

int run_jk_device(iqcp_ctx* ctx, const double* dD, bool want_k) {
  const size_t bytes = sizeof(double) * (size_t)ctx->packed;
  ctx->launches_total = 1;
  CK(launch_scale_density(dD, ctx->d_ang, ctx->pack, ctx->d_Ds, ctx->stream));
  ctx->mixed_call = ctx->opt.precision == IQCP_MIXED;
  if (ctx->mixed_call) {
    int rc = prepare_mixed(ctx, dD, 0);
    if (rc) return rc;
  }
  CK(cudaMemsetAsync(ctx->d_Jt, 0, bytes, ctx->stream));
  if (want_k) CK(cudaMemsetAsync(ctx->d_Kt, 0, bytes, ctx->stream));
  return run_ranges(ctx, 0, [&](const TaskRange& r, int pass, int* counter, cudaStream_t st) {
    const JKArgs a = jk_args(ctx, r, ctx->d_Ds, ctx->d_Jt, want_k ? ctx->d_Kt : nullptr,
                             pass == 2 ? r.mode32[0] : r.mode[0], pass, counter);
    return launch_jk(r.X, r.Y, a, st);
  });
}

int finish_stats(iqcp_ctx* ctx) {
  if (ctx->in_capture) return IQCP_OK;
  float ms = 0.f;
  CK(cudaEventSynchronize(ctx->ev1));
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ctx->stats[2] = ms * 1e3;
  ctx->stats[3] = 0.0;
  if (ctx->mixed_call) {
    unsigned long long c = 0;
    CK(cudaMemcpyAsync(&c, ctx->d_fp32, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->stats[3] = (double)c;
  }
  if (ctx->profile) {
    for (auto& rec : ctx->launch_log) {
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, ctx->pev[rec.ev], ctx->pev[rec.ev + 1]));
      rec.ms = t;
    }
  }
  return IQCP_OK;
}

}  // namespace

// Accessors for the other translation units of the library (internal.h).
namespace iqcp {
cudaStream_t ctx_stream(const iqcp_ctx* c) { return c->stream; }
int ctx_fail(iqcp_ctx* c, int code, const char* msg) { return fail(c, code, msg); }
int ctx_device(const iqcp_ctx* c) { return c->device; }
int ctx_n_mol(const iqcp_ctx* c) { return c->n_mol; }
const Packing& ctx_packing(const iqcp_ctx* c) { return c->pack; }
const std::vector<long long>& ctx_mol_base(const iqcp_ctx* c) { return c->mol_base; }
const std::vector<int>& ctx_mol_nbf(const iqcp_ctx* c) { return c->mol_nbf; }
const std::vector<int>& ctx_mol_atom0(const iqcp_ctx* c) { return c->mol_atom0; }
const std::vector<int>& ctx_atom_z(const iqcp_ctx* c) { return c->atom_z; }
const std::vector<double>& ctx_atom_xyz(const iqcp_ctx* c) { return c->atom_xyz; }
void ctx_set_mol_active(iqcp_ctx* c, const int* d_flags) { c->mol_active = d_flags; }
}  // namespace iqcp

extern "C" {

void iqcp_default_options(iqcp_options* o) {
  o->schwarz_threshold = 1e-12;
  o->prim_threshold = 1e-15;
  o->precision = IQCP_FP64;
  o->mixed_cutoff = 1e-9;
  o->device = 0;
}

int iqcp_basis_build(const char* basis_name, int n_atoms, const int* z, const double* xyz,
                     int* n_shells, int* n_prims, int* nbf, int* l, int* nprim, int* atom_of_shell,
                     double* center, double* exps, double* coefs) {
  if (!basis_name || n_atoms <= 0 || !z || !xyz) return IQCP_ERR_ARG;
  const int bid = basis_id(basis_name);
  if (bid < 0) return IQCP_ERR_BASIS;
  int ns = 0, np = 0, nb = 0;
  for (int a = 0; a < n_atoms; ++a) {
    if (z[a] < 1 || z[a] > 18) return IQCP_ERR_BASIS;
    for (int r = 0; r < kNumShellRecords; ++r) {
      const int* rec = kShellRecords[r];
      if (rec[0] != bid || rec[1] != z[a]) continue;
      if (l) {
        l[ns] = rec[2];
        nprim[ns] = rec[3];
        atom_of_shell[ns] = a;
        for (int d = 0; d < 3; ++d) center[3 * ns + d] = xyz[3 * a + d];
        for (int k = 0; k < rec[3]; ++k) {
          exps[np + k] = kPrimitives[rec[4] + k][0];
          coefs[np + k] = kPrimitives[rec[4] + k][1];
        }
      }
      ++ns;
      np += rec[3];
      nb += ncart(rec[2]);
    }
  }
  if (n_shells) *n_shells = ns;
  if (n_prims) *n_prims = np;
  if (nbf) *nbf = nb;
  return IQCP_OK;
}

const char* iqcp_last_error(const iqcp_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }
int iqcp_nbf(const iqcp_ctx* ctx) { return ctx ? ctx->nbf : 0; }

static int create_batch(int nmol, const iqcp_basis_desc* descs, const iqcp_options* opts, iqcp_ctx** out) {
  if (!descs || !out || nmol <= 0) return IQCP_ERR_ARG;
  for (int m = 0; m < nmol; ++m)
    if (descs[m].n_shells <= 0 || descs[m].n_atoms <= 0) return IQCP_ERR_ARG;
  iqcp_ctx* ctx = new iqcp_ctx();
  *out = ctx;
  if (opts) ctx->opt = *opts;
  else iqcp_default_options(&ctx->opt);
  ctx->device = ctx->opt.device;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= ctx->device)
    return fail(ctx, IQCP_ERR_NODEVICE, "no CUDA device available");
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, ctx->device));
  if (prop.major != 10) return fail(ctx, IQCP_ERR_NODEVICE, "libiqcp_gpu is built for sm_100a only");
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking));
  ctx->stream = ctx->own_stream;
  CK(cudaEventCreate(&ctx->ev0));
  CK(cudaEventCreate(&ctx->ev1));
  CK(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming));
  for (int s = 0; s < iqcp_ctx::kSide; ++s) {
    CK(cudaStreamCreateWithFlags(&ctx->side[s], cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&ctx->join_ev[s], cudaEventDisableTiming));
  }
  ctx->n_mol = nmol;
  const double kthr = ctx->opt.prim_threshold;

  // concatenate the molecules: global shell, atom, primitive and basis-function
  // numbering; basis offsets inside a pair stay local to its molecule block
  std::vector<int> bl, bnp, bps, boff, bz, bat;
  std::vector<double> bc, bex, bco, bxyz, ang;
  std::vector<PrimPair> pps;
  long long base = 0;
  for (int m = 0; m < nmol; ++m) {
    const iqcp_basis_desc* b = descs + m;
    const int s0 = ctx->n_shells, a0 = ctx->n_atoms, p0 = (int)bex.size();
    ctx->mol_shell0.push_back(s0);
    ctx->mol_atom0.push_back(a0);
    ctx->mol_bf0.push_back(ctx->nbf);
    std::vector<int> pstart(b->n_shells + 1, 0);
    int off = 0;
    for (int s = 0; s < b->n_shells; ++s) {
      if (b->l[s] < 0 || b->l[s] > kMaxL) return fail(ctx, IQCP_ERR_ARG, "angular momentum above d");
      if (b->nprim[s] <= 0) return fail(ctx, IQCP_ERR_ARG, "shell without primitives");
      if (b->atom_of_shell[s] < 0 || b->atom_of_shell[s] >= b->n_atoms)
        return fail(ctx, IQCP_ERR_ARG, "bad atom index");
      for (int d = 0; d < 3; ++d)
        if (!std::isfinite(b->center[3 * s + d])) return fail(ctx, IQCP_ERR_NUMERIC, "non-finite shell centre");
      ctx->shell_l.push_back(b->l[s]);
      ctx->shell_off.push_back(off);
      ctx->shell_atom.push_back(a0 + b->atom_of_shell[s]);
      for (int c = 0; c < ncart(b->l[s]); ++c) ang.push_back(ang_host(b->l[s], c));
      bl.push_back(b->l[s]);
      bat.push_back(b->atom_of_shell[s]);
      bnp.push_back(b->nprim[s]);
      bps.push_back(p0 + pstart[s]);
      boff.push_back(off);
      for (int d = 0; d < 3; ++d) bc.push_back(b->center[3 * s + d]);
      off += ncart(b->l[s]);
      pstart[s + 1] = pstart[s] + b->nprim[s];
    }
    for (int p = 0; p < pstart[b->n_shells]; ++p) {
      if (!(b->exps[p] > 0.0) || !std::isfinite(b->coefs[p])) return fail(ctx, IQCP_ERR_ARG, "bad primitive");
      bex.push_back(b->exps[p]);
      bco.push_back(b->coefs[p]);
    }
    for (int a = 0; a < b->n_atoms; ++a) {
      bz.push_back(b->z[a]);
      for (int d = 0; d < 3; ++d) bxyz.push_back(b->atom_xyz[3 * a + d]);
    }
    // shell pairs si >= sj (reference order), A = higher-L shell
    for (int si = 0; si < b->n_shells; ++si)
      for (int sj = 0; sj <= si; ++sj) {
        int sa = si, sb = sj;
        if (b->l[sj] > b->l[si]) std::swap(sa, sb);
        ShellPair sp;
        std::memset(&sp, 0, sizeof(sp));
        for (int d = 0; d < 3; ++d) {
          sp.A[d] = b->center[3 * sa + d];
          sp.B[d] = b->center[3 * sb + d];
        }
        sp.sa = s0 + sa;
        sp.sb = s0 + sb;
        sp.oa = ctx->shell_off[s0 + sa];
        sp.ob = ctx->shell_off[s0 + sb];
        sp.atom_a = a0 + b->atom_of_shell[sa];
        sp.atom_b = a0 + b->atom_of_shell[sb];
        sp.comp = si * (si + 1) / 2 + sj;
        sp.mol = m;
        sp.pstart = (int)pps.size();
        double ab2 = 0;
        for (int d = 0; d < 3; ++d) ab2 += (sp.A[d] - sp.B[d]) * (sp.A[d] - sp.B[d]);
        for (int i = 0; i < b->nprim[sa]; ++i)
          for (int j = 0; j < b->nprim[sb]; ++j) {
            const double ea = b->exps[pstart[sa] + i], eb = b->exps[pstart[sb] + j];
            const double K = std::exp(-(ea * eb / (ea + eb)) * ab2);
            if (K < kthr) continue;
            PrimPair q;
            q.p = ea + eb;
            for (int d = 0; d < 3; ++d) q.P[d] = (ea * sp.A[d] + eb * sp.B[d]) / q.p;
            q.K = K;
            q.cK = K * b->coefs[pstart[sa] + i] * rad_norm(ea, b->l[sa]) * b->coefs[pstart[sb] + j] *
                   rad_norm(eb, b->l[sb]);
            q.aa = ea;
            q.inv_p = 1.0 / q.p;
            pps.push_back(q);
          }
        sp.np = (int)pps.size() - sp.pstart;
        ctx->pairs.push_back(sp);
      }
    ctx->n_shells += b->n_shells;
    ctx->n_atoms += b->n_atoms;
    ctx->nbf += off;
    ctx->mol_nbf.push_back(off);
    ctx->mol_base.push_back(base);
    base += (long long)off * off;
  }
  ctx->mol_base.push_back(base);
  ctx->mol_atom0.push_back(ctx->n_atoms);
  ctx->atom_z = bz;
  ctx->atom_xyz = bxyz;
  ctx->mol_shell0.push_back(ctx->n_shells);
  ctx->packed = base;
  ctx->n_prims = (int)bex.size();
  {
    std::vector<int> bi;
    bi.insert(bi.end(), bl.begin(), bl.end());
    bi.insert(bi.end(), bnp.begin(), bnp.end());
    bi.insert(bi.end(), bps.begin(), bps.end());
    bi.insert(bi.end(), boff.begin(), boff.end());
    bi.insert(bi.end(), bz.begin(), bz.end());
    bi.insert(bi.end(), bat.begin(), bat.end());
    std::vector<double> bd;
    bd.insert(bd.end(), bc.begin(), bc.end());
    bd.insert(bd.end(), bex.begin(), bex.end());
    bd.insert(bd.end(), bco.begin(), bco.end());
    bd.insert(bd.end(), bxyz.begin(), bxyz.end());
    CK(cudaMalloc(&ctx->d_bint, sizeof(int) * bi.size()));
    CK(cudaMalloc(&ctx->d_bdbl, sizeof(double) * bd.size()));
    CK(cudaMemcpy(ctx->d_bint, bi.data(), sizeof(int) * bi.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_bdbl, bd.data(), sizeof(double) * bd.size(), cudaMemcpyHostToDevice));
  }
  CK(cudaMalloc(&ctx->d_mol_base, sizeof(long long) * (nmol + 1)));
  CK(cudaMalloc(&ctx->d_mol_n, sizeof(int) * nmol));
  CK(cudaMalloc(&ctx->d_mol_bf0, sizeof(int) * nmol));
  CK(cudaMemcpy(ctx->d_mol_base, ctx->mol_base.data(), sizeof(long long) * (nmol + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_mol_n, ctx->mol_nbf.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_mol_bf0, ctx->mol_bf0.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice));
  ctx->pack = Packing{ctx->d_mol_base, ctx->d_mol_n, ctx->d_mol_bf0, nmol, ctx->packed};

  if (pps.empty()) pps.push_back(PrimPair());
  const int npairs = (int)ctx->pairs.size();
  CK(cudaMalloc(&ctx->d_pairs, sizeof(ShellPair) * npairs));
  CK(cudaMalloc(&ctx->d_pp, sizeof(PrimPair) * pps.size()));
  CK(cudaMemcpy(ctx->d_pairs, ctx->pairs.data(), sizeof(ShellPair) * npairs, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_pp, pps.data(), sizeof(PrimPair) * pps.size(), cudaMemcpyHostToDevice));

  // Schwarz bounds on the device, one launch per pair class
  {
    std::vector<std::vector<int>> by_cls(kNumPairClasses);
    for (int i = 0; i < npairs; ++i) {
      const ShellPair& p = ctx->pairs[i];
      by_cls[pair_class(ctx->shell_l[p.sa], ctx->shell_l[p.sb])].push_back(i);
    }
    int* d_list = nullptr;
    CK(cudaMalloc(&d_list, sizeof(int) * npairs));
    int pos = 0;
    for (int c = 0; c < kNumPairClasses; ++c) {
      if (by_cls[c].empty()) continue;
      CK(cudaMemcpy(d_list + pos, by_cls[c].data(), sizeof(int) * by_cls[c].size(), cudaMemcpyHostToDevice));
      CK(launch_schwarz(c, ctx->d_pairs, ctx->d_pp, d_list + pos, (int)by_cls[c].size(), kthr, ctx->stream));
      pos += (int)by_cls[c].size();
    }
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaFree(d_list));
    CK(cudaMemcpy(ctx->pairs.data(), ctx->d_pairs, sizeof(ShellPair) * npairs, cudaMemcpyDeviceToHost));
  }
  std::vector<int> ket_list;
  std::vector<QuartetTask> tasks;
  build_tasks(ctx, ket_list, tasks);
  if (ket_list.empty()) ket_list.push_back(0);
  if (tasks.empty()) tasks.push_back(QuartetTask());
  ctx->n_tasks = (int)tasks.size();
  CK(cudaMalloc(&ctx->d_mask, sizeof(unsigned) * tasks.size()));
  CK(cudaMalloc(&ctx->d_ket_list, sizeof(int) * ket_list.size()));
  CK(cudaMemcpy(ctx->d_ket_list, ket_list.data(), sizeof(int) * ket_list.size(), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&ctx->d_tasks, sizeof(QuartetTask) * tasks.size()));
  CK(cudaMemcpy(ctx->d_tasks, tasks.data(), sizeof(QuartetTask) * tasks.size(), cudaMemcpyHostToDevice));

  const size_t nn = (size_t)ctx->packed;
  CK(cudaMalloc(&ctx->d_ang, sizeof(double) * ctx->nbf));
  CK(cudaMemcpy(ctx->d_ang, ang.data(), sizeof(double) * ctx->nbf, cudaMemcpyHostToDevice));
  CK(cudaMalloc(&ctx->d_Ds, sizeof(double) * nn));
  CK(cudaMalloc(&ctx->d_Jt, sizeof(double) * nn));
  CK(cudaMalloc(&ctx->d_Kt, sizeof(double) * nn));
  for (int i = 0; i < 4; ++i) CK(cudaMalloc(&ctx->d_io[i], sizeof(double) * nn));
  CK(cudaMalloc(&ctx->d_grad, sizeof(double) * 3 * ctx->n_atoms));
  {
    std::vector<long long> dbase(nmol + 1, 0);
    std::vector<int> ns(nmol);
    for (int m = 0; m < nmol; ++m) {
      ns[m] = ctx->mol_shell0[m + 1] - ctx->mol_shell0[m];
      dbase[m + 1] = dbase[m] + (long long)ns[m] * ns[m];
    }
    ctx->dmax_total = dbase[nmol];
    CK(cudaMalloc(&ctx->d_dmax, sizeof(double) * ctx->dmax_total));
    CK(cudaMalloc(&ctx->d_dbase, sizeof(long long) * (nmol + 1)));
    CK(cudaMalloc(&ctx->d_mol_shell0, sizeof(int) * nmol));
    CK(cudaMalloc(&ctx->d_mol_ns, sizeof(int) * nmol));
    CK(cudaMemcpy(ctx->d_dbase, dbase.data(), sizeof(long long) * (nmol + 1), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_mol_shell0, ctx->mol_shell0.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_mol_ns, ns.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice));
  }
  CK(cudaMalloc(&ctx->d_counters, sizeof(int) * 4 * (ctx->ranges.size() + 1)));
  CK(cudaMalloc(&ctx->d_fp32, sizeof(unsigned long long)));
  return IQCP_OK;
}

int iqcp_create(const iqcp_basis_desc* b, const iqcp_options* opts, iqcp_ctx** out) {
  if (!b || !out || b->n_shells <= 0 || b->n_atoms <= 0) return IQCP_ERR_ARG;
  return create_batch(1, b, opts, out);
}

int iqcp_create_batch(int n_mol, const iqcp_basis_desc* bases, const iqcp_options* opts, iqcp_ctx** out) {
  return create_batch(n_mol, bases, opts, out);
}

int iqcp_batch_layout(const iqcp_ctx* ctx, long long* mat_offset, int* nbf, int* atom_offset) {
  if (!ctx) return IQCP_ERR_ARG;
  for (int m = 0; m <= ctx->n_mol; ++m) {
    if (mat_offset) mat_offset[m] = ctx->mol_base[m];
    if (atom_offset) atom_offset[m] = ctx->mol_atom0[m];
    if (nbf && m < ctx->n_mol) nbf[m] = ctx->mol_nbf[m];
  }
  return ctx->n_mol;
}

void iqcp_destroy(iqcp_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  cudaFree(ctx->d_pairs);
  cudaFree(ctx->d_pp);
  cudaFree(ctx->d_ket_list);
  cudaFree(ctx->d_tasks);
  cudaFree(ctx->d_ang);
  cudaFree(ctx->d_Ds);
  cudaFree(ctx->d_Jt);
  cudaFree(ctx->d_Kt);
  for (int i = 0; i < 4; ++i) cudaFree(ctx->d_io[i]);
  cudaFree(ctx->d_grad);
  cudaFree(ctx->d_bint);
  cudaFree(ctx->d_bdbl);
  cudaFree(ctx->d_dmax);
  cudaFree(ctx->d_dbase);
  cudaFree(ctx->d_mol_shell0);
  cudaFree(ctx->d_mol_ns);
  cudaFree(ctx->d_mask);
  cudaFree(ctx->d_mol_base);
  cudaFree(ctx->d_mol_n);
  cudaFree(ctx->d_mol_bf0);
  cudaFree(ctx->d_counters);
  cudaFree(ctx->d_fp32);
  cudaFree(ctx->d_multi);
  cudaFree(ctx->d_multi_io);
  cudaFree(ctx->d_cart_info);
  cudaFree(ctx->d_sph_info);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  for (int s = 0; s < iqcp_ctx::kSide; ++s) {
    if (ctx->join_ev[s]) cudaEventDestroy(ctx->join_ev[s]);
    if (ctx->side[s]) cudaStreamDestroy(ctx->side[s]);
  }
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

int iqcp_set_stream(iqcp_ctx* ctx, void* stream) {
  if (!ctx) return IQCP_ERR_ARG;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return IQCP_OK;
}

int iqcp_jk_device(iqcp_ctx* ctx, const double* dD, double* dJ, double* dK) {
  if (!ctx || !dD || !dJ) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  rc = run_jk_device(ctx, dD, dK != nullptr);
  if (rc) return rc;
  CK(launch_symmetrize(ctx->d_Jt, ctx->d_ang, ctx->pack, dJ, ctx->stream));
  ctx->launches_total += 1;
  if (dK) {
    CK(launch_symmetrize(ctx->d_Kt, ctx->d_ang, ctx->pack, dK, ctx->stream));
    ctx->launches_total += 1;
  }
  return finish_stats(ctx);
}

int iqcp_fock_device(iqcp_ctx* ctx, const double* dH, const double* dD, double k_scale, double* dF) {
  if (!ctx || !dH || !dD || !dF) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  rc = run_jk_device(ctx, dD, k_scale != 0.0);
  if (rc) return rc;
  CK(launch_fock(dH, ctx->d_Jt, k_scale != 0.0 ? ctx->d_Kt : nullptr, ctx->d_ang, ctx->pack, k_scale, dF,
                 ctx->stream));
  ctx->launches_total += 1;
  return finish_stats(ctx);
}

// ---------------------------------------------------------------------------
// J/K build that allocates nothing.
//
// Some callers cannot call cudaMalloc at the point where they need a Fock
// build: a serving process that has handed all of HBM to its own memory pool
// (a cudaMalloc there fails), or a solver loop that must not stall on the
// implicit device synchronisation an allocation can cause.  For them this
// entry point keeps its scratch -- the angular-scaled density and the two
// unsymmetrised J/K accumulators -- in one file-scope device array of fixed
// size instead of the context's own buffers.  The context itself (pair tables,
// quartet lists, the mixed form's density-bound table and masks) is built
// beforehand by iqcp_create, where allocation is allowed.
//
// Limits and rules:
//   * nbf <= IQCP_NOALLOC_MAX_NBF (512): the array holds 3 * 512 * 512 doubles
//     (6 MiB), reserved on every GPU that loads the library until exit;
//     larger bases are rejected with IQCP_ERR_ARG.
//   * The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current); make
//     that first call before any stream capture.
//   * All calls share the one array, which keeps the last call's contents;
//     the accumulators are cleared at the start of every call.  Calls whose
//     work overlaps on the GPU (other streams, other host threads) race on the
//     array: serialise them.
//   * The call only enqueues work on the context stream and returns without
//     waiting for the GPU; iqcp_last_stats reports its screened quartets and
//     launches, not its device time or FP32 count (both 0).
#define IQCP_NOALLOC_MAX_NBF 512
static __device__ __align__(256) double g_noalloc_scratch[3 * IQCP_NOALLOC_MAX_NBF * IQCP_NOALLOC_MAX_NBF];
static double* g_noalloc_ptr[64] = {nullptr};

static int noalloc_scratch(iqcp_ctx* ctx, double** out) {
  if (ctx->device < 0 || ctx->device >= 64) return fail(ctx, IQCP_ERR_ARG, "device ordinal out of range");
  if (!g_noalloc_ptr[ctx->device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(ctx, IQCP_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") +
                                          cudaGetErrorString(e));
    g_noalloc_ptr[ctx->device] = static_cast<double*>(p);
  }
  *out = g_noalloc_ptr[ctx->device];
  return IQCP_OK;
}

int iqcp_jk_device_noalloc(iqcp_ctx* ctx, const double* dD, double* dJ, double* dK) {
  if (!ctx || !dD || !dJ) return IQCP_ERR_ARG;
  if (ctx->n_mol != 1) return fail(ctx, IQCP_ERR_ARG, "iqcp_jk_device_noalloc takes single-geometry contexts");
  if (ctx->nbf > IQCP_NOALLOC_MAX_NBF)
    return fail(ctx, IQCP_ERR_ARG, "iqcp_jk_device_noalloc supports nbf <= 512 (static scratch size); nbf = " +
                                       std::to_string(ctx->nbf));
  int rc = ensure_device(ctx);
  if (rc) return rc;
  double* scratch = nullptr;
  rc = noalloc_scratch(ctx, &scratch);
  if (rc) return rc;
  const int n = ctx->nbf;
  const size_t nn = (size_t)n * n;
  double* Ds = scratch;
  double* Jt = scratch + nn;
  double* Kt = scratch + 2 * nn;
  const bool want_k = dK != nullptr;
  // per-launch timing would create events: off for this call, restored on every exit
  struct ProfileOff {
    iqcp_ctx* c;
    bool saved;
    ~ProfileOff() { c->profile = saved; }
  } guard{ctx, ctx->profile};
  ctx->profile = false;
  ctx->stats[2] = ctx->stats[3] = 0.0;
  ctx->launches_total = 1;
  CK(launch_scale_density(dD, ctx->d_ang, ctx->pack, Ds, ctx->stream));
  // the mixed form uses only context buffers (density bounds, task masks)
  ctx->mixed_call = ctx->opt.precision == IQCP_MIXED;
  if (ctx->mixed_call) {
    rc = prepare_mixed(ctx, dD, 0);
    if (rc) return rc;
  }
  CK(cudaMemsetAsync(Jt, 0, sizeof(double) * nn, ctx->stream));
  if (want_k) CK(cudaMemsetAsync(Kt, 0, sizeof(double) * nn, ctx->stream));
  rc = run_ranges(ctx, 0, [&](const TaskRange& r, int pass, int* counter, cudaStream_t st) {
    const JKArgs a = jk_args(ctx, r, Ds, Jt, want_k ? Kt : nullptr, pass == 2 ? r.mode32[0] : r.mode[0], pass,
                             counter);
    return launch_jk(r.X, r.Y, a, st);
  });
  if (rc) return rc;
  CK(launch_symmetrize(Jt, ctx->d_ang, ctx->pack, dJ, ctx->stream));
  ctx->launches_total += 1;
  if (want_k) {
    CK(launch_symmetrize(Kt, ctx->d_ang, ctx->pack, dK, ctx->stream));
    ctx->launches_total += 1;
  }
  return IQCP_OK;  // enqueued only: no wait for the GPU
}

int iqcp_jk(iqcp_ctx* ctx, const double* D, double* J, double* K) {
  if (!ctx || !D || !J) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  const size_t bytes = sizeof(double) * (size_t)ctx->packed;
  CK(cudaMemcpyAsync(ctx->d_io[0], D, bytes, cudaMemcpyHostToDevice, ctx->stream));
  rc = iqcp_jk_device(ctx, ctx->d_io[0], ctx->d_io[1], K ? ctx->d_io[2] : nullptr);
  if (rc) return rc;
  CK(cudaMemcpyAsync(J, ctx->d_io[1], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (K) CK(cudaMemcpyAsync(K, ctx->d_io[2], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return IQCP_OK;
}

int iqcp_fock(iqcp_ctx* ctx, const double* H, const double* D, double k_scale, double* F) {
  if (!ctx || !H || !D || !F) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  const size_t bytes = sizeof(double) * (size_t)ctx->packed;
  CK(cudaMemcpyAsync(ctx->d_io[0], D, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_io[1], H, bytes, cudaMemcpyHostToDevice, ctx->stream));
  rc = iqcp_fock_device(ctx, ctx->d_io[1], ctx->d_io[0], k_scale, ctx->d_io[2]);
  if (rc) return rc;
  CK(cudaMemcpyAsync(F, ctx->d_io[2], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return IQCP_OK;
}

// Grow a device buffer to at least `need` doubles (contents are not kept).
static int grow(iqcp_ctx* ctx, double** buf, long long* cap, long long need) {
  if (*cap >= need) return IQCP_OK;
  if (*buf) CK(cudaFree(*buf));
  *buf = nullptr;
  *cap = 0;
  if (cudaMalloc(buf, sizeof(double) * (size_t)need) != cudaSuccess)
    return fail(ctx, IQCP_ERR_NOMEM, "device buffer of " + std::to_string(need) + " doubles");
  *cap = need;
  return IQCP_OK;
}

int iqcp_jk_multi_device(iqcp_ctx* ctx, int nset, const double* dD, double* dJ, double* dK) {
  if (!ctx || nset < 1 || !dD || !dJ) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  const long long nn = ctx->packed;
  rc = grow(ctx, &ctx->d_multi, &ctx->multi_cap, 3 * nn * nset);
  if (rc) return rc;
  double* Ds = ctx->d_multi;
  double* Jt = Ds + nn * nset;
  double* Kt = Jt + nn * nset;
  const bool want_k = dK != nullptr;
  ctx->launches_total = 0;
  for (int s = 0; s < nset; ++s)
    CK(launch_scale_density(dD + s * nn, ctx->d_ang, ctx->pack, Ds + s * nn, ctx->stream));
  ctx->launches_total += nset;
  ctx->mixed_call = false;  // response densities: FP64 quadrature
  CK(cudaMemsetAsync(Jt, 0, sizeof(double) * nn * nset, ctx->stream));
  if (want_k) CK(cudaMemsetAsync(Kt, 0, sizeof(double) * nn * nset, ctx->stream));
  rc = run_ranges(ctx, 0, [&](const TaskRange& r, int pass, int* counter, cudaStream_t st) {
    JKArgs a = jk_args(ctx, r, Ds, Jt, want_k ? Kt : nullptr, r.mode[0], pass, counter);
    a.nset = nset;
    a.set_stride = nn;
    return launch_jk(r.X, r.Y, a, st);
  });
  if (rc) return rc;
  for (int s = 0; s < nset; ++s) {
    CK(launch_symmetrize(Jt + s * nn, ctx->d_ang, ctx->pack, dJ + s * nn, ctx->stream));
    if (want_k) CK(launch_symmetrize(Kt + s * nn, ctx->d_ang, ctx->pack, dK + s * nn, ctx->stream));
  }
  ctx->launches_total += nset * (want_k ? 2 : 1);
  return finish_stats(ctx);
}

int iqcp_jk_multi(iqcp_ctx* ctx, int nset, const double* D, double* J, double* K) {
  if (!ctx || nset < 1 || !D || !J) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  const long long nn = ctx->packed;
  rc = grow(ctx, &ctx->d_multi_io, &ctx->multi_io_cap, 3 * nn * nset);
  if (rc) return rc;
  double* dD = ctx->d_multi_io;
  double* dJ = dD + nn * nset;
  double* dK = dJ + nn * nset;
  const size_t bytes = sizeof(double) * (size_t)(nn * nset);
  CK(cudaMemcpyAsync(dD, D, bytes, cudaMemcpyHostToDevice, ctx->stream));
  rc = iqcp_jk_multi_device(ctx, nset, dD, dJ, K ? dK : nullptr);
  if (rc) return rc;
  CK(cudaMemcpyAsync(J, dJ, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (K) CK(cudaMemcpyAsync(K, dK, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return IQCP_OK;
}

// G = J - 1/2 k_scale K and F = H + G, element by element over the packed matrices.
static __global__ void fock_parts_kernel(const double* __restrict__ H, const double* __restrict__ J,
                                  const double* __restrict__ K, double kscale, long long n, double* __restrict__ G,
                                  double* __restrict__ F) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double g = J[i] - 0.5 * kscale * K[i];
    if (G) G[i] = g;
    if (F) F[i] = H[i] + g;
  }
}

int iqcp_fock_decomposition(iqcp_ctx* ctx, const double* H, const double* D, double k_scale, double* J, double* K,
                            double* G, double* F) {
  if (!ctx || !D || (F && !H)) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  const long long nn = ctx->packed;
  const size_t bytes = sizeof(double) * (size_t)nn;
  // staging: D, then H (after the build) in io[0]; J io[1], K io[2], G io[3]; F over H
  CK(cudaMemcpyAsync(ctx->d_io[0], D, bytes, cudaMemcpyHostToDevice, ctx->stream));
  rc = iqcp_jk_device(ctx, ctx->d_io[0], ctx->d_io[1], ctx->d_io[2]);
  if (rc) return rc;
  if (H) CK(cudaMemcpyAsync(ctx->d_io[0], H, bytes, cudaMemcpyHostToDevice, ctx->stream));
  const int blocks = (int)std::min<long long>((nn + 255) / 256, 4096);
  fock_parts_kernel<<<blocks, 256, 0, ctx->stream>>>(H ? ctx->d_io[0] : nullptr, ctx->d_io[1], ctx->d_io[2],
                                                      k_scale, nn, ctx->d_io[3], H ? ctx->d_io[0] : nullptr);
  CK(cudaGetLastError());
  if (J) CK(cudaMemcpyAsync(J, ctx->d_io[1], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (K) CK(cudaMemcpyAsync(K, ctx->d_io[2], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (G) CK(cudaMemcpyAsync(G, ctx->d_io[3], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (F) CK(cudaMemcpyAsync(F, ctx->d_io[0], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return IQCP_OK;
}

// ---------------------------------------------------------------------------
// Spherical basis.  Real solid harmonics from Cartesian functions with the
// coefficients C[cart][sph] the reference uses (CART2SPH_D, integrals/spherical.rs:71,
// libcint cart2sph): AO_sph = C^T AO_cart per shell; identity for s and p.
// Both the ERI transform of the reference's spherical path (EriSphericalTransform,
// spherical.rs:390-470, then J/K from the transformed ERIs) and J/K linearity
// give J_sph[D_sph] = C^T J_cart[C D_sph C^T] C, likewise K.
__constant__ double kCart2SphD[6][5] = {
    {0.0, 0.0, -0.315391565252520002, 0.0, 0.546274215296039535},
    {1.092548430592079070, 0.0, 0.0, 0.0, 0.0},
    {0.0, 0.0, 0.0, 1.092548430592079070, 0.0},
    {0.0, 0.0, -0.315391565252520002, 0.0, -0.546274215296039535},
    {0.0, 1.092548430592079070, 0.0, 0.0, 0.0},
    {0.0, 0.0, 0.630783130505040012, 0.0, 0.0}};

__device__ __forceinline__ double cart2sph(int l, int c, int m) {
  return l == 2 ? kCart2SphD[c][m] : (c == m ? 1.0 : 0.0);
}

// Dc = C Ds C^T (Cartesian from spherical), element per thread
static __global__ void sph_to_cart_kernel(int nc, int ns, const int4* __restrict__ cinfo,
                                          const double* __restrict__ Ds, double* __restrict__ Dc) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)nc * nc) return;
  const int a = int(e / nc), b = int(e - (long long)a * nc);
  const int4 ia = cinfo[a], ib = cinfo[b];  // {sph offset, position, l, -}
  double v = 0.0;
  for (int i = 0; i < 2 * ia.z + 1; ++i) {
    const double ca = cart2sph(ia.z, ia.y, i);
    if (ca == 0.0) continue;
    for (int j = 0; j < 2 * ib.z + 1; ++j)
      v = fma(ca * cart2sph(ib.z, ib.y, j), Ds[(long long)(ia.x + i) * ns + ib.x + j], v);
  }
  Dc[e] = v;
}

// Xs = C^T Xc C (spherical from Cartesian), element per thread
static __global__ void cart_to_sph_kernel(int nc, int ns, const int4* __restrict__ sinfo,
                                          const double* __restrict__ Xc, double* __restrict__ Xs) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)ns * ns) return;
  const int i = int(e / ns), j = int(e - (long long)i * ns);
  const int4 si = sinfo[i], sj = sinfo[j];  // {Cartesian offset, m, l, -}
  const int na = (si.z + 1) * (si.z + 2) / 2, nb = (sj.z + 1) * (sj.z + 2) / 2;
  double v = 0.0;
  for (int a = 0; a < na; ++a) {
    const double ca = cart2sph(si.z, a, si.y);
    if (ca == 0.0) continue;
    for (int b = 0; b < nb; ++b)
      v = fma(ca * cart2sph(sj.z, b, sj.y), Xc[(long long)(si.x + a) * nc + sj.x + b], v);
  }
  Xs[e] = v;
}

static int spherical_tables(iqcp_ctx* ctx) {
  if (ctx->d_cart_info) return IQCP_OK;
  std::vector<int4> ci, si;
  int os = 0;
  for (int s = 0; s < ctx->n_shells; ++s) {
    const int l = ctx->shell_l[s], oc = ctx->shell_off[s];
    for (int c = 0; c < ncart(l); ++c) ci.push_back(make_int4(os, c, l, 0));
    for (int m = 0; m < 2 * l + 1; ++m) si.push_back(make_int4(oc, m, l, 0));
    os += 2 * l + 1;
  }
  ctx->nsph = os;
  CK(cudaMalloc(&ctx->d_cart_info, sizeof(int4) * ci.size()));
  CK(cudaMalloc(&ctx->d_sph_info, sizeof(int4) * si.size()));
  CK(cudaMemcpy(ctx->d_cart_info, ci.data(), sizeof(int4) * ci.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_sph_info, si.data(), sizeof(int4) * si.size(), cudaMemcpyHostToDevice));
  return IQCP_OK;
}

int iqcp_nbf_spherical(iqcp_ctx* ctx) {
  if (!ctx) return 0;
  int n = 0;
  for (int s = 0; s < ctx->n_shells; ++s) n += 2 * ctx->shell_l[s] + 1;
  return n;
}

int iqcp_jk_spherical(iqcp_ctx* ctx, const double* Ds, double* Js, double* Ks) {
  if (!ctx || !Ds || !Js) return IQCP_ERR_ARG;
  if (ctx->n_mol != 1) return fail(ctx, IQCP_ERR_ARG, "iqcp_jk_spherical takes single-geometry contexts");
  int rc = ensure_device(ctx);
  if (rc) return rc;
  if ((rc = spherical_tables(ctx))) return rc;
  const int nc = ctx->nbf, ns = ctx->nsph;
  const long long ncc = (long long)nc * nc, nss = (long long)ns * ns;
  const int4* cinfo = reinterpret_cast<const int4*>(ctx->d_cart_info);
  const int4* sinfo = reinterpret_cast<const int4*>(ctx->d_sph_info);
  // io[3] <- D_sph; io[0] <- D_cart; J_cart, K_cart in io[1], io[2]; results back through io[3], io[0]
  CK(cudaMemcpyAsync(ctx->d_io[3], Ds, sizeof(double) * nss, cudaMemcpyHostToDevice, ctx->stream));
  sph_to_cart_kernel<<<(int)((ncc + 255) / 256), 256, 0, ctx->stream>>>(nc, ns, cinfo, ctx->d_io[3], ctx->d_io[0]);
  CK(cudaGetLastError());
  rc = iqcp_jk_device(ctx, ctx->d_io[0], ctx->d_io[1], Ks ? ctx->d_io[2] : nullptr);
  if (rc) return rc;
  cart_to_sph_kernel<<<(int)((nss + 255) / 256), 256, 0, ctx->stream>>>(nc, ns, sinfo, ctx->d_io[1], ctx->d_io[3]);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(Js, ctx->d_io[3], sizeof(double) * nss, cudaMemcpyDeviceToHost, ctx->stream));
  if (Ks) {
    cart_to_sph_kernel<<<(int)((nss + 255) / 256), 256, 0, ctx->stream>>>(nc, ns, sinfo, ctx->d_io[2],
                                                                           ctx->d_io[0]);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(Ks, ctx->d_io[0], sizeof(double) * nss, cudaMemcpyDeviceToHost, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return IQCP_OK;
}

int iqcp_eri_grad_device(iqcp_ctx* ctx, const double* dD, double hf_frac, double* dgrad) {
  if (!ctx || !dD || !dgrad) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  ctx->launches_total = 1;
  CK(launch_scale_density(dD, ctx->d_ang, ctx->pack, ctx->d_Ds, ctx->stream));
  ctx->mixed_call = ctx->opt.precision == IQCP_MIXED;
  if (ctx->mixed_call) {
    rc = prepare_mixed(ctx, dD, 1);
    if (rc) return rc;
  }
  rc = run_ranges(ctx, 1, [&](const TaskRange& r, int pass, int* counter, cudaStream_t st) {
    const GradArgs a = grad_args(ctx, r, ctx->d_Ds, 0.25 * hf_frac, dgrad, pass == 2 ? r.mode32[1] : r.mode[1],
                                 pass, counter);
    return launch_grad(r.X, r.Y, a, st);
  });
  if (rc) return rc;
  return finish_stats(ctx);
}

int iqcp_eri_grad(iqcp_ctx* ctx, const double* D, double hf_frac, double* grad) {
  if (!ctx || !D || !grad) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  const size_t bytes = sizeof(double) * (size_t)ctx->packed;
  CK(cudaMemcpyAsync(ctx->d_io[0], D, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_grad, grad, sizeof(double) * 3 * ctx->n_atoms, cudaMemcpyHostToDevice, ctx->stream));
  rc = iqcp_eri_grad_device(ctx, ctx->d_io[0], hf_frac, ctx->d_grad);
  if (rc) return rc;
  CK(cudaMemcpyAsync(grad, ctx->d_grad, sizeof(double) * 3 * ctx->n_atoms, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return IQCP_OK;
}

int iqcp_eri_compressed(iqcp_ctx* ctx, double* out, long long out_len) {
  if (!ctx || !out) return IQCP_ERR_ARG;
  if (ctx->n_mol != 1) return fail(ctx, IQCP_ERR_ARG, "iqcp_eri_compressed takes single-geometry contexts");
  const long long n = ctx->nbf, np = n * (n + 1) / 2, ne = np * (np + 1) / 2;
  if (out_len < ne) return fail(ctx, IQCP_ERR_ARG, "output too small for the compressed ERI array");
  int rc = ensure_device(ctx);
  if (rc) return rc;
  double* d_out = nullptr;
  if (cudaMalloc(&d_out, sizeof(double) * ne) != cudaSuccess)
    return fail(ctx, IQCP_ERR_NOMEM, "compressed ERI array does not fit on the device");
  CK(cudaMemsetAsync(d_out, 0, sizeof(double) * ne, ctx->stream));
  for (const TaskRange& r : ctx->ranges) {
    if (r.count == 0) continue;
    StoreArgs a;
    a.pairs = ctx->d_pairs;
    a.pp = ctx->d_pp;
    a.ket_list = ctx->d_ket_list;
    a.tasks = ctx->d_tasks + r.first;
    a.ntasks = r.count;
    a.out = d_out;
    a.prim_thr = ctx->opt.prim_threshold;
    CK(launch_store(r.X, r.Y, a, ctx->stream));
  }
  CK(cudaMemcpyAsync(out, d_out, sizeof(double) * ne, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaFree(d_out));
  return IQCP_OK;
}

static OneEArgs one_e_args(const iqcp_ctx* ctx, int m) {
  const int ns = ctx->n_shells;
  const int s0 = ctx->mol_shell0[m], a0 = ctx->mol_atom0[m];
  OneEArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n_shells = ctx->mol_shell0[m + 1] - s0;
  a.n_atoms = ctx->mol_atom0[m + 1] - a0;
  a.nbf = ctx->mol_nbf[m];
  a.l = ctx->d_bint + s0;
  a.nprim = ctx->d_bint + ns + s0;
  a.pstart = ctx->d_bint + 2 * ns + s0;
  a.off = ctx->d_bint + 3 * ns + s0;
  a.z = ctx->d_bint + 4 * ns + a0;
  a.atom = ctx->d_bint + 4 * ns + ctx->n_atoms + s0;
  a.center = ctx->d_bdbl + 3 * s0;
  a.exps = ctx->d_bdbl + 3 * ns;
  a.coefs = a.exps + ctx->n_prims;
  a.atom_xyz = a.coefs + ctx->n_prims + 3 * a0;
  return a;
}

int iqcp_one_electron(iqcp_ctx* ctx, double* S, double* T, double* V) {
  if (!ctx) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  const size_t bytes = sizeof(double) * (size_t)ctx->packed;
  // one launch per molecule block of the packed matrices
  for (int m = 0; m < ctx->n_mol; ++m) {
    const long long mb = ctx->mol_base[m];
    OneEArgs a = one_e_args(ctx, m);
    a.S = S ? ctx->d_io[0] + mb : nullptr;
    a.T = T ? ctx->d_io[1] + mb : nullptr;
    a.V = V ? ctx->d_io[2] + mb : nullptr;
    CK(launch_one_electron(a, ctx->stream));
  }
  if (S) CK(cudaMemcpyAsync(S, ctx->d_io[0], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (T) CK(cudaMemcpyAsync(T, ctx->d_io[1], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (V) CK(cudaMemcpyAsync(V, ctx->d_io[2], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return IQCP_OK;
}

int iqcp_one_electron_grad_device(iqcp_ctx* ctx, const double* dD, const double* dW, double* dgrad) {
  if (!ctx || !dD || !dW || !dgrad) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  for (int m = 0; m < ctx->n_mol; ++m) {
    const long long mb = ctx->mol_base[m];
    OneEArgs a = one_e_args(ctx, m);
    a.D = dD + mb;
    a.W = dW + mb;
    a.grad = dgrad + 3 * ctx->mol_atom0[m];
    a.gsmem = a.n_atoms <= 2048 ? 1 : 0;
    CK(launch_one_electron_grad(a, ctx->stream));
  }
  return IQCP_OK;
}

int iqcp_one_electron_grad(iqcp_ctx* ctx, const double* D, const double* W, double* grad) {
  if (!ctx || !D || !W || !grad) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  const size_t bytes = sizeof(double) * (size_t)ctx->packed;
  const size_t gb = sizeof(double) * 3 * ctx->n_atoms;
  CK(cudaMemcpyAsync(ctx->d_io[0], D, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_io[1], W, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_grad, grad, gb, cudaMemcpyHostToDevice, ctx->stream));
  rc = iqcp_one_electron_grad_device(ctx, ctx->d_io[0], ctx->d_io[1], ctx->d_grad);
  if (rc) return rc;
  CK(cudaMemcpyAsync(grad, ctx->d_grad, gb, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return IQCP_OK;
}

int iqcp_rhf_gradient(iqcp_ctx* ctx, const double* D, const double* W, double* grad) {
  if (!ctx || !D || !W || !grad) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  const size_t bytes = sizeof(double) * (size_t)ctx->packed;
  const size_t gb = sizeof(double) * 3 * ctx->n_atoms;
  CK(cudaMemcpyAsync(ctx->d_io[0], D, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_io[1], W, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_grad, 0, gb, ctx->stream));
  rc = iqcp_one_electron_grad_device(ctx, ctx->d_io[0], ctx->d_io[1], ctx->d_grad);
  if (rc) return rc;
  rc = iqcp_eri_grad_device(ctx, ctx->d_io[0], 1.0, ctx->d_grad);
  if (rc) return rc;
  CK(cudaMemcpyAsync(grad, ctx->d_grad, gb, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return IQCP_OK;
}

int iqcp_schwarz(iqcp_ctx* ctx, double* Q) {
  if (!ctx || !Q) return IQCP_ERR_ARG;
  const int ns = ctx->n_shells;
  for (const ShellPair& p : ctx->pairs) {
    Q[p.sa * ns + p.sb] = p.Q;
    Q[p.sb * ns + p.sa] = p.Q;
  }
  return IQCP_OK;
}

int iqcp_set_precision(iqcp_ctx* ctx, int precision, double mixed_cutoff) {
  if (!ctx || (precision != IQCP_FP64 && precision != IQCP_MIXED) || !(mixed_cutoff >= 0.0)) return IQCP_ERR_ARG;
  ctx->opt.precision = precision;
  ctx->opt.mixed_cutoff = mixed_cutoff;
  return IQCP_OK;
}

int iqcp_set_profiling(iqcp_ctx* ctx, int on) {
  if (!ctx) return IQCP_ERR_ARG;
  ctx->profile = on != 0;
  return IQCP_OK;
}

int iqcp_launch_profile(const iqcp_ctx* ctx, int max, int* kind, int* X, int* Y, double* ms,
                        long long* quartets) {
  if (!ctx) return IQCP_ERR_ARG;
  const int n = (int)ctx->launch_log.size();
  for (int i = 0; i < n && i < max; ++i) {
    kind[i] = ctx->launch_log[i].kind;
    X[i] = ctx->launch_log[i].X;
    Y[i] = ctx->launch_log[i].Y;
    ms[i] = ctx->launch_log[i].ms;
    quartets[i] = ctx->launch_log[i].quartets;
  }
  return n;
}

int iqcp_kernel_launches(const iqcp_ctx* ctx) { return ctx ? ctx->launches_total : 0; }

// Autotuner: time every class range with every kernel variant on this
// density (best of `reps` runs each) and keep the fastest variant per class
// and per kind (J/K, gradient).  In the mixed form the FP64 and FP32 shares
// are tuned separately at the current cutoff, and a class is split into the
// two passes only where that beats running it wholly in FP64.  Results are
// the same up to rounding whichever variant runs; only the speed differs.
int iqcp_autotune(iqcp_ctx* ctx, const double* dD, int reps) {
  if (!ctx || !dD) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  if (reps < 1) reps = 1;
  const size_t bytes = sizeof(double) * (size_t)ctx->packed;
  CK(launch_scale_density(dD, ctx->d_ang, ctx->pack, ctx->d_Ds, ctx->stream));
  const bool mixed = ctx->opt.precision == IQCP_MIXED;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  // best time over the variants of one (range, kind, pass); mode_out gets the winner
  auto tune = [&](TaskRange& r, int kind, int pass, int* mode_out, float* t_out) -> int {
    // a batched context times a sample of the range: the tasks of about eight
    // molecules' worth (tasks run molecule by molecule)
    const int ntune = ctx->n_mol > 8 ? std::min(r.count, std::max(4096, int((long long)r.count * 8 / ctx->n_mol)))
                                     : r.count;
    float best = 1e30f;
    for (int mode = 0; mode < kNumModes; ++mode) {
      if (pass == 2 && mode == 3) continue;  // the FP32 share has no 32-lane variant
      float tmin = 1e30f;
      for (int rep = 0; rep < reps + 1; ++rep) {  // first run warms caches and sets attributes
        CK(cudaMemsetAsync(ctx->d_Jt, 0, bytes, ctx->stream));
        CK(cudaMemsetAsync(ctx->d_Kt, 0, bytes, ctx->stream));
        CK(cudaMemsetAsync(ctx->d_grad, 0, sizeof(double) * 3 * ctx->n_atoms, ctx->stream));
        CK(cudaMemsetAsync(ctx->d_counters, 0, sizeof(int), ctx->stream));
        CK(cudaEventRecord(e0, ctx->stream));
        if (kind == 0) {
          JKArgs a = jk_args(ctx, r, ctx->d_Ds, ctx->d_Jt, ctx->d_Kt, mode, pass, ctx->d_counters);
          a.ntasks = ntune;
          CK(launch_jk(r.X, r.Y, a, ctx->stream));
        } else {
          GradArgs a = grad_args(ctx, r, ctx->d_Ds, 0.25, ctx->d_grad, mode, pass, ctx->d_counters);
          a.ntasks = ntune;
          CK(launch_grad(r.X, r.Y, a, ctx->stream));
        }
        CK(cudaEventRecord(e1, ctx->stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0) tmin = std::min(tmin, ms);
      }
      if (tmin < best) {
        best = tmin;
        *mode_out = mode;
      }
    }
    *t_out = best;
    return IQCP_OK;
  };
  for (int kind = 0; kind < 2; ++kind) {
    if (mixed) {
      rc = prepare_mixed(ctx, dD, kind);
      if (rc) return rc;
    }
    for (TaskRange& r : ctx->ranges) {
      if (r.count == 0) continue;
      int m0 = r.mode[kind];
      float t0 = 0.f;
      if ((rc = tune(r, kind, 0, &m0, &t0))) return rc;
      r.mode[kind] = m0;
      if (!mixed) continue;
      int m1 = m0, m2 = r.mode32[kind];
      float t1 = 0.f, t2 = 0.f;
      if ((rc = tune(r, kind, 1, &m1, &t1))) return rc;
      if ((rc = tune(r, kind, 2, &m2, &t2))) return rc;
      r.mode32[kind] = m2;
      r.split[kind] = (t1 + t2 < t0) ? 1 : 0;
      if (r.split[kind]) r.mode[kind] = m1;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return IQCP_OK;
}

// Current kernel variant per (kind, bra class, ket class): modes[2*6*6], -1 when no work.
int iqcp_kernel_modes(const iqcp_ctx* ctx, int* modes) {
  if (!ctx || !modes) return IQCP_ERR_ARG;
  for (int i = 0; i < 4 * kNumPairClasses * kNumPairClasses; ++i) modes[i] = -1;
  for (const TaskRange& r : ctx->ranges)
    if (r.count > 0)
      for (int kind = 0; kind < 4; ++kind)
        modes[(kind * kNumPairClasses + r.X) * kNumPairClasses + r.Y] =
            kind < 2 ? r.mode[kind] : (r.split[kind - 2] ? r.mode32[kind - 2] : kNumModes);
  return IQCP_OK;
}

int iqcp_set_kernel_mode(iqcp_ctx* ctx, int kind, int X, int Y, int mode) {
  if (!ctx || kind < 0 || kind > 3 || mode < 0 || mode > kNumModes || (kind < 2 && mode == kNumModes))
    return IQCP_ERR_ARG;
  for (TaskRange& r : ctx->ranges) {
    if (!((X < 0 || r.X == X) && (Y < 0 || r.Y == Y))) continue;
    if (kind < 2) {
      r.mode[kind] = mode;
    } else if (mode == kNumModes) {
      r.split[kind - 2] = 0;
    } else {
      r.split[kind - 2] = 1;
      r.mode32[kind - 2] = mode;
    }
  }
  return IQCP_OK;
}

static int count_prim_quartets(iqcp_ctx* ctx) {
  if (!ctx->prim_quartets.empty()) return IQCP_OK;
  unsigned long long* d_cnt = nullptr;
  const size_t nr = ctx->ranges.size();
  CK(cudaMalloc(&d_cnt, sizeof(unsigned long long) * (nr + 1)));
  CK(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * (nr + 1), ctx->stream));
  for (size_t i = 0; i < nr; ++i) {
    const TaskRange& r = ctx->ranges[i];
    if (r.count == 0) continue;
    CK(launch_count_prim_quartets(ctx->d_pairs, ctx->d_pp, ctx->d_ket_list, ctx->d_tasks + r.first, r.count,
                                  ctx->opt.prim_threshold, d_cnt + i, ctx->stream));
  }
  std::vector<unsigned long long> h(nr + 1);
  CK(cudaMemcpyAsync(h.data(), d_cnt, sizeof(unsigned long long) * (nr + 1), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaFree(d_cnt));
  ctx->prim_quartets.assign(h.begin(), h.begin() + nr);
  return IQCP_OK;
}

// Closed-form algorithmic FLOP model per surviving primitive quartet of class
// (la lb|lc ld), counting the recurrences as the reference writes them
// (vrr_2d.rs:169-193, iterative transfer htr_4d.rs:107-224) -- FMA = 2:
//   F = 40 + sum_roots [17 + 3 VRR(nb,nk) + sum_comp (sum_axes HTR1(j,l) + 8)]
//   VRR(nb,nk) = 4 max(nb-1,0) + [nk>0](1 + 4(nk-1)) + 7 nb nk
//   HTR1(j,l)  = (j+1) l (l+1) + j (j+1)
// plus 12 per contracted integral for the 8-fold J/K digestion.  Gradient:
// tables extended by one on bra and ket, the reference's root count, and per component
// 4 centres x 3 axes of (2 HTR1 + 7), digested with 12 FMAs per component.
static double vrr_cost(int nb, int nk) {
  return 4.0 * (nb > 1 ? nb - 1 : 0) + (nk > 0 ? 1.0 + 4.0 * (nk - 1) : 0.0) + 7.0 * nb * nk;
}
static double htr1(int j, int l) { return double((j + 1) * l * (l + 1) + j * (j + 1)); }

static void class_cost(int X, int Y, bool grad, double* per_prim, double* per_quartet) {
  const int la = class_la(X), lb = class_lb(X), lc = class_la(Y), ld = class_lb(Y);
  const int L = la + lb + lc + ld;
  // the reference's root counts (eri/mod.rs:2146-2147 for the gradient): the
  // model counts the reference's work, whatever the kernels save
  const int nr = grad ? (L + 2) / 2 + 1 : L / 2 + 1;
  const int nb = la + lb + (grad ? 1 : 0), nk = lc + ld + (grad ? 1 : 0);
  double comp = 0.0;
  int ncomp = 0;
  for (int a = 0; a < ncart(la); ++a)
    for (int b = 0; b < ncart(lb); ++b)
      for (int c = 0; c < ncart(lc); ++c)
        for (int d = 0; d < ncart(ld); ++d) {
          ++ncomp;
          double s = 8.0;
          for (int ax = 0; ax < 3; ++ax) {
            const int j = cart_pow(lb, b, ax), l = cart_pow(ld, d, ax);
            s += htr1(j, l);
            // centres A, C shift i or k (cost of HTR1(j,l)); B shifts j; D shifts l
            if (grad) s += (2.0 * htr1(j, l) + 7.0) + (2.0 * htr1(j + 1, l) + 7.0) +
                           (2.0 * htr1(j, l) + 7.0) + (2.0 * htr1(j, l + 1) + 7.0);
          }
          comp += s;
        }
  *per_prim = 40.0 + nr * (17.0 + 3.0 * vrr_cost(nb, nk) + comp);
  *per_quartet = (grad ? 24.0 : 12.0) * ncomp;
}

int iqcp_model_flops(iqcp_ctx* ctx, int kind, double* flops_xy, long long* prim_xy, long long* quart_xy) {
  if (!ctx || !flops_xy) return IQCP_ERR_ARG;
  int rc = ensure_device(ctx);
  if (rc) return rc;
  rc = count_prim_quartets(ctx);
  if (rc) return rc;
  for (int i = 0; i < kNumPairClasses * kNumPairClasses; ++i) {
    flops_xy[i] = 0.0;
    if (prim_xy) prim_xy[i] = 0;
    if (quart_xy) quart_xy[i] = 0;
  }
  for (size_t i = 0; i < ctx->ranges.size(); ++i) {
    const TaskRange& r = ctx->ranges[i];
    double pp, pq;
    class_cost(r.X, r.Y, kind == 1, &pp, &pq);
    const int o = r.X * kNumPairClasses + r.Y;
    flops_xy[o] = pp * (double)ctx->prim_quartets[i] + pq * (double)r.quartets;
    if (prim_xy) prim_xy[o] = ctx->prim_quartets[i];
    if (quart_xy) quart_xy[o] = r.quartets;
  }
  return IQCP_OK;
}

int iqcp_measure_peak(int which, double* tflops) {
  if (!tflops) return IQCP_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return IQCP_ERR_NODEVICE;
  double flops = 0.0;
  float ms = 0.f;
  if (launch_fma_peak(which, &flops, &ms) != cudaSuccess) return IQCP_ERR_CUDA;
  *tflops = flops / (ms * 1e-3) * 1e-12;
  return IQCP_OK;
}

int iqcp_last_stats(const iqcp_ctx* ctx, double* s) {
  if (!ctx || !s) return IQCP_ERR_ARG;
  for (int i = 0; i < 4; ++i) s[i] = ctx->stats[i];
  return IQCP_OK;
}

static int batch_common(int n, const double* T) {
  if (n <= 0 || !T) return IQCP_ERR_ARG;
  for (int i = 0; i < n; ++i)
    if (!(T[i] >= 0.0) || !std::isfinite(T[i])) return IQCP_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return IQCP_ERR_NODEVICE;
  return IQCP_OK;
}

int iqcp_boys_batch(int m_max, int n, const double* T, double* F) {
  if (m_max < 0 || m_max > 31 || !F) return IQCP_ERR_ARG;
  int rc = batch_common(n, T);
  if (rc) return rc;
  double *dT = nullptr, *dF = nullptr;
  if (cudaMalloc(&dT, sizeof(double) * n) != cudaSuccess) return IQCP_ERR_NOMEM;
  if (cudaMalloc(&dF, sizeof(double) * n * (m_max + 1)) != cudaSuccess) { cudaFree(dT); return IQCP_ERR_NOMEM; }
  cudaMemcpy(dT, T, sizeof(double) * n, cudaMemcpyHostToDevice);
  cudaError_t e = launch_boys_batch(m_max, n, dT, dF, 0);
  if (e == cudaSuccess) e = cudaMemcpy(F, dF, sizeof(double) * n * (m_max + 1), cudaMemcpyDeviceToHost);
  cudaFree(dT);
  cudaFree(dF);
  return e == cudaSuccess ? IQCP_OK : IQCP_ERR_CUDA;
}

int iqcp_rys_batch(int nroots, int n, const double* T, double* roots, double* weights) {
  if (nroots < 1 || nroots > 7 || !roots || !weights) return IQCP_ERR_ARG;
  int rc = batch_common(n, T);
  if (rc) return rc;
  double *dT = nullptr, *dR = nullptr, *dW = nullptr;
  if (cudaMalloc(&dT, sizeof(double) * n) != cudaSuccess) return IQCP_ERR_NOMEM;
  if (cudaMalloc(&dR, sizeof(double) * n * nroots) != cudaSuccess) { cudaFree(dT); return IQCP_ERR_NOMEM; }
  if (cudaMalloc(&dW, sizeof(double) * n * nroots) != cudaSuccess) { cudaFree(dT); cudaFree(dR); return IQCP_ERR_NOMEM; }
  cudaMemcpy(dT, T, sizeof(double) * n, cudaMemcpyHostToDevice);
  cudaError_t e = launch_rys_batch(nroots, n, dT, dR, dW, 0);
  if (e == cudaSuccess) e = cudaMemcpy(roots, dR, sizeof(double) * n * nroots, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(weights, dW, sizeof(double) * n * nroots, cudaMemcpyDeviceToHost);
  cudaFree(dT);
  cudaFree(dR);
  cudaFree(dW);
  return e == cudaSuccess ? IQCP_OK : IQCP_ERR_CUDA;
}

}  // extern "C"
