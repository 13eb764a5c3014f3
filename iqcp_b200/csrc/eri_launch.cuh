// Launchers for one bra class (LA, LB) against every ket class Y <= X.
// Classes with many components use the warp-cooperative kernels
// (eri_team.cuh); the small ones keep one quartet per thread.
#pragma once
#include "eri_group.cuh"

namespace iqcp {


template <typename K>
inline cudaError_t set_smem(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Persistent grid: as many 128-thread blocks as are resident at once (capped
// by the work), each looping over tasks; per-block set-up (the staged Rys
// table, the gradient accumulator) is then paid once per resident block.
template <typename K>
inline int persistent_blocks(K kernel, size_t smem, int ntasks, int threads = 128) {
  int per_sm = 0, dev = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int wpb = threads / 32;
  const int need = (ntasks + wpb - 1) / wpb;
  const int cap = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  return need < cap ? need : cap;
}

#define IQCP_LAUNCH_T(KERNEL, THREADS, SMEM, ARGS, ST)                                             \
  do {                                                                                             \
    cudaError_t e_ = set_smem(KERNEL, SMEM);                                                       \
    if (e_ != cudaSuccess) return e_;                                                              \
    KERNEL<<<persistent_blocks(KERNEL, SMEM, (ARGS).ntasks, THREADS), THREADS, SMEM, ST>>>(ARGS); \
  } while (0)
#define IQCP_LAUNCH(KERNEL, SMEM, ARGS, ST) IQCP_LAUNCH_T(KERNEL, 128, SMEM, ARGS, ST)

// Team kernels walk a task's kets in one warp, one after the other.  A class
// with fewer tasks than twice the resident warps ((dd|dd) on a 40-atom
// molecule: ~700 tasks for ~1300 warps) would leave SMs idle and end on its
// longest task, so its tasks are split into 2, 4 or 8 slices of kets, each
// a work item of its own.
template <typename K>
inline int team_ket_split(K kernel, size_t smem, int ntasks, int threads) {
  int per_sm = 0, dev = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long warps = (long long)(per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1) * (threads / 32);
  int s = 1;
  while (s < 8 && (long long)ntasks * s < 2 * warps) s *= 2;
  return s;
}

#define IQCP_LAUNCH_TEAM(KERNEL, THREADS, SMEM, ARGS, ST)                                                \
  do {                                                                                                   \
    cudaError_t e_ = set_smem(KERNEL, SMEM);                                                             \
    if (e_ != cudaSuccess) return e_;                                                                    \
    (ARGS).ket_split = team_ket_split(KERNEL, SMEM, (ARGS).ntasks, THREADS);                             \
    KERNEL<<<persistent_blocks(KERNEL, SMEM, (ARGS).ntasks * (ARGS).ket_split, THREADS), THREADS, SMEM, \
             ST>>>(ARGS);                                                                                \
  } while (0)

// mode: 0 one quartet per thread, 1 warp-cooperative (eri_team.cuh),
// 2 / 3 eight / thirty-two lanes share one quartet's primitive quartets
// (J/K: small classes only; gradient: see launch_grad_variant; requests a
// class has no kernel for fall back to mode 0).  The FP32 share
// of a mixed call (pass 2) has modes 0 (up to 324 components), 1, and 2 for
// the small classes; other requests map onto those.
template <typename R, int LA, int LB, int LC, int LD>
cudaError_t launch_jk_variant(const JKArgs& a, cudaStream_t st) {
  using C = Cls<LA, LB, LC, LD>;
  constexpr bool F32 = sizeof(R) == 4;
  const size_t tb = sizeof(double) * rys_tab_doubles<C::NR>();
  const bool team = a.mode == 1 || (F32 && C::NCOMP > 324);
  if (team) {
    const size_t bytes = sizeof(double) * 4 * TeamJK<LA, LB, LC, LD>::PER_WARP + tb;
    JKArgs b = a;
    if (a.K) IQCP_LAUNCH_TEAM((jk_team_kernel<R, LA, LB, LC, LD, true>), 128, bytes, b, st);
    else IQCP_LAUNCH_TEAM((jk_team_kernel<R, LA, LB, LC, LD, false>), 128, bytes, b, st);
  } else if (C::NCOMP <= 27 && (a.mode == 2 || a.mode == 3)) {
    if constexpr (C::NCOMP <= 27) {
      if (a.mode == 2 || F32) {
        if (a.K) IQCP_LAUNCH((jk_kernel<R, LA, LB, LC, LD, 8, true>), tb, a, st);
        else IQCP_LAUNCH((jk_kernel<R, LA, LB, LC, LD, 8, false>), tb, a, st);
      } else {
        if (a.K) IQCP_LAUNCH((jk_kernel<R, LA, LB, LC, LD, 32, true>), tb, a, st);
        else IQCP_LAUNCH((jk_kernel<R, LA, LB, LC, LD, 32, false>), tb, a, st);
      }
    }
  } else if constexpr (!F32 || C::NCOMP <= 324) {
    if (a.K) IQCP_LAUNCH((jk_kernel<R, LA, LB, LC, LD, 1, true>), tb, a, st);
    else IQCP_LAUNCH((jk_kernel<R, LA, LB, LC, LD, 1, false>), tb, a, st);
  }
  return cudaGetLastError();
}

template <int LA, int LB, int LC, int LD>
cudaError_t launch_jk_class(const JKArgs& a, cudaStream_t st) {
  if (a.mx.pass == 2) return launch_jk_variant<float, LA, LB, LC, LD>(a, st);
  return launch_jk_variant<double, LA, LB, LC, LD>(a, st);
}

inline size_t max_smem_optin() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return (size_t)v;
}

// Gradient variants: mode 2 is one quartet per thread with the D x D weights
// in shared memory (classes of kWshMinComp..kWshMaxComp components; others map
// to mode 0), mode 3 the grouped kernel of eri_group.cuh (up to
// kGroupGradMaxComp components, 32 lanes per quartet; the FP32 share uses 8).
constexpr int kWshMinComp = 18, kWshMaxComp = 108;
constexpr int kGroupGradMaxComp = 108;

template <typename R, int LA, int LB, int LC, int LD>
cudaError_t launch_grad_variant(const GradArgs& args, cudaStream_t st) {
  using C = Cls<LA, LB, LC, LD>;
  constexpr bool F32 = sizeof(R) == 4;
  constexpr int NRG = grad_nroots(LA + LB + LC + LD);
  constexpr bool WSH_OK = !F32 && C::NCOMP >= kWshMinComp && C::NCOMP <= kWshMaxComp;
  using TG = TeamGrad2<LA, LB, LC, LD>;
  const bool team = args.mode == 1 || (F32 && C::NCOMP > 324);
  const bool wsh = !team && args.mode == 2 && WSH_OK;
  const bool group = !team && !wsh && (args.mode == 3 || (F32 && args.mode == 2)) && C::NCOMP <= kGroupGradMaxComp;
  // the team variant reads the Rys coefficients through L1 (no staged table)
  size_t fixed = sizeof(double) * rys_tab_doubles<NRG>();
  if (team) fixed = sizeof(double) * TG::WPB * TG::PER_WARP;
  else if (wsh)
    fixed = sizeof(double) * (grad_stages_rys<LA, LB, LC, LD, true>() ? rys_tab_doubles<NRG>() : 0) +
            sizeof(R) * grad_wsh_doubles<LA, LB, LC, LD>();
  else if (group)
    fixed += sizeof(double) * (F32 ? GroupGrad<R, LA, LB, LC, LD, 8>::WDOUBLES : GroupGrad<R, LA, LB, LC, LD, 32>::WDOUBLES);
  // the per-block gradient accumulator only when it fits beside the tables
  GradArgs a = args;
  if (a.gsmem && fixed + sizeof(double) * 3 * a.natoms > max_smem_optin()) a.gsmem = 0;
  const size_t gacc = a.gsmem ? sizeof(double) * 3 * a.natoms : 0;
  const size_t bytes = fixed + gacc;
  if (team) {
    IQCP_LAUNCH_TEAM((grad_team2_kernel<R, LA, LB, LC, LD>), 32 * TG::WPB, bytes, a, st);
  } else if (wsh) {
    if constexpr (WSH_OK) IQCP_LAUNCH((grad_kernel<R, LA, LB, LC, LD, 1, true>), bytes, a, st);
  } else if (group) {
    if constexpr (C::NCOMP <= kGroupGradMaxComp) {
      if (F32) IQCP_LAUNCH((grad_group_kernel<R, LA, LB, LC, LD, 8>), bytes, a, st);
      else IQCP_LAUNCH((grad_group_kernel<R, LA, LB, LC, LD, 32>), bytes, a, st);
    }
  } else if constexpr (!F32 || C::NCOMP <= 324) {
    IQCP_LAUNCH((grad_kernel<R, LA, LB, LC, LD, 1>), bytes, a, st);
  }
  return cudaGetLastError();
}

template <int LA, int LB, int LC, int LD>
cudaError_t launch_grad_class(const GradArgs& a, cudaStream_t st) {
  if (a.mx.pass == 2) return launch_grad_variant<float, LA, LB, LC, LD>(a, st);
  return launch_grad_variant<double, LA, LB, LC, LD>(a, st);
}

#define IQCP_KET_DISPATCH(X, Y, MACRO)                \
  switch (Y) {                                        \
    case 0: MACRO(0, 0); break;                       \
    case 1: if (X >= 1) { MACRO(1, 0); } break;       \
    case 2: if (X >= 2) { MACRO(1, 1); } break;       \
    case 3: if (X >= 3) { MACRO(2, 0); } break;       \
    case 4: if (X >= 4) { MACRO(2, 1); } break;       \
    case 5: if (X >= 5) { MACRO(2, 2); } break;       \
    default: return cudaErrorInvalidValue;            \
  }

template <int LA, int LB>
cudaError_t launch_jk_bra(int Y, const JKArgs& a, cudaStream_t st) {
  constexpr int X = pair_class(LA, LB);
#define LJK(lc, ld) \
  if constexpr (pair_class(lc, ld) <= X) { return launch_jk_class<LA, LB, lc, ld>(a, st); }
  IQCP_KET_DISPATCH(X, Y, LJK)
#undef LJK
  return cudaErrorInvalidValue;
}

template <int LA, int LB>
cudaError_t launch_store_bra(int Y, const StoreArgs& a, cudaStream_t st) {
  constexpr int X = pair_class(LA, LB);
  const int blocks = (a.ntasks + 3) / 4;
#define LST(lc, ld) \
  if constexpr (pair_class(lc, ld) <= X) { store_kernel<LA, LB, lc, ld><<<blocks, 128, 0, st>>>(a); }
  IQCP_KET_DISPATCH(X, Y, LST)
#undef LST
  return cudaGetLastError();
}

template <int LA, int LB>
cudaError_t launch_grad_bra(int Y, const GradArgs& a, cudaStream_t st) {
  constexpr int X = pair_class(LA, LB);
#define LGR(lc, ld) \
  if constexpr (pair_class(lc, ld) <= X) { return launch_grad_class<LA, LB, lc, ld>(a, st); }
  IQCP_KET_DISPATCH(X, Y, LGR)
#undef LGR
  return cudaErrorInvalidValue;
}

}  // namespace iqcp
