// Fused-step kernels (scalar, vectorised, TMA row-staged) and their launch
// logic.  Included by lbm_flow.cu (declarations only) and by
// lbm_step_inst.cu, which the build compiles once per (velocity set,
// storage) with -DLBM_Q / -DLBM_S.
#pragma once
#include <algorithm>

#include "lbm_api.cuh"
#include "lbm_tma.cuh"

namespace lbm {

constexpr int kThreads = 256;

// ---------------------------------------------------------------------------
// Fused step
// ---------------------------------------------------------------------------
struct StepArgs {
  Geom g;
  NodeDecomp dec;    // dense node index -> (x, y, z)
  NodeDecomp pdec;   // population index (x ny + y) pz + z -> (x, y, z)
  const void *fa;
  void *fb;
  float go[3], gn[3];
  // fields, face densities and observation buffers hold the storage's
  // arithmetic type (float64 for LBM_STORAGE_FP64, float32 otherwise)
  const void *fol_old, *fol_new;
  const uint8_t *ch_old, *ch_new;
  const void *face_rho_in;
  void *face_rho_out;
  void *obs_f, *obs_rho, *obs_u;
  unsigned *status;
  StepPlanes p;
};

template <int Q, typename R>
__device__ __forceinline__ void write_face_rho(const Geom &g, R *out, int x, int y, int z, R rho) {
  if (x == 0) out[plane_index(g, 0, x, y, z)] = rho;
  if (x == g.nx - 1) out[plane_index(g, 1, x, y, z)] = rho;
  if (y == 0) out[plane_index(g, 2, x, y, z)] = rho;
  if (y == g.ny - 1) out[plane_index(g, 3, x, y, z)] = rho;
  if (z == 0) out[plane_index(g, 4, x, y, z)] = rho;
  if (z == g.nz - 1) out[plane_index(g, 5, x, y, z)] = rho;
}

template <typename R>
__device__ __forceinline__ unsigned bad_bits(R rho, R ux, R uy, R uz) {
  unsigned b = 0;
  if (!(rho > R(0)) || !(rho < R(3.0e38))) b |= LBM_STATUS_RHO_BAD;
  if (!(fabs(ux) + fabs(uy) + fabs(uz) < R(3.0e38))) b |= LBM_STATUS_U_BAD;
  return b;
}

// Everything after the pull for one node: the previous / new forcing, the
// moment passes, cul_equ2, status bits (accumulated in `bad`), face
// densities, observation, and (when fb is set) the next step's collision, in
// place in f.  DEV: f holds deviations d = f - w (shifted storage), handled
// by dev_moments / collide_dev.
// Whether the previous / this step's force field applies in the 32-node
// chunk of node idx.  A thread's nodes always share one chunk, so the kernels
// read the flags once, before their population loads.
struct ChunkForce {
  bool old_here, new_here;
};

template <bool FORCE>
__device__ __forceinline__ ChunkForce chunk_force(const StepArgs &a, unsigned idx) {
  ChunkForce c{false, false};
  if constexpr (FORCE) {
    c.old_here = a.fol_old != nullptr && (a.ch_old == nullptr || a.ch_old[idx >> 5]);
    c.new_here = a.fol_new != nullptr && (a.ch_new == nullptr || a.ch_new[idx >> 5]);
  }
  return c;
}

// finish_node_m also hands the node's end-of-step moments (the second
// update_u_rou) to the caller.
template <int Q, bool FORCE, bool DEV, int SH, typename R>
__device__ __forceinline__ void finish_node_m(const StepArgs &a, R f[Q], unsigned idx, int x,
                                              int y, int z, bool face, ChunkForce cf,
                                              unsigned &bad, R &rho_out, R &ux_out, R &uy_out,
                                              R &uz_out) {
  using V = VSet<Q>;
  R fox = a.go[0], foy = a.go[1], foz = a.go[2];
  R fnx = a.gn[0], fny = a.gn[1], fnz = a.gn[2];
  if (cf.old_here) {
    const R *fol = static_cast<const R *>(a.fol_old);
    fox += fol[3ull * idx];
    foy += fol[3ull * idx + 1];
    foz += fol[3ull * idx + 2];
  }
  if (cf.new_here) {
    const R *fol = static_cast<const R *>(a.fol_new);
    fnx += fol[3ull * idx];
    fny += fol[3ull * idx + 1];
    fnz += fol[3ull * idx + 2];
  }
  R rho, drho = R(0), ux, uy, uz;
  if constexpr (DEV)
    dev_moments<Q, SH>(f, fox, foy, foz, face, rho, drho, ux, uy, uz);
  else
    moments<Q>(f, fox, foy, foz, face, rho, ux, uy, uz);
  // Where both the previous and this step's force are zero (everywhere
  // outside the spread chunks when there is no uniform force) cul_equ2 adds
  // nothing and the second moment pass repeats the first, so such nodes skip
  // them -- the same rule in every kernel.  (A zero new force alone is not
  // enough: the second pass drops the previous force from u.)
  if (FORCE && (fnx != R(0) || fny != R(0) || fnz != R(0) || fox != R(0) || foy != R(0) ||
                foz != R(0))) {
    add_force<Q, SH>(f, a.g, ux, uy, uz, fnx, fny, fnz);
    if constexpr (DEV)
      dev_moments<Q, SH>(f, fnx, fny, fnz, face, rho, drho, ux, uy, uz);
    else
      moments<Q>(f, fnx, fny, fnz, face, rho, ux, uy, uz);
  }
  bad |= bad_bits(rho, ux, uy, uz);
  if (face && a.face_rho_out != nullptr)
    write_face_rho<Q>(a.g, static_cast<R *>(a.face_rho_out), x, y, z, rho);
  if (a.obs_f != nullptr) {
    R *of = static_cast<R *>(a.obs_f);
    static_for<Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      of[(long long)i * a.g.n + idx] =
          DEV ? f[i] * (R(1) / R(1 << SH)) + V::template wr<R>(i) : f[i];
    });
  }
  if (a.obs_rho != nullptr) static_cast<R *>(a.obs_rho)[idx] = rho;
  if (a.obs_u != nullptr) {
    R *ou = static_cast<R *>(a.obs_u);
    ou[3ull * idx] = ux;
    ou[3ull * idx + 1] = uy;
    ou[3ull * idx + 2] = uz;
  }
  rho_out = rho;
  ux_out = ux;
  uy_out = uy;
  uz_out = uz;
  if (a.fb != nullptr) {
    if constexpr (DEV)
      collide_dev<Q, SH>(f, a.g, rho, drho, ux, uy, uz);
    else
      collide<Q>(f, a.g, rho, ux, uy, uz);
  }
}

template <int Q, bool FORCE, bool DEV, int SH, typename R>
__device__ __forceinline__ void finish_node(const StepArgs &a, R f[Q], unsigned idx, int x,
                                            int y, int z, bool face, ChunkForce cf,
                                            unsigned &bad) {
  R rho, ux, uy, uz;
  finish_node_m<Q, FORCE, DEV, SH>(a, f, idx, x, y, z, face, cf, bad, rho, ux, uy, uz);
}

__device__ __forceinline__ void report_bad(unsigned *status, unsigned bad) {
  if (bad != 0 && status != nullptr) atomicOr(status, bad);
}

// Row padding of a pitched lattice (population index p, p + 1, ... up to the
// row's pitch) is written by the kernel that writes the row's last node,
// with any value: it is never a pull source and never observed, but a
// 32-byte sector that a step writes only in part makes L2 fetch the rest
// from DRAM before it can write the sector back (measured on B200 at 257^3
// in FP32: +2 % DRAM reads and 16 % longer steps while the padding was left
// unwritten).
template <int Q, int S>
__device__ __forceinline__ void put_row_padding(const StepArgs &a, unsigned p, int count,
                                                const typename Storage<S>::R f[Q]) {
  using St = Storage<S>;
  using T = typename St::T;
#pragma unroll 1
  for (int j = 0; j < count; ++j) {
    static_for<Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      St::put(static_cast<T *>(a.p.dst[i]) + p + j, f[i]);
    });
  }
}

// A vector of padding only (a pitched row's last vector, past its nodes):
// zero words, stored for the same reason.
template <int Q, int S, int NZ>
__device__ __forceinline__ void put_padding_vector(const StepArgs &a, unsigned pidx0) {
  using St = Storage<S>;
  using T = typename St::T;
  constexpr int kWords = NZ * St::kBits / 32;
  if (a.fb == nullptr) return;
  Words<kWords> zero;
#pragma unroll
  for (int k = 0; k < kWords; ++k) zero.w[k] = 0u;
  static_for<Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    st_words(static_cast<T *>(a.p.dst[i]) + pidx0, zero);
  });
}

// One node per thread, nodes in memory order so that each warp owns one
// 32-node chunk.  Rows with interior (x, y) pull through pull_row_node;
// rows on an x / y face take the general face rules.  FORCE adds cul_equ2
// and the second moment pass; without it both are exact no-ops (the
// reference adds zeros and recomputes identical moments), so they are
// skipped.
template <int Q, int S, bool FORCE>
__device__ __forceinline__ void step_scalar_body(const StepArgs &a, const unsigned idx) {
  using St = Storage<S>;
  using T = typename St::T;
  if (idx >= (unsigned)a.g.n) return;
  int x, y, z;
  const ChunkForce cf = chunk_force<FORCE>(a, idx);
  a.dec(idx, x, y, z);
  const unsigned pidx = (unsigned)(x * a.g.ny + y) * (unsigned)a.g.pz + (unsigned)z;
  if (!lbm_in(x < a.g.nx && y < a.g.ny && z < a.g.nz && pidx < (unsigned)a.g.np)) return;
  using R = typename St::R;
  const R *face_rho = static_cast<const R *>(a.face_rho_in);
  const bool row_in = x > 0 && x < a.g.nx - 1 && y > 0 && y < a.g.ny - 1;
  R f[Q];
  if (row_in)
    pull_row_node<Q, S, true>(a.p, a.g, face_rho, pidx, x, y, z, f);
  else
    pull_general<Q, S, true>(static_cast<const T *>(a.fa), a.g, x, y, z, face_rho, f);
  unsigned bad = 0;
  finish_node<Q, FORCE, St::kDev, St::kShift>(a, f, idx, x, y, z, !row_in || z == 0 || z == a.g.nz - 1, cf,
                                  bad);
  report_bad(a.status, bad);
  if (a.fb != nullptr) {
    static_for<Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      St::put(static_cast<T *>(a.p.dst[i]) + pidx, f[i]);
    });
    if (z == a.g.nz - 1 && a.g.pz > a.g.nz)
      put_row_padding<Q, S>(a, pidx + 1, a.g.pz - a.g.nz, f);
  }
}

// Register cap of the one-node kernel (resident blocks per SM asked of the
// compiler, 0 = none).  The one-node kernel runs the rows of odd length (the
// reference's size + 1 nodes) and is latency-bound there: an ncu capture of
// the forced D3Q27 FP32 step on 257 x 129 x 129 nodes showed 74 registers,
// 3 resident blocks of 256 (24 warps / SM) and 7.7 long-scoreboard stalls
// per issue.  D3Q19 in FP32 and 16-bit storage: 48 registers (5 blocks; the
// forced 16-bit kernel spills a few words); D3Q27 in FP32 and 16-bit: 64
// registers (4 blocks), no spills.
template <int Q, int S>
constexpr int scalar_min_blocks() {
  constexpr int bits = Storage<S>::kBits;
  if (bits == 64) return 0;
  if (Q == 19) return 5;
  if (Q == 27) return 4;
  return 0;
}

template <int Q, int S, bool FORCE>
__global__ void __launch_bounds__(kThreads, (scalar_min_blocks<Q, S>())) k_step(const __grid_constant__ StepArgs a) {
  chain_enter();
  step_scalar_body<Q, S, FORCE>(a, blockIdx.x * kThreads + threadIdx.x);
}

// ---------------------------------------------------------------------------
// Step statistics: min / sum / max of f, u and rho at the end of the step the
// populations `fa` stream into (FlowD3.to_json, flow/base.py:183-206, as
// LBMBase._log_step_info logs it, lbm/base.py:105-144), in one read of the
// populations and nothing written but 9 numbers.  Grid-stride, one node per
// thread per iteration; per-block reduction, then one atomic per quantity
// and block into `out`: min / max as order-preserving 64-bit keys of the
// doubles, sums as doubles (k_stats_finish turns them into min, mean, max).
// ---------------------------------------------------------------------------
constexpr int kStatsThreads = 256;

__device__ __forceinline__ unsigned long long ordered_bits(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ double from_ordered_bits(unsigned long long o) {
  const unsigned long long b = (o >> 63) ? (o & 0x7fffffffffffffffull) : ~o;
  return __longlong_as_double((long long)b);
}

struct StatAcc {
  double mn[3], sm[3], mx[3];
};

__device__ __forceinline__ void stat_add(StatAcc &s, int k, double v) {
  s.mn[k] = fmin(s.mn[k], v);
  s.mx[k] = fmax(s.mx[k], v);
  s.sm[k] += v;
}

template <int Q, int S, bool FORCE>
__global__ void __launch_bounds__(kStatsThreads) k_stats(const __grid_constant__ StepArgs a,
                                                         unsigned long long *out) {
  using St = Storage<S>;
  using T = typename St::T;
  using R = typename St::R;
  using V = VSet<Q>;
  __shared__ StatAcc sh[kStatsThreads / 32];
  StatAcc acc;
  for (int k = 0; k < 3; ++k) {
    acc.mn[k] = INFINITY;
    acc.mx[k] = -INFINITY;
    acc.sm[k] = 0.0;
  }
  const R *face_rho = static_cast<const R *>(a.face_rho_in);
  unsigned bad = 0;
  for (unsigned idx = blockIdx.x * kStatsThreads + threadIdx.x; idx < (unsigned)a.g.n;
       idx += gridDim.x * kStatsThreads) {
    int x, y, z;
    const ChunkForce cf = chunk_force<FORCE>(a, idx);
    a.dec(idx, x, y, z);
    const bool row_in = x > 0 && x < a.g.nx - 1 && y > 0 && y < a.g.ny - 1;
    const unsigned pidx = (unsigned)(x * a.g.ny + y) * (unsigned)a.g.pz + (unsigned)z;
    if (!lbm_in(x < a.g.nx && y < a.g.ny && z < a.g.nz && pidx < (unsigned)a.g.np)) continue;
    R f[Q];
    if (row_in)
      pull_row_node<Q, S, true>(a.p, a.g, face_rho, pidx, x, y, z, f);
    else
      pull_general<Q, S, true>(static_cast<const T *>(a.fa), a.g, x, y, z, face_rho, f);
    R rho, ux, uy, uz;
    finish_node_m<Q, FORCE, St::kDev, St::kShift>(a, f, idx, x, y, z, !row_in || z == 0 || z == a.g.nz - 1,
                                      cf, bad, rho, ux, uy, uz);
    R fmn = R(INFINITY), fmx = -R(INFINITY);
    double fsum = 0.0;
    static_for<Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      const R v = St::kDev ? f[i] * (R(1) / R(1 << St::kShift)) + V::template wr<R>(i) : f[i];
      fsum += (double)v;
      fmn = fmin(fmn, v);
      fmx = fmax(fmx, v);
    });
    acc.mn[0] = fmin(acc.mn[0], (double)fmn);
    acc.mx[0] = fmax(acc.mx[0], (double)fmx);
    acc.sm[0] += fsum;
    stat_add(acc, 1, (double)ux);
    stat_add(acc, 1, (double)uy);
    stat_add(acc, 1, (double)uz);
    stat_add(acc, 2, (double)rho);
  }
  report_bad(a.status, bad);
  for (int k = 0; k < 3; ++k) {
    for (int o = 16; o > 0; o >>= 1) {
      acc.mn[k] = fmin(acc.mn[k], __shfl_xor_sync(0xffffffffu, acc.mn[k], o));
      acc.mx[k] = fmax(acc.mx[k], __shfl_xor_sync(0xffffffffu, acc.mx[k], o));
      acc.sm[k] += __shfl_xor_sync(0xffffffffu, acc.sm[k], o);
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    StatAcc t = sh[0];
    for (int w = 1; w < kStatsThreads / 32; ++w)
      for (int k = 0; k < 3; ++k) {
        t.mn[k] = fmin(t.mn[k], sh[w].mn[k]);
        t.mx[k] = fmax(t.mx[k], sh[w].mx[k]);
        t.sm[k] += sh[w].sm[k];
      }
    for (int k = 0; k < 3; ++k) {
      atomicMin(out + 3 * k, ordered_bits(t.mn[k]));
      atomicAdd(reinterpret_cast<double *>(out + 3 * k + 1), t.sm[k]);
      atomicMax(out + 3 * k + 2, ordered_bits(t.mx[k]));
    }
  }
}

// slots of the 9 statistics: min / max keys of +inf / -inf, sums 0 (a
// template, instantiated beside each k_stats, so that every translation unit
// that includes this header may carry it)
template <int Q>
__global__ void k_stats_init(unsigned long long *out) {
  const int k = threadIdx.x;
  if (k >= 9) return;
  const int c = k % 3;
  out[k] = c == 0 ? ordered_bits(INFINITY)
                  : c == 2 ? ordered_bits(-INFINITY) : (unsigned long long)__double_as_longlong(0.0);
}

// in place: keys -> min / max, sums -> means over n*q, 3n and n values
template <int Q>
__global__ void k_stats_finish(unsigned long long *out, double n) {
  const int k = threadIdx.x;
  if (k >= 9) return;
  const int c = k % 3;
  double v;
  if (c == 1) {
    const double count = k == 1 ? n * Q : k == 4 ? 3.0 * n : n;
    v = __longlong_as_double((long long)out[k]) / count;
  } else {
    v = from_ordered_bits(out[k]);
  }
  reinterpret_cast<double *>(out)[k] = v;
}

// ---------------------------------------------------------------------------
// Vectorised fused step: thread = NZ consecutive nodes of one z-row (nz a
// multiple of NZ), populations moved as NZ-element vectors (16 / 8 / 4 byte
// loads and stores).  For rows whose (x, y) is interior every source of
// direction i lies in row (x - ex, y - ey): one aligned vector load gives
// NZ - |ez| of the NZ values, one scalar load the remaining one -- from the
// neighbouring vector, or at z = 0 / z = nz - 1 from the bottom / top face
// rule, picked by an address select so that all loads issue together.
// Rows on an x / y face take the per-node face rules (face_row_nodes).
// ---------------------------------------------------------------------------
// Whether a vector kernel processes face rows node by node (face_row_nodes)
// or unrolled with the rest: node by node makes the kernel ~40 % smaller,
// which measured faster on B200 for the forced kernels and for D3Q13 in
// 16-bit storage, and slower for the other unforced ones.
template <int Q, int S, bool FORCE>
__host__ __device__ constexpr bool compact_face_rows() {
  return FORCE || (Q == 13 && Storage<S>::kBits == 16);
}

// Nodes of a row on an x / y face (under 1 % of a large lattice), or the
// last nodes of a pitched row under a WALL_WITH_SPEED top face: one at a
// time through the general face rules, in a loop that is not unrolled and a
// function that is not inlined, so a vector kernel carries one copy of this
// code however many places call it (it is reached from two).  The kernels
// take their StepArgs as __grid_constant__ parameters, so the reference it
// receives points at the parameter itself (no per-thread copy).  Same
// per-node arithmetic.  idx0 / pidx0: dense / population index of node (x, y, z0).
template <int Q, int S, bool FORCE>
__device__ __forceinline__ void face_row_nodes(const StepArgs &a, unsigned idx0, unsigned pidx0,
                                            int count, int pad, int x, int y, int z0) {
  using St = Storage<S>;
  using T = typename St::T;
  using R = typename St::R;
  const T *fa = static_cast<const T *>(a.fa);
  const R *face_rho = static_cast<const R *>(a.face_rho_in);
  unsigned bad = 0;
#pragma unroll 1
  for (int k = 0; k < count; ++k) {
    if (!lbm_in(z0 + k < a.g.nz && pidx0 + k < (unsigned)a.g.np && idx0 + k < (unsigned)a.g.n))
      continue;
    R f[Q];
    pull_general<Q, S, true>(fa, a.g, x, y, z0 + k, face_rho, f);
    // the nodes may lie in two chunks
    finish_node<Q, FORCE, St::kDev, St::kShift>(a, f, idx0 + k, x, y, z0 + k, on_any_face(a.g, x, y, z0 + k),
                                    chunk_force<FORCE>(a, idx0 + k), bad);
    if (a.fb != nullptr) {
      static_for<Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        St::put(static_cast<T *>(a.p.dst[i]) + pidx0 + k, f[i]);
      });
      if (k == count - 1 && pad > 0) put_row_padding<Q, S>(a, pidx0 + count, pad, f);
    }
  }
  report_bad(a.status, bad);
}

// 16-bit storage: the vectors stay packed in registers and are unpacked one
// node pair at a time, right before that pair is finished and stored (one
// 32-bit word per direction), so a thread holds 2 x Q floats instead of
// NZ x Q.  Measured on B200 it is the faster form for 2 nodes per thread
// (fewer registers, more resident warps); for 4 and 8 the fully unpacked
// form below keeps more independent work per thread and wins.  Same
// arithmetic per node as every other shape.
// ALIGNED = false: the pair starts at any index (rows of odd length), so
// its elements are loaded and stored one by one and its nodes may lie in two
// different force chunks.
template <int Q, int S, bool FORCE, int NZ, bool COMPACT, bool ALIGNED = true, bool PITCH = false>
__device__ __forceinline__ void step_vec_pairs_at(const StepArgs &a, const unsigned pidx0) {
  using St = Storage<S>;
  using T = typename St::T;
  using V = VSet<Q>;
  static_assert(St::kBits == 16 && NZ % 2 == 0, "pairs of 16-bit elements");
  static_assert(ALIGNED || NZ == 2, "unaligned pairs are single pairs");
  constexpr int kWords = NZ / 2;
  if (pidx0 >= (unsigned)a.g.np) return;
  int x, y, z0;
  a.pdec(pidx0, x, y, z0);
  if constexpr (PITCH) {
    if (z0 >= a.g.nz) {                      // row padding only
      put_padding_vector<Q, S, NZ>(a, pidx0);
      return;
    }
  }
  const unsigned idx0 = (unsigned)(x * a.g.ny + y) * (unsigned)a.g.nz + (unsigned)z0;
  // nodes inside the row (fewer than NZ in the last vector of a pitched row:
  // the other lanes are padding, loaded and stored but not finished)
  const int nv = PITCH && a.g.nz - z0 < NZ ? a.g.nz - z0 : NZ;
  if (PITCH && nv < NZ && a.g.face[5] == LBM_BC_WALL_WITH_SPEED) {
    face_row_nodes<Q, S, FORCE>(a, idx0, pidx0, nv, NZ - nv, x, y, z0);
    return;
  }
  if (!lbm_in(x < a.g.nx && y < a.g.ny && pidx0 + NZ <= (unsigned)a.g.np &&
              idx0 + nv <= (unsigned)a.g.n))
    return;
  constexpr bool kCompact = COMPACT;
  bool row_in = x > 0 && x < a.g.nx - 1 && y > 0 && y < a.g.ny - 1;
  if constexpr (kCompact) {
    if (!row_in) {
      face_row_nodes<Q, S, FORCE>(a, idx0, pidx0, nv, NZ - nv, x, y, z0);
      return;
    }
    row_in = true;
  }
  const bool bottom = z0 == 0, top = z0 + NZ >= a.g.nz;
  // lane of the row's last node when it lies inside this vector (else NZ)
  const int last = nv < NZ ? nv - 1 : NZ;
  Words<kWords> raw[Q];
  T extra[Q];
  if (row_in) {
    static_for<Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      constexpr int ez = V::ez(i);
      const T *ps = static_cast<const T *>(a.p.src[i]) + pidx0;
      if constexpr (ALIGNED)
        raw[i] = ld_words<kWords>(ps);
      else
        raw[i].w[0] = (unsigned)bits16(St::raw(ps)) | ((unsigned)bits16(St::raw(ps + 1)) << 16);
      if constexpr (ez > 0)
        extra[i] = St::raw(bottom ? static_cast<const T *>(a.p.zlo[i]) + pidx0 : ps - 1);
      if constexpr (ez < 0)
        extra[i] = St::raw(top ? static_cast<const T *>(a.p.zhi[i]) + (pidx0 + (nv - 1)) : ps + NZ);
    });
  }
  unsigned bad = 0;
#pragma unroll
  for (int pr = 0; pr < kWords; ++pr) {
    float f0[Q], f1[Q];
    const int za = z0 + 2 * pr;
    if (row_in) {
      static_for<Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        constexpr int ez = V::ez(i);
        const float2 v = work2<S>(raw[i].w[pr]);
        if constexpr (ez == 0) {
          f0[i] = v.x;
          f1[i] = v.y;
        } else if constexpr (ez > 0) {
          f0[i] = pr == 0 ? St::cvt(extra[i]) : work2<S>(raw[i].w[pr > 0 ? pr - 1 : 0]).y;
          f1[i] = v.x;
        } else {
          // (the row's last node pulls the top face's value; a padding lane
          // after it keeps any value: it is not finished)
          f0[i] = 2 * pr == last ? St::cvt(extra[i]) : v.y;
          f1[i] = pr == kWords - 1 || 2 * pr + 1 == last
                      ? St::cvt(extra[i])
                      : work2<S>(raw[i].w[pr < kWords - 1 ? pr + 1 : pr]).x;
        }
      });
      if (pr == 0 && bottom && a.g.face[4] == LBM_BC_WALL_WITH_SPEED)
        zface_wws<Q, 4, St::kShift>(a.g, static_cast<const float *>(a.face_rho_in), x, y, 0, f0);
      if (pr == kWords - 1 && top && a.g.face[5] == LBM_BC_WALL_WITH_SPEED)
        zface_wws<Q, 5, St::kShift>(a.g, static_cast<const float *>(a.face_rho_in), x, y, a.g.nz - 1, f1);
    } else if constexpr (!kCompact) {
      const T *fa = static_cast<const T *>(a.fa);
      const float *face_rho = static_cast<const float *>(a.face_rho_in);
      // (padding lanes repeat the row's last node; they are not finished)
      pull_general<Q, S, true>(fa, a.g, x, y, 2 * pr < nv ? za : a.g.nz - 1, face_rho, f0);
      pull_general<Q, S, true>(fa, a.g, x, y, 2 * pr + 1 < nv ? za + 1 : a.g.nz - 1, face_rho, f1);
    }
    // (a pair may straddle two force chunks: dense rows of any length)
    if (2 * pr < nv)
      finish_node<Q, FORCE, true, St::kShift>(a, f0, idx0 + 2 * pr, x, y, za,
                                  !row_in || za == 0 || za == a.g.nz - 1,
                                  chunk_force<FORCE>(a, idx0 + 2 * pr), bad);
    if (2 * pr + 1 < nv)
      finish_node<Q, FORCE, true, St::kShift>(a, f1, idx0 + 2 * pr + 1, x, y, za + 1,
                                  !row_in || za + 1 == a.g.nz - 1,
                                  chunk_force<FORCE>(a, idx0 + 2 * pr + 1), bad);
    if (a.fb != nullptr) {
      static_for<Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        T *dst = static_cast<T *>(a.p.dst[i]) + pidx0 + 2 * pr;
        const unsigned word = put2<S>(f0[i], f1[i]);
        if constexpr (ALIGNED) {
          st_words(dst, Words<1>{{word}});
        } else {
          reinterpret_cast<unsigned short *>(dst)[0] = (unsigned short)(word & 0xffffu);
          reinterpret_cast<unsigned short *>(dst)[1] = (unsigned short)(word >> 16);
        }
      });
    }
  }
  report_bad(a.status, bad);
}

template <int Q, int S, bool FORCE, int NZ, bool COMPACT, bool PITCH>
__device__ __forceinline__ void step_vec_pairs(const StepArgs &a, const unsigned t) {
  step_vec_pairs_at<Q, S, FORCE, NZ, COMPACT, true, PITCH>(a, t * NZ);
}


// PITCH: rows may carry padding (pz > nz) -- the kernel then handles a
// partial last vector per row and writes the padding; lattices without
// padding run the variant that has none of that code.
template <int Q, int S, bool FORCE, int NZ, bool PITCH,
          bool COMPACT = compact_face_rows<Q, S, FORCE>()>
__device__ __forceinline__ void step_vec_body(const StepArgs &a, const unsigned t) {
  using St = Storage<S>;
  using T = typename St::T;
  using V = VSet<Q>;
  if constexpr (St::kBits == 16 && NZ == 2) {
    step_vec_pairs<Q, S, FORCE, NZ, COMPACT, PITCH>(a, t);
    return;
  }
  using R = typename St::R;
  constexpr int kWords = NZ * St::kBits / 32;
  const unsigned pidx0 = t * NZ;
  if (pidx0 >= (unsigned)a.g.np) return;
  int x, y, z0;
  a.pdec(pidx0, x, y, z0);
  if constexpr (PITCH) {
    if (z0 >= a.g.nz) {                      // row padding only
      put_padding_vector<Q, S, NZ>(a, pidx0);
      return;
    }
  }
  const unsigned idx0 = (unsigned)(x * a.g.ny + y) * (unsigned)a.g.nz + (unsigned)z0;
  // Nodes of this vector inside the row: fewer than NZ in the last vector of
  // a pitched row, whose other lanes are row padding -- loaded and stored
  // with the vector (never a pull source, never observed) but not finished.
  const int nv = PITCH && a.g.nz - z0 < NZ ? a.g.nz - z0 : NZ;
  if (PITCH && nv < NZ && a.g.face[5] == LBM_BC_WALL_WITH_SPEED) {
    face_row_nodes<Q, S, FORCE>(a, idx0, pidx0, nv, NZ - nv, x, y, z0);
    return;
  }
  if (!lbm_in(x < a.g.nx && y < a.g.ny && pidx0 + NZ <= (unsigned)a.g.np &&
              idx0 + nv <= (unsigned)a.g.n))
    return;
  constexpr bool kCompact = COMPACT;
  bool row_in = x > 0 && x < a.g.nx - 1 && y > 0 && y < a.g.ny - 1;
  if constexpr (kCompact) {
    if (!row_in) {
      face_row_nodes<Q, S, FORCE>(a, idx0, pidx0, nv, NZ - nv, x, y, z0);
      return;
    }
    row_in = true;
  }
  const R *face_rho = static_cast<const R *>(a.face_rho_in);
  R f[NZ][Q];
  if (row_in) {
    // top: the row's last node is in this vector (lane nv - 1)
    const bool bottom = z0 == 0, top = z0 + NZ >= a.g.nz;
    static_for<Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      constexpr int ez = V::ez(i);
      const T *ps = static_cast<const T *>(a.p.src[i]) + pidx0;
      const Words<kWords> raw = ld_words<kWords>(ps);
      R v[NZ];
      if constexpr (St::kBits == 32) {
#pragma unroll
        for (int k = 0; k < NZ; ++k) v[k] = __uint_as_float(raw.w[k]);
      } else if constexpr (St::kBits == 64) {
#pragma unroll
        for (int k = 0; k < NZ; ++k) v[k] = __hiloint2double((int)raw.w[2 * k + 1], (int)raw.w[2 * k]);
      } else {
#pragma unroll
        for (int k = 0; k < NZ / 2; ++k) {
          const float2 p2 = work2<S>(raw.w[k]);
          v[2 * k] = p2.x;
          v[2 * k + 1] = p2.y;
        }
      }
      if constexpr (ez == 0) {
#pragma unroll
        for (int k = 0; k < NZ; ++k) f[k][i] = v[k];
      } else if constexpr (ez > 0) {
#pragma unroll
        for (int k = 1; k < NZ; ++k) f[k][i] = v[k - 1];
        f[0][i] = St::work(bottom ? static_cast<const T *>(a.p.zlo[i]) + pidx0 : ps - 1);
      } else {
        // the row's last node (lane nv - 1) pulls the top face's value; in a
        // partial vector the padding lanes after it take any value (a
        // select per lane, not a store at a computed lane, which would put
        // f in local memory)
        const R e = St::work(top ? static_cast<const T *>(a.p.zhi[i]) + (pidx0 + (nv - 1))
                                 : ps + NZ);
#pragma unroll
        for (int k = 0; k < NZ - 1; ++k) f[k][i] = k == nv - 1 ? e : v[k + 1];
        f[NZ - 1][i] = e;
      }
    });
    if (bottom && a.g.face[4] == LBM_BC_WALL_WITH_SPEED)
      zface_wws<Q, 4, St::kShift>(a.g, face_rho, x, y, 0, f[0]);
    if (top && a.g.face[5] == LBM_BC_WALL_WITH_SPEED)
      zface_wws<Q, 5, St::kShift>(a.g, face_rho, x, y, a.g.nz - 1, f[NZ - 1]);
  } else if constexpr (!kCompact) {
    const T *fa = static_cast<const T *>(a.fa);
    // (padding lanes repeat the row's last node; they are not finished)
#pragma unroll
    for (int k = 0; k < NZ; ++k)
      pull_general<Q, S, true>(fa, a.g, x, y, k < nv ? z0 + k : a.g.nz - 1, face_rho, f[k]);
  }

  unsigned bad = 0;
#pragma unroll
  for (int k = 0; k < NZ; ++k) {
    const int z = z0 + k;
    // (a thread's nodes may straddle two force chunks: dense rows of any length)
    if (k < nv)
      finish_node<Q, FORCE, St::kDev, St::kShift>(a, f[k], idx0 + k, x, y, z,
                                      !row_in || z == 0 || z == a.g.nz - 1,
                                      chunk_force<FORCE>(a, idx0 + k), bad);
  }
  report_bad(a.status, bad);
  if (a.fb == nullptr) return;
  static_for<Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    Words<kWords> raw;
    if constexpr (St::kBits == 32) {
#pragma unroll
      for (int k = 0; k < NZ; ++k) raw.w[k] = __float_as_uint(f[k][i]);
    } else if constexpr (St::kBits == 64) {
#pragma unroll
      for (int k = 0; k < NZ; ++k) {
        raw.w[2 * k] = (unsigned)__double2loint(f[k][i]);
        raw.w[2 * k + 1] = (unsigned)__double2hiint(f[k][i]);
      }
    } else {
#pragma unroll
      for (int k = 0; k < NZ / 2; ++k) raw.w[k] = put2<S>(f[2 * k][i], f[2 * k + 1][i]);
    }
    st_words(static_cast<T *>(a.p.dst[i]) + pidx0, raw);
  });
}

// Register cap of the vectorised step for 16-bit storage, as resident blocks
// per SM asked of the compiler (0 = no cap).  A 16-bit population costs a
// whole float register once unpacked, so the 16-bit kernels hold too few
// bytes in flight per SM to cover HBM latency unless enough warps are
// resident; these caps (measured on B200 at 512^3 and on lattices with
// particles; none of them spills) trade register slack for resident warps.
// FP32 runs uncapped.
template <int Q, int S, int NZ, bool FORCE>
constexpr int vec_reg_cap() {
  if (Storage<S>::kBits != 16) return 0;
  if (NZ == 2 && FORCE) return Q == 19 ? 72 : Q == 27 ? 96 : 0;
  if (NZ == 4) return Q == 15 || Q == 19 ? 128 : 0;
  return 0;
}
template <int Q, int S, int NZ, int TB, bool FORCE>
constexpr int vec_min_blocks() {
  return vec_reg_cap<Q, S, NZ, FORCE>() == 0 ? 0 : 65536 / (vec_reg_cap<Q, S, NZ, FORCE>() * TB);
}

template <int Q, int S, bool FORCE, int NZ, int TB, bool PITCH>
__global__ void __launch_bounds__(TB, (vec_min_blocks<Q, S, NZ, TB, FORCE>()))
    k_step_vec(const __grid_constant__ StepArgs a) {
  chain_enter();
  step_vec_body<Q, S, FORCE, NZ, PITCH>(a, blockIdx.x * TB + threadIdx.x);
}

// Rows of odd length in 16-bit storage: thread k of a row takes the node pair
// (2k, 2k + 1) through the pair code with element-wise loads, and the last
// thread of the row the single node nz - 1 through the one-node code.  Same
// per-node arithmetic as every other shape.  Measured on B200 it beats one
// node per thread only for unforced D3Q19 (+7 % at 257^3) and loses for
// D3Q27, so it is a tuner candidate, not a default.
template <int Q, int S, bool FORCE, int TB>
__global__ void __launch_bounds__(TB, (vec_min_blocks<Q, S, 2, TB, FORCE>()))
    k_step_odd(const __grid_constant__ StepArgs a, const FastDiv per_row, unsigned rows) {
  chain_enter();
  const unsigned t = blockIdx.x * TB + threadIdx.x;
  const unsigned row = fdiv(t, per_row);
  if (row >= rows) return;
  const unsigned z = 2u * (t - row * per_row.d);
  const unsigned idx = row * (unsigned)a.g.nz + z;
  if (z + 1u < (unsigned)a.g.nz)
    step_vec_pairs_at<Q, S, FORCE, 2, compact_face_rows<Q, S, FORCE>(), false>(a, idx);
  else
    step_scalar_body<Q, S, FORCE>(a, idx);
}

// ---------------------------------------------------------------------------
// Multi-lattice step: one launch advances `count` independent lattices of one
// velocity set and storage by one step.  Lattice e owns blocks
// [block_begin[e], block_begin[e+1]); each block finds its lattice by binary
// search, copies that lattice's StepArgs into shared memory and runs the
// same per-node code as the single-lattice kernels (NZ = 1: k_step's body,
// NZ > 1: k_step_vec's) on kBatchTiles consecutive tiles, so a lattice's
// result does not depend on which other lattices share the launch.
// ---------------------------------------------------------------------------
constexpr int kBatchTiles = 4;   // tiles of TB threads per block (amortises the lookup)

template <int Q, int S, bool FORCE, int NZ, int TB>
__global__ void __launch_bounds__(TB, (vec_min_blocks<Q, S, NZ, TB, FORCE>()))
    k_step_batch(const StepArgs *__restrict__ entries, const unsigned *__restrict__ block_begin,
                 int count) {
  __shared__ __align__(16) StepArgs sa;
  __shared__ unsigned s_entry;
  if (threadIdx.x == 0) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (block_begin[mid] <= blockIdx.x)
        lo = mid;
      else
        hi = mid - 1;
    }
    s_entry = (unsigned)lo;
  }
  __syncthreads();
  const unsigned e = s_entry;
  constexpr int kWordsArgs = (int)(sizeof(StepArgs) / 4);
  static_assert(sizeof(StepArgs) % 4 == 0, "StepArgs is copied as 32-bit words");
  const unsigned *src = reinterpret_cast<const unsigned *>(entries + e);
  unsigned *dst = reinterpret_cast<unsigned *>(&sa);
  for (int w = threadIdx.x; w < kWordsArgs; w += TB) dst[w] = src[w];
  __syncthreads();
  const unsigned t0 = (blockIdx.x - block_begin[e]) * (TB * kBatchTiles) + threadIdx.x;
#pragma unroll 1
  for (int it = 0; it < kBatchTiles; ++it) {
    if constexpr (NZ == 1)
      step_scalar_body<Q, S, FORCE>(sa, t0 + it * TB);
    else
      step_vec_body<Q, S, FORCE, NZ, true>(sa, t0 + it * TB);
  }
}


// ---------------------------------------------------------------------------
// TMA-staged persistent step.  Each CTA walks groups of R whole z-rows
// (row = (x, y)); for a row with interior (x, y) the source of direction i is
// row (x - ex, y - ey) of plane i, so one elected thread brings the group in
// with Q * R bulk copies (cp.async.bulk, completion counted on an mbarrier)
// into a ring of `stages` shared-memory stages, several groups ahead of the
// compute.  Threads then read their two consecutive nodes per direction from
// shared memory (z-1 / z+1 neighbours included; z = 0 / nz - 1 take the
// bottom / top face rule from global memory), finish the nodes and store
// them as 8-byte (fp32) / 4-byte (16-bit) pairs.  Rows on an x / y face are
// pulled from global memory with the full face rules.  Bytes in flight are
// bounded by shared memory, not registers -- what the 16-bit storage needs
// to reach HBM bandwidth.  Every barrier wait is bounded; a timeout sets
// LBM_STATUS_WAIT_TIMEOUT and the CTA drains its copies (bounded by the
// default limit) and stops; a drain that also times out sets
// LBM_STATUS_DRAIN_FAILED.
// ---------------------------------------------------------------------------
constexpr int kTmaThreads = 256;
constexpr unsigned kTmaWaitPolls = kTmaWaitPollsDefault;

struct TmaPlan {
  int rows_per_stage;
  int stages;
  unsigned row_bytes;
  long long groups;
  unsigned wait_polls;   // limit of the consumer waits (the drain keeps kTmaWaitPolls)
};


// working value(s) of one / two staged elements
template <int S>
__device__ __forceinline__ float sm_elem(const typename Storage<S>::T *p) {
  if constexpr (Storage<S>::kBits == 32)
    return *p;
  else if constexpr (S == LBM_STORAGE_FP16S)
    return __half2float(*p);
  else
    return __bfloat162float(*p);
}

template <int S>
__device__ __forceinline__ float2 sm_pair(const typename Storage<S>::T *p) {
  if constexpr (Storage<S>::kBits == 32)
    return *reinterpret_cast<const float2 *>(p);
  else
    return work2<S>(*reinterpret_cast<const unsigned *>(p));
}

template <int Q, int S, bool FORCE>
__global__ void __launch_bounds__(kTmaThreads) k_step_tma(const __grid_constant__ StepArgs a, const TmaPlan p) {
  using St = Storage<S>;
  using T = typename St::T;
  using V = VSet<Q>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  T *buf = reinterpret_cast<T *>(smem + 128);
  const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
  const int R = p.rows_per_stage;
  const T *__restrict__ fa = static_cast<const T *>(a.fa);
  const float *face_rho = static_cast<const float *>(a.face_rho_in);
  const int tid = threadIdx.x;
  const long long G = gridDim.x;
  if (tid == 0) {
    for (int s = 0; s < p.stages; ++s) mbar_init(&bars[s], 1);
    mbar_init_fence();
  }
  __syncthreads();

  auto row_xy = [&](long long r, int &x, int &y) {
    x = (int)(r / ny);
    y = (int)(r - (long long)x * ny);
  };
  auto interior = [&](int x, int y) { return x > 0 && x < nx - 1 && y > 0 && y < ny - 1; };
  auto issue = [&](int s, long long g) {
    const long long r0 = g * R;
    unsigned bytes = 0;
    for (int j = 0; j < R; ++j) {
      int x, y;
      row_xy(r0 + j, x, y);
      if (interior(x, y)) bytes += Q * p.row_bytes;
    }
    if (bytes == 0) {
      mbar_arrive(&bars[s]);
      return;
    }
    mbar_arrive_expect_tx(&bars[s], bytes);
    for (int j = 0; j < R; ++j) {
      int x, y;
      row_xy(r0 + j, x, y);
      if (!interior(x, y)) continue;
      T *dst = buf + (long long)(s * R + j) * Q * nz;
      static_for<Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        const T *src = fa + (long long)i * a.g.n +
                       ((long long)(x - V::ex(i)) * ny + (y - V::ey(i))) * nz;
        bulk_copy_g2s(dst + (long long)i * nz, src, p.row_bytes, &bars[s]);
      });
    }
  };
  if (tid == 0) {
    for (int s = 0; s < p.stages; ++s) {
      const long long g = blockIdx.x + s * G;
      if (g < p.groups) issue(s, g);
    }
  }

  const int half = nz / 2;
  long long k = 0;
  bool timed_out = false;
  for (;; ++k) {
    const long long g = blockIdx.x + k * G;
    if (g >= p.groups) break;
    const int s = (int)(k % p.stages);
    const unsigned par = (unsigned)((k / p.stages) & 1);
    const bool ok = mbar_wait_bounded(&bars[s], par, p.wait_polls);
    if (__syncthreads_or(!ok)) {
      timed_out = true;
      break;
    }
    for (int pi = tid; pi < R * half; pi += kTmaThreads) {
      const int j = pi / half, zp = pi - j * half;
      const long long r = g * R + j;
      int x, y;
      row_xy(r, x, y);
      const int z = 2 * zp;
      const unsigned idx = (unsigned)(r * nz + z);
      const ChunkForce cf = chunk_force<FORCE>(a, idx);
      float f0[Q], f1[Q];
      const bool row_in = interior(x, y);
      if (row_in) {
        const T *srow = buf + (long long)(s * R + j) * Q * nz;
        static_for<Q>([&](auto ic) {
          constexpr int i = decltype(ic)::value;
          constexpr int ez = V::ez(i);
          const T *rp = srow + (long long)i * nz;
          if constexpr (ez == 0) {
            const float2 v = sm_pair<S>(rp + z);
            f0[i] = v.x;
            f1[i] = v.y;
          } else if constexpr (ez > 0) {
            f1[i] = sm_elem<S>(rp + z);
            f0[i] = z == 0 ? St::work(static_cast<const T *>(a.p.zlo[i]) + idx)
                           : sm_elem<S>(rp + z - 1);
          } else {
            f0[i] = sm_elem<S>(rp + z + 1);
            f1[i] = z + 2 == nz ? St::work(static_cast<const T *>(a.p.zhi[i]) + (idx + 1))
                                : sm_elem<S>(rp + z + 2);
          }
        });
        if (z == 0 && a.g.face[4] == LBM_BC_WALL_WITH_SPEED)
          zface_wws<Q, 4, St::kShift>(a.g, face_rho, x, y, 0, f0);
        if (z + 2 == nz && a.g.face[5] == LBM_BC_WALL_WITH_SPEED)
          zface_wws<Q, 5, St::kShift>(a.g, face_rho, x, y, nz - 1, f1);
      } else {
        pull_general<Q, S, true>(fa, a.g, x, y, z, face_rho, f0);
        pull_general<Q, S, true>(fa, a.g, x, y, z + 1, face_rho, f1);
      }
      unsigned bad = 0;
      finish_node<Q, FORCE, St::kDev, St::kShift>(a, f0, idx, x, y, z, !row_in || z == 0, cf, bad);
      finish_node<Q, FORCE, St::kDev, St::kShift>(a, f1, idx + 1, x, y, z + 1, !row_in || z + 1 == nz - 1, cf,
                                      bad);
      report_bad(a.status, bad);
      if (a.fb != nullptr) {
        static_for<Q>([&](auto ic) {
          constexpr int i = decltype(ic)::value;
          T *dst = static_cast<T *>(a.p.dst[i]) + idx;
          if constexpr (St::kBits == 32)
            *reinterpret_cast<float2 *>(dst) = make_float2(f0[i], f1[i]);
          else
            *reinterpret_cast<unsigned *>(dst) = put2<S>(f0[i], f1[i]);
        });
      }
    }
    __syncthreads();
    if (tid == 0) {
      const long long g2 = g + (long long)p.stages * G;
      if (g2 < p.groups) {
        fence_proxy_async_smem();
        issue(s, g2);
      }
    }
  }
  if (timed_out && tid == 0) {
    unsigned bits = LBM_STATUS_WAIT_TIMEOUT;
    // drain the copies still in flight into this CTA's shared memory
    for (long long kk = k; kk < k + p.stages; ++kk) {
      if (blockIdx.x + kk * G >= p.groups) break;
      if (!mbar_wait_bounded(&bars[kk % p.stages], (unsigned)((kk / p.stages) & 1), kTmaWaitPolls))
        bits |= LBM_STATUS_DRAIN_FAILED;
    }
    if (a.status != nullptr) atomicOr(a.status, bits);
  }
}

// Launch shape of the fused step: nodes per thread (1 = scalar kernel, or
// NZ consecutive z-nodes moved as 4 / 8 / 16-byte vectors, the row pitch pz a
// multiple of NZ; the last nodes of a row that does not fill a thread's NZ
// take the per-node path) and threads per block.
// Shapes lbm_flow_step accepts: the above, plus 2 nodes per thread for
// unpitched 16-bit rows of odd length (k_step_odd).
inline bool step_shape_ok(int nodes, int pz, int bits);
inline bool step_shape_legal(int nodes, int pz, int bits) {
  return step_shape_ok(nodes, pz, bits) || (nodes == 2 && bits == 16 && pz % 2 == 1 && pz >= 3);
}

inline bool step_shape_ok(int nodes, int pz, int bits) {
  if (nodes == 1) return true;
  if (nodes != 2 && nodes != 4 && nodes != 8) return false;
  if (nodes * bits / 32 < 1 || nodes * bits / 32 > 4) return false;
  return pz % nodes == 0 && pz >= 2 * nodes;
}

// Shared-memory plan of the TMA-staged step for this device, or false when
// the lattice does not qualify (rows must be a multiple of 16 bytes, the
// population buffer 16-byte aligned, and two stages must fit).
struct DeviceInfo {
  int sms = 0, smem_sm = 0, smem_optin = 0;
};

inline bool device_info(DeviceInfo &d) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return false;
  if (cudaDeviceGetAttribute(&d.smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) !=
      cudaSuccess)
    return false;
  if (cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
      cudaSuccess)
    return false;
  return true;
}

inline bool tma_plan(const Geom &g, int q, int bits, const void *fa, TmaPlan &p, int &ctas,
                     size_t &smem, unsigned &grid) {
  const int elem = bits / 8;
  const long long row_bytes = (long long)g.nz * elem;
  if (g.pz != g.nz) return false;   // whole rows are copied: no padding between them
  if (row_bytes % 16 != 0 || g.nz < 16 || ((uintptr_t)fa & 15u) != 0) return false;
  DeviceInfo d;
  if (!device_info(d)) return false;
  const long long rows = (long long)g.nx * g.ny;
  int R = 2 * kTmaThreads / g.nz;
  if (R < 1 || rows % R != 0) R = 1;
  const long long stage = (long long)R * q * row_bytes;
  const long long reserve = 1024 + 128;
  int stages = (int)std::min<long long>(8, (d.smem_sm / 2 - reserve) / stage);
  ctas = 2;
  if (stages < 3) {
    ctas = 1;
    stages = (int)std::min<long long>(8, (std::min(d.smem_optin, d.smem_sm) - reserve) / stage);
  }
  if (stages < 2) return false;
  p.rows_per_stage = R;
  p.stages = stages;
  p.row_bytes = (unsigned)row_bytes;
  p.groups = rows / R;
  p.wait_polls = tma_wait_polls();
  smem = 128 + (size_t)stages * stage;
  const long long want = (long long)ctas * d.sms;
  grid = (unsigned)std::min<long long>(p.groups, want);
  return true;
}

template <int Q, int S>
struct StepLauncher {
  template <bool FORCE>
  static int go_tma_f(const StepArgs &a, cudaStream_t s) {
    TmaPlan p;
    int ctas;
    size_t smem;
    unsigned grid;
    if (!tma_plan(a.g, Q, Storage<S>::kBits, a.fa, p, ctas, smem, grid)) {
      set_error("lbm_flow_step: this lattice does not qualify for row staging (rows must be a "
                "multiple of 16 bytes and at least 16 nodes, buffers 16-byte aligned)");
      return LBM_ERR_INVALID;
    }
    cudaError_t e = cudaFuncSetAttribute(k_step_tma<Q, S, FORCE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return fail_cuda(e, "lbm_flow_step");
    k_step_tma<Q, S, FORCE><<<grid, kTmaThreads, smem, s>>>(a, p);
    return LBM_OK;
  }
  static int go_tma(const StepArgs &a, bool force, cudaStream_t s) {
    if constexpr (Storage<S>::kBits == 64) {
      set_error("lbm_flow_step: row staging is not built for FP64 storage");
      return LBM_ERR_UNSUPPORTED;
    } else {
      return force ? go_tma_f<true>(a, s) : go_tma_f<false>(a, s);
    }
  }

  template <int NZ, int TB>
  static void go_vec(const StepArgs &a, bool force, cudaStream_t s) {
    const unsigned nb = blocks_for(a.g.np / NZ, TB);
    if (a.g.pz != a.g.nz) {
      if (force)
        launch_chained(k_step_vec<Q, S, true, NZ, TB, true>, nb, TB, 0, s, a);
      else
        launch_chained(k_step_vec<Q, S, false, NZ, TB, true>, nb, TB, 0, s, a);
    } else {
      if (force)
        launch_chained(k_step_vec<Q, S, true, NZ, TB, false>, nb, TB, 0, s, a);
      else
        launch_chained(k_step_vec<Q, S, false, NZ, TB, false>, nb, TB, 0, s, a);
    }
  }
  template <int NZ>
  static void go_nz(const StepArgs &a, bool force, int threads, cudaStream_t s) {
    if (threads == 128)
      go_vec<NZ, 128>(a, force, s);
    else
      go_vec<NZ, 256>(a, force, s);
  }
  template <bool FORCE, int TB>
  static void go_odd_f(const StepArgs &a, cudaStream_t s) {
    if constexpr (Storage<S>::kBits == 16) {
      const unsigned per_row = (unsigned)(a.g.nz + 1) / 2;
      const unsigned rows = (unsigned)(a.g.nx * a.g.ny);
      const unsigned nb = blocks_for((long long)rows * per_row, TB);
      launch_chained(k_step_odd<Q, S, FORCE, TB>, nb, TB, 0, s, a, make_fastdiv(per_row), rows);
    }
  }
  static void go_odd(const StepArgs &a, bool force, int threads, cudaStream_t s) {
    if (threads == 256)
      force ? go_odd_f<true, 256>(a, s) : go_odd_f<false, 256>(a, s);
    else
      force ? go_odd_f<true, 128>(a, s) : go_odd_f<false, 128>(a, s);
  }
  static int go(const StepArgs &a, bool force, int nodes, int threads, cudaStream_t s) {
    constexpr int bits = Storage<S>::kBits;
    if (nodes == LBM_STEP_ROWS) return go_tma(a, force, s);
    const bool odd_pairs = bits == 16 && a.g.pz % 2 == 1 && a.g.nz >= 3;
    if (nodes == 0) {
      // Measured on B200 at 512^3: node pairs with 128-thread blocks are the
      // fastest shape wherever rows allow them (D3Q19 FP32 3027 us, one node
      // per thread 3045 us; 3035 against 3132 us over seconds under the
      // power cap, where the pair kernel holds 1935 MHz and the other 1845),
      // except unforced D3Q13 / D3Q19 in 16-bit storage, where 4 nodes per
      // thread are (D3Q19 fp16s 1818 against 1881 us, bf16s 2075 against
      // 2325; D3Q13 fp16s 1594 against 1768).  Rows of odd length without
      // pitch take one node per thread (on the walled 161x65x65 and
      // 257x129x129 lattices also faster than pitched pairs); the odd-row
      // pair kernel is a tuner candidate only.
      const int want = (bits == 16 && (Q == 13 || Q == 19) && !force) ? 4 : 2;
      nodes = step_shape_ok(want, a.g.pz, bits) ? want : step_shape_ok(2, a.g.pz, bits) ? 2 : 1;
      threads = threads ? threads : 128;
    }
    if (nodes == 2 && odd_pairs) {
      go_odd(a, force, threads, s);
      return LBM_OK;
    }
    if (nodes == 2) {
      go_nz<2>(a, force, threads, s);
      return LBM_OK;
    }
    if constexpr (bits != 64) {
      if (nodes == 4) {
        go_nz<4>(a, force, threads, s);
        return LBM_OK;
      }
    }
    if constexpr (bits == 16) {
      if (nodes == 8) {
        go_nz<8>(a, force, threads, s);
        return LBM_OK;
      }
    }
    const unsigned nb = blocks_for(a.g.n, kThreads);
    if (force)
      launch_chained(k_step<Q, S, true>, nb, kThreads, 0, s, a);
    else
      launch_chained(k_step<Q, S, false>, nb, kThreads, 0, s, a);
    return LBM_OK;
  }
};

// Step statistics of velocity set Q and storage S: init, k_stats (eight
// blocks per SM at most; the kernel streams the populations once), finish.
template <int Q, int S>
int run_stats_qs(const StepArgs &a, bool force, unsigned long long *out, cudaStream_t s) {
  DeviceInfo d;
  int sms = 148;
  if (device_info(d)) sms = d.sms;
  const unsigned blocks = (unsigned)std::min<long long>(blocks_for(a.g.n, kStatsThreads),
                                                        (long long)sms * 8);
  k_stats_init<Q><<<1, 32, 0, s>>>(out);
  if (force)
    k_stats<Q, S, true><<<blocks, kStatsThreads, 0, s>>>(a, out);
  else
    k_stats<Q, S, false><<<blocks, kStatsThreads, 0, s>>>(a, out);
  k_stats_finish<Q><<<1, 32, 0, s>>>(out, (double)a.g.n);
  LBM_LAUNCH_CHECK("lbm_flow_stats");
  return LBM_OK;
}

// Multi-lattice launch for velocity set Q and storage S: nodes per thread 1
// (256 threads), 2 or 4 (128 threads).
template <int Q, int S>
int run_step_batch_qs(const StepArgs *entries, const unsigned *block_begin, int count,
                      unsigned total_blocks, bool force, int nodes, cudaStream_t s) {
  if (nodes == 2) {
    if (force)
      k_step_batch<Q, S, true, 2, 128><<<total_blocks, 128, 0, s>>>(entries, block_begin, count);
    else
      k_step_batch<Q, S, false, 2, 128><<<total_blocks, 128, 0, s>>>(entries, block_begin, count);
  } else if (nodes == 4 && Storage<S>::kBits != 64) {
    if constexpr (Storage<S>::kBits != 64) {
      if (force)
        k_step_batch<Q, S, true, 4, 128><<<total_blocks, 128, 0, s>>>(entries, block_begin, count);
      else
        k_step_batch<Q, S, false, 4, 128><<<total_blocks, 128, 0, s>>>(entries, block_begin, count);
    }
  } else {
    if (force)
      k_step_batch<Q, S, true, 1, 256><<<total_blocks, 256, 0, s>>>(entries, block_begin, count);
    else
      k_step_batch<Q, S, false, 1, 256><<<total_blocks, 256, 0, s>>>(entries, block_begin, count);
  }
  LBM_LAUNCH_CHECK("lbm_flow_step_batch");
  return LBM_OK;
}

// One fused step for velocity set Q and storage S (explicitly instantiated
// once per (Q, S) in lbm_step_inst.cu, so the launch-shape variants compile
// in parallel translation units).
template <int Q, int S>
int run_step_qs(const StepArgs &a, bool force, int nodes, int threads, cudaStream_t s) {
  const int rc = StepLauncher<Q, S>::go(a, force, nodes, threads, s);
  if (rc) return rc;
  LBM_LAUNCH_CHECK("lbm_flow_step");
  return LBM_OK;
}

#define LBM_FOR_EACH_QS(X)                                                                  \
  X(13, 0) X(13, 1) X(13, 2) X(13, 3) X(15, 0) X(15, 1) X(15, 2) X(15, 3) X(19, 0) X(19, 1) \
  X(19, 2) X(19, 3) X(27, 0) X(27, 1) X(27, 2) X(27, 3)

}  // namespace lbm
