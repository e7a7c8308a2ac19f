// Velocity sets, population storage and the per-node pieces of one LBM step
// (pull streaming with the reference's face rules, moments, forcing, BGK),
// shared by every kernel of the library.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#include "../../include/funlbm_b200.h"

namespace lbm {

// Bounds-checked build (-DLBM_BOUNDS_CHECK): kernels verify their index
// invariants before each access (node inside the lattice, population index
// inside the pitched buffer, pull source inside the lattice, field index
// inside the field); a violation is counted in this translation unit's
// g_lbm_oob and the access is skipped or clamped to a valid index
// (lbm_debug_bounds_faults reads the counts).  Without the flag lbm_in is
// always true and the checks compile away.
#ifdef LBM_BOUNDS_CHECK
static __device__ unsigned long long g_lbm_oob;
__device__ __forceinline__ bool lbm_in(bool ok) {
  if (!ok) atomicAdd(&g_lbm_oob, 1ull);
  return ok;
}
#else
__device__ __forceinline__ constexpr bool lbm_in(bool) { return true; }
#endif

// Chained launches (programmatic dependent launch).  The kernels of one
// lattice step -- interpolation, spreading, the rigid update and the fused
// step -- are launched with programmatic stream serialization
// (launch_chained): the GPU may schedule such a kernel while the kernel
// before it in the stream is still running.  chain_wait() is therefore the
// first statement of each of them, executed by every thread before any
// memory access: it returns once the previous kernel has completed and its
// writes are visible, so every access happens in plain stream order.
// chain_release() right after it lets the next kernel be scheduled while
// this one runs (a kernel is only scheduled once every block of the one
// before it has started, so a waiting kernel never holds resources the
// running one still needs).  Launched without the attribute, both are no-ops.
__device__ __forceinline__ void chain_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void chain_release() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void chain_enter() {
  chain_wait();
  chain_release();
}

// Compile-time loop: calls fn(std::integral_constant<int, I>) for I < N, so
// every population index is a constant and f[Q] stays in registers.
template <typename F, int... I>
__host__ __device__ __forceinline__ void static_for_impl(F &&fn, std::integer_sequence<int, I...>) {
  (fn(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
__host__ __device__ __forceinline__ void static_for(F &&fn) {
  static_for_impl(fn, std::make_integer_sequence<int, N>{});
}

// ---------------------------------------------------------------------------
// Velocity sets.  Direction order is the reference's (flow/d3/d3q13.py:7-21,
// d3q15.py:7-23, d3q19.py:8-28, d3q27.py:8-36): the opposite-direction table
// and the population layout depend on it.  Weights by speed class
// (d3q13.py:23-39, d3q15.py:25-43, d3q19.py:30-54, d3q27.py:38-71).
// Tables live inside constexpr functions so that fully unrolled loops fold
// every lookup to an immediate.
// ---------------------------------------------------------------------------
template <int Q>
struct VSet;

#define LBM_VSET_BODY(QN, EX, EY, EZ, W0, W1, W2, W3)                                   \
  static constexpr int kQ = QN;                                                           \
  __host__ __device__ static constexpr int ex(int i) {                                    \
    constexpr int t[QN] = EX;                                                             \
    return t[i];                                                                          \
  }                                                                                       \
  __host__ __device__ static constexpr int ey(int i) {                                    \
    constexpr int t[QN] = EY;                                                             \
    return t[i];                                                                          \
  }                                                                                       \
  __host__ __device__ static constexpr int ez(int i) {                                    \
    constexpr int t[QN] = EZ;                                                             \
    return t[i];                                                                          \
  }                                                                                       \
  __host__ __device__ static constexpr int speed2(int i) {                                \
    return ex(i) * ex(i) + ey(i) * ey(i) + ez(i) * ez(i);                                \
  }                                                                                       \
  __host__ __device__ static constexpr double wd(int i) {                                 \
    return speed2(i) == 0 ? (W0) : speed2(i) == 1 ? (W1) : speed2(i) == 2 ? (W2) : (W3); \
  }                                                                                       \
  __host__ __device__ static constexpr float w(int i) { return (float)wd(i); }           \
  template <typename R>                                                                   \
  __host__ __device__ static constexpr R wr(int i) { return (R)wd(i); }                   \
  __host__ __device__ static constexpr int rev(int i) {                                   \
    int r = 0;                                                                            \
    for (int j = 0; j < QN; ++j)                                                          \
      if (ex(j) == -ex(i) && ey(j) == -ey(i) && ez(j) == -ez(i)) r = j;                   \
    return r;                                                                             \
  }

#define LBM_ARR(...) {__VA_ARGS__}

template <>
struct VSet<13> {
  LBM_VSET_BODY(13,
                LBM_ARR(0, 1, 1, 1, 1, 0, 0, -1, -1, -1, -1, 0, 0),
                LBM_ARR(0, 1, -1, 0, 0, 1, 1, -1, 1, 0, 0, -1, -1),
                LBM_ARR(0, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1),
                1.0 / 2, 0.0, 1.0 / 24, 0.0)
};
template <>
struct VSet<15> {
  LBM_VSET_BODY(15,
                LBM_ARR(0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1),
                LBM_ARR(0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1),
                LBM_ARR(0, 0, 0, 0, 0, 1, -1, 1, 1, 1, 1, -1, -1, -1, -1),
                2.0 / 9, 1.0 / 9, 0.0, 1.0 / 72)
};
template <>
struct VSet<19> {
  LBM_VSET_BODY(19,
                LBM_ARR(0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1),
                LBM_ARR(0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 1, -1, 1, -1, 0, 0, 0, 0),
                LBM_ARR(0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1),
                1.0 / 3, 1.0 / 18, 1.0 / 36, 0.0)
};
template <>
struct VSet<27> {
  LBM_VSET_BODY(27,
                LBM_ARR(0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, 1, 1,
                        -1, -1, -1, -1),
                LBM_ARR(0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1,
                        1, 1, -1, -1),
                LBM_ARR(0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1, 1, -1, 1, -1,
                        1, -1, 1, -1),
                8.0 / 27, 2.0 / 27, 1.0 / 54, 1.0 / 216)
};

#undef LBM_ARR
#undef LBM_VSET_BODY

// ---------------------------------------------------------------------------
// Population storage.  FP32 stores f; the shifted 16-bit forms store f - w_i
// (the deviation from the rest-state weight carries all the information and
// keeps the 16-bit mantissa busy), collided in float32.
// ---------------------------------------------------------------------------
template <int S>
struct Storage;

// The fused step works on the stored quantity itself (its "working value"):
// the deviation d = f - w_i for the shifted forms (kDev: FP32 and both 16-bit
// storages), whose moments and collision are restated for d (dev_moments /
// collide_dev), so no weight is added on load or subtracted on store; f
// itself for FP64.  work / put / work2 / put2 move working values; load /
// store always give f.
//
// FP32 stores the deviation too.  At the low Mach numbers of the reference's
// cases a population f ~ w_i ~ 0.05 carries its velocity part (w rho e.u /
// cs^2 ~ 1e-6) in its last ten bits, and a body or IBM force adds ~17 units
// in the last place per step: stored as f, those increments round with the
// same bias every step of a nearly steady flow, and the float32 run drifts
// from the float64 one (measured on B200: twice the reference's own float32
// drift on the 33 x 33 x 65 Poiseuille channel after 2000 steps, ten times
// in the sedimenting sphere's velocity after 5000).  Stored as d ~ 1e-6 the
// same 32 bits resolve the signal to ~1e-7 of itself, at the same bytes per
// node.
template <>
struct Storage<LBM_STORAGE_FP32> {
  using T = float;
  using R = float;   // arithmetic type of the kernels
  static constexpr int kBits = 32;
  static constexpr bool kDev = true;
  static constexpr int kShift = 0;   // working value = d * 2^kShift
  __device__ __forceinline__ static T raw(const T *p) { return __ldg(p); }
  __device__ __forceinline__ static float cvt(T v) { return v; }
  __device__ __forceinline__ static float work(const T *p) { return __ldg(p); }
  __device__ __forceinline__ static void put(T *p, float v) { *p = v; }
  __device__ __forceinline__ static float load(const T *p, float w) { return w + __ldg(p); }
  __device__ __forceinline__ static void store(T *p, float v, float w) { *p = v - w; }
};
// FP16 holds the deviation scaled by 2^12: float16's normal range starts at
// 6.1e-5, and at the velocities of the reference's particle cases (|u| ~
// 1e-6) a deviation w rho e.u / cs^2 ~ 1e-7 would fall among its subnormals
// (spacing 6e-8: a 90 % velocity error measured over 3000 steps of the
// 32-ellipsoid case).  Scaled, deviations from 1.5e-8 up to 16 keep the full
// 11-bit significand; populations stay in [0, 1], so |d| < 1.  The scale is
// a power of two: the scaling itself is exact.  The fused step keeps the
// scaled value as its working value (kShift): the moments unscale their sums
// and the collision and forcing carry the scale in their weight constants,
// so no element is multiplied on load or store.
constexpr float kFp16Scale = 4096.f;
constexpr float kFp16Unscale = 1.f / 4096.f;

template <>
struct Storage<LBM_STORAGE_FP16S> {
  using T = __half;
  using R = float;
  static constexpr int kBits = 16;
  static constexpr bool kDev = true;
  static constexpr int kShift = 12;
  __device__ __forceinline__ static T raw(const T *p) { return __ldg(p); }
  __device__ __forceinline__ static float cvt(T v) { return __half2float(v); }
  __device__ __forceinline__ static float work(const T *p) { return __half2float(__ldg(p)); }
  __device__ __forceinline__ static void put(T *p, float v) { *p = __float2half_rn(v); }
  __device__ __forceinline__ static float load(const T *p, float w) {
    return w + __half2float(__ldg(p)) * kFp16Unscale;
  }
  __device__ __forceinline__ static void store(T *p, float v, float w) {
    *p = __float2half_rn((v - w) * kFp16Scale);
  }
};
template <>
struct Storage<LBM_STORAGE_BF16S> {
  using T = __nv_bfloat16;
  using R = float;
  static constexpr int kBits = 16;
  static constexpr bool kDev = true;
  static constexpr int kShift = 0;
  __device__ __forceinline__ static T raw(const T *p) { return __ldg(p); }
  __device__ __forceinline__ static float cvt(T v) { return __bfloat162float(v); }
  __device__ __forceinline__ static float work(const T *p) { return __bfloat162float(__ldg(p)); }
  __device__ __forceinline__ static void put(T *p, float v) { *p = __float2bfloat16_rn(v); }
  __device__ __forceinline__ static float load(const T *p, float w) {
    return w + __bfloat162float(__ldg(p));
  }
  __device__ __forceinline__ static void store(T *p, float v, float w) {
    *p = __float2bfloat16_rn(v - w);
  }
};

// FP64: populations, moments, forcing and collision in double -- the
// comparison run against which the float32 and 16-bit storages are measured.
template <>
struct Storage<LBM_STORAGE_FP64> {
  using T = double;
  using R = double;
  static constexpr int kBits = 64;
  static constexpr bool kDev = false;
  static constexpr int kShift = 0;
  __device__ __forceinline__ static T raw(const T *p) { return __ldg(p); }
  __device__ __forceinline__ static double cvt(T v) { return v; }
  __device__ __forceinline__ static double work(const T *p) { return __ldg(p); }
  __device__ __forceinline__ static void put(T *p, double v) { *p = v; }
  __device__ __forceinline__ static double load(const T *p, double) { return __ldg(p); }
  __device__ __forceinline__ static void store(T *p, double v, double) { *p = v; }
};

// Raw 16 bits of one stored element.
__device__ __forceinline__ unsigned short bits16(__half h) { return __half_as_ushort(h); }
__device__ __forceinline__ unsigned short bits16(__nv_bfloat16 h) { return __bfloat16_as_ushort(h); }

// Two consecutive stored elements <-> two working values (low element first).
template <int S>
__device__ __forceinline__ float2 work2(unsigned word);
template <>
__device__ __forceinline__ float2 work2<LBM_STORAGE_FP16S>(unsigned word) {
  __half2 h;
  memcpy(&h, &word, 4);
  return __half22float2(h);
}
template <>
__device__ __forceinline__ float2 work2<LBM_STORAGE_BF16S>(unsigned word) {
  return make_float2(__uint_as_float(word << 16), __uint_as_float(word & 0xffff0000u));
}
template <int S>
__device__ __forceinline__ unsigned put2(float a, float b);
template <>
__device__ __forceinline__ unsigned put2<LBM_STORAGE_FP16S>(float a, float b) {
  const __half2 h = __floats2half2_rn(a, b);
  unsigned word;
  memcpy(&word, &h, 4);
  return word;
}
template <>
__device__ __forceinline__ unsigned put2<LBM_STORAGE_BF16S>(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  unsigned word;
  memcpy(&word, &h, 4);
  return word;
}

// Aligned vector loads / stores of WORDS 32-bit words (4, 8 or 16 bytes).
template <int WORDS>
struct Words {
  unsigned w[WORDS];
};
template <int WORDS>
__device__ __forceinline__ Words<WORDS> ld_words(const void *p);
template <>
__device__ __forceinline__ Words<1> ld_words<1>(const void *p) {
  return Words<1>{{__ldg(static_cast<const unsigned *>(p))}};
}
template <>
__device__ __forceinline__ Words<2> ld_words<2>(const void *p) {
  const uint2 v = __ldg(static_cast<const uint2 *>(p));
  return Words<2>{{v.x, v.y}};
}
template <>
__device__ __forceinline__ Words<4> ld_words<4>(const void *p) {
  const uint4 v = __ldg(static_cast<const uint4 *>(p));
  return Words<4>{{v.x, v.y, v.z, v.w}};
}
__device__ __forceinline__ void st_words(void *p, const Words<1> &v) {
  *static_cast<unsigned *>(p) = v.w[0];
}
__device__ __forceinline__ void st_words(void *p, const Words<2> &v) {
  *static_cast<uint2 *>(p) = make_uint2(v.w[0], v.w[1]);
}
__device__ __forceinline__ void st_words(void *p, const Words<4> &v) {
  *static_cast<uint4 *>(p) = make_uint4(v.w[0], v.w[1], v.w[2], v.w[3]);
}

// ---------------------------------------------------------------------------
// Lattice constants passed by value to every kernel.
// ---------------------------------------------------------------------------
struct Geom {
  int nx, ny, nz;
  long long n;      // nodes
  long long nyz;    // ny * nz
  int pz;           // row pitch of the population buffers (>= nz)
  long long np;     // population plane: nx * ny * pz elements
  long long nyzp;   // ny * pz
  int face[LBM_NFACES];
  float uw[LBM_NFACES][3];
  long long plane_off[LBM_NFACES];  // offsets of the face-density planes
  float tau, inv_tau, cs2, inv_cs2, inv_cs4, force_c;  // force_c = 1 - 1/(2 tau)
  float re_mu;
  const double *neq_profile;
  // the same constants in double, for FP64 storage: tau as given, cs^2 =
  // double(sqrt(1/3))^2, wall velocities widened
  double inv_tau_d, inv_cs2_d, inv_cs4_d, force_c_d;
  double uw_d[LBM_NFACES][3];
};

// Lattice constants in the arithmetic type R of a kernel.
template <typename R>
struct Cst;
template <>
struct Cst<float> {
  __device__ __forceinline__ static float inv_tau(const Geom &g) { return g.inv_tau; }
  __device__ __forceinline__ static float inv_cs2(const Geom &g) { return g.inv_cs2; }
  __device__ __forceinline__ static float inv_cs4(const Geom &g) { return g.inv_cs4; }
  __device__ __forceinline__ static float force_c(const Geom &g) { return g.force_c; }
  __device__ __forceinline__ static float uw(const Geom &g, int fc, int k) { return g.uw[fc][k]; }
};
template <>
struct Cst<double> {
  __device__ __forceinline__ static double inv_tau(const Geom &g) { return g.inv_tau_d; }
  __device__ __forceinline__ static double inv_cs2(const Geom &g) { return g.inv_cs2_d; }
  __device__ __forceinline__ static double inv_cs4(const Geom &g) { return g.inv_cs4_d; }
  __device__ __forceinline__ static double force_c(const Geom &g) { return g.force_c_d; }
  __device__ __forceinline__ static double uw(const Geom &g, int fc, int k) { return g.uw_d[fc][k]; }
};

// face-plane index of node (x, y, z) on face `fc`
__device__ __forceinline__ long long plane_index(const Geom &g, int fc, int x, int y, int z) {
  switch (fc >> 1) {
    case 0: return g.plane_off[fc] + (long long)y * g.nz + z;
    case 1: return g.plane_off[fc] + (long long)x * g.nz + z;
    default: return g.plane_off[fc] + (long long)x * g.ny + y;
  }
}

__device__ __forceinline__ bool on_any_face(const Geom &g, int x, int y, int z) {
  return x == 0 || x == g.nx - 1 || y == 0 || y == g.ny - 1 || z == 0 || z == g.nz - 1;
}

// ---------------------------------------------------------------------------
// Pull streaming with the reference's rules (flow/d3/base.py:161-323).
// For target node t and direction i the reference rolls every population
// periodically and then overrides, face by face in the order input, output,
// back, forward, bottom, top, the directions entering through that face; the
// last matching override wins.  Rolling wraps only where some face override
// applies, so the source is:
//   no face applies      -> (t - e_i, i)
//   PERIODICAL face      -> t with that axis moved to the opposite plane (no
//                           transverse shift), direction i
//   WALL face            -> (t, rev(i))                 half-way bounce-back
//   WALL_WITH_SPEED face -> (t, rev(i)) - 2 rho_t w_i (e_i . uw) / cs^2
// NON_EQUILIBRIUM x faces are handled by the caller (they need moments).
// ---------------------------------------------------------------------------
// Pull population I with face rules.  The governing face is the last one in
// the order x, y, z whose plane holds the node and through which direction I
// enters; -1 means none.  `face_rho` is consulted only for WALL_WITH_SPEED
// faces (density of the previous step at this face node).
// WORK: return the storage's working value (d for the shifted forms) instead
// of f; the WALL_WITH_SPEED correction is the same in both (in working
// units: times 2^kShift).
template <int Q, int S, int I, bool WORK = false>
__device__ __forceinline__ typename Storage<S>::R pull_one(
    const typename Storage<S>::T *__restrict__ fa, const Geom &g, int x, int y, int z,
    const typename Storage<S>::R *__restrict__ face_rho) {
  using V = VSet<Q>;
  using R = typename Storage<S>::R;
  constexpr int ex = V::ex(I), ey = V::ey(I), ez = V::ez(I);
  int fc = -1;
  if (ex > 0 && x == 0) fc = 0;
  if (ex < 0 && x == g.nx - 1) fc = 1;
  if (ey > 0 && y == 0) fc = 2;
  if (ey < 0 && y == g.ny - 1) fc = 3;
  if (ez > 0 && z == 0) fc = 4;
  if (ez < 0 && z == g.nz - 1) fc = 5;
  int sx = x - ex, sy = y - ey, sz = z - ez, sd = I;
  R corr = R(0);
  if (fc >= 0) {
    const int code = g.face[fc];
    sx = x;
    sy = y;
    sz = z;
    if (code == LBM_BC_PERIODICAL) {
      const int axis = fc >> 1;
      const bool first = (fc & 1) == 0;
      if (axis == 0) sx = first ? g.nx - 1 : 0;
      else if (axis == 1) sy = first ? g.ny - 1 : 0;
      else sz = first ? g.nz - 1 : 0;
    } else {
      sd = V::rev(I);
      if (code == LBM_BC_WALL_WITH_SPEED) {
        const R rho_t = face_rho[plane_index(g, fc, x, y, z)];
        const R eu = (R)ex * Cst<R>::uw(g, fc, 0) + (R)ey * Cst<R>::uw(g, fc, 1) +
                     (R)ez * Cst<R>::uw(g, fc, 2);
        corr = R(2) * (rho_t * V::template wr<R>(I)) * eu * Cst<R>::inv_cs2(g);
      }
    }
  }
  if (!lbm_in(sx >= 0 && sx < g.nx && sy >= 0 && sy < g.ny && sz >= 0 && sz < g.nz)) {
    sx = 0;
    sy = 0;
    sz = 0;
  }
  const long long src = ((long long)sx * g.ny + sy) * g.pz + sz;
  const R w_sd = sd == I ? V::template wr<R>(I) : V::template wr<R>(V::rev(I));
  if constexpr (WORK)
    return Storage<S>::work(fa + (long long)sd * g.np + src) -
           corr * R(1 << Storage<S>::kShift);
  else
    return Storage<S>::load(fa + (long long)sd * g.np + src, w_sd) - corr;
}

template <int Q, int S, bool WORK, int I = 0>
struct PullGeneral {
  using R = typename Storage<S>::R;
  __device__ __forceinline__ static void run(const typename Storage<S>::T *__restrict__ fa,
                                             const Geom &g, int x, int y, int z,
                                             const R *__restrict__ face_rho, R f[Q]) {
    f[I] = pull_one<Q, S, I, WORK>(fa, g, x, y, z, face_rho);
    PullGeneral<Q, S, WORK, I + 1>::run(fa, g, x, y, z, face_rho, f);
  }
};
template <int Q, int S, bool WORK>
struct PullGeneral<Q, S, WORK, Q> {
  using R = typename Storage<S>::R;
  __device__ __forceinline__ static void run(const typename Storage<S>::T *__restrict__,
                                             const Geom &, int, int, int,
                                             const R *__restrict__, R *) {}
};

template <int Q, int S, bool WORK = false>
__device__ __forceinline__ void pull_general(const typename Storage<S>::T *__restrict__ fa,
                                             const Geom &g, int x, int y, int z,
                                             const typename Storage<S>::R *__restrict__ face_rho,
                                             typename Storage<S>::R f[Q]) {
  PullGeneral<Q, S, WORK>::run(fa, g, x, y, z, face_rho, f);
}

constexpr int kMaxQ = 27;

// Per-direction plane pointers of one step, computed on the host
// (fill_step_planes), so that every population address in the kernels is
// one 32 x 32 -> 64-bit multiply-add of the node's population index
// (x ny + y) pz + z onto a parameter:
//   src[i] + idx   row (x - ex, y - ey) of plane i of fa at the node's z: the
//                  pull source of an interior row is src[i] + idx - ez;
//   zlo[i] + idx   (ez > 0) source of a node at z = 0 under the bottom face
//                  rule: PERIODICAL -> (i, x, y, nz - 1), else (rev i, x, y, 0);
//   zhi[i] + idx   (ez < 0) source of a node at z = nz - 1 under the top face
//                  rule: PERIODICAL -> (i, x, y, 0), else (rev i, x, y, nz - 1);
//   dst[i] + idx   plane i of fb.
struct StepPlanes {
  const void *src[kMaxQ];
  const void *zlo[kMaxQ];
  const void *zhi[kMaxQ];
  void *dst[kMaxQ];
};

// WALL_WITH_SPEED correction of the directions entering through z face FC
// (4 = bottom, 5 = top) at a node of an interior row, applied after the
// plain bounce-back pull: the same expression as pull_one's.
template <int Q, int FC, int SH = 0, typename R>
__device__ __forceinline__ void zface_wws(const Geom &g, const R *__restrict__ face_rho,
                                          int x, int y, int z, R f[Q]) {
  using V = VSet<Q>;
  const R rho_t = face_rho[plane_index(g, FC, x, y, z)];
  static_for<Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    constexpr int ez = V::ez(i);
    if constexpr ((FC == 4 && ez > 0) || (FC == 5 && ez < 0)) {
      const R eu = (R)V::ex(i) * Cst<R>::uw(g, FC, 0) + (R)V::ey(i) * Cst<R>::uw(g, FC, 1) +
                   (R)ez * Cst<R>::uw(g, FC, 2);
      constexpr R w = V::template wr<R>(i) * R(1 << SH);   // working units
      f[i] = f[i] - R(2) * (rho_t * w) * eu * Cst<R>::inv_cs2(g);
    }
  });
}

// Pull of one node of an interior row (x, y not on a face): every source is
// in row (x - ex, y - ey) except where the z face rule applies, which is
// chosen by a select on the address (no branch, so all Q loads issue
// together).  WORK: working values (d for the shifted storages) as the fused
// step uses them; otherwise f, with the same values and corrections as
// pull_general.
template <int Q, int S, bool WORK>
__device__ __forceinline__ void pull_row_node(const StepPlanes &p, const Geom &g,
                                              const typename Storage<S>::R *__restrict__ face_rho,
                                              unsigned idx, int x, int y, int z,
                                              typename Storage<S>::R f[Q]) {
  using St = Storage<S>;
  using T = typename St::T;
  using V = VSet<Q>;
  const bool bottom = z == 0, top = z == g.nz - 1;
  static_for<Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    constexpr int ez = V::ez(i);
    const T *ps = static_cast<const T *>(p.src[i]) + idx;
    const T *src = ps;
    if constexpr (ez > 0) src = bottom ? static_cast<const T *>(p.zlo[i]) + idx : ps - 1;
    if constexpr (ez < 0) src = top ? static_cast<const T *>(p.zhi[i]) + idx : ps + 1;
    if constexpr (WORK)
      f[i] = St::work(src);
    else
      f[i] = St::load(src, V::template wr<typename St::R>(i));
  });
  constexpr int kSh = WORK ? St::kShift : 0;
  if (bottom && g.face[4] == LBM_BC_WALL_WITH_SPEED) zface_wws<Q, 4, kSh>(g, face_rho, x, y, z, f);
  if (top && g.face[5] == LBM_BC_WALL_WITH_SPEED) zface_wws<Q, 5, kSh>(g, face_rho, x, y, z, f);
}

// Rolled value (periodic wrap on every axis, no face rule): what the
// reference's f holds at a node before the face overrides run.  Used by the
// NON_EQUILIBRIUM faces, which read plane 1 / plane X-2 right after the roll.
template <int Q>
__device__ __forceinline__ float pull_rolled(const float *__restrict__ fa, const Geom &g, int i,
                                             int x, int y, int z) {
  using V = VSet<Q>;
  int sx = x - V::ex(i), sy = y - V::ey(i), sz = z - V::ez(i);
  sx = sx < 0 ? sx + g.nx : (sx >= g.nx ? sx - g.nx : sx);
  sy = sy < 0 ? sy + g.ny : (sy >= g.ny ? sy - g.ny : sy);
  sz = sz < 0 ? sz + g.nz : (sz >= g.nz ? sz - g.nz : sz);
  const long long src = ((long long)sx * g.ny + sy) * g.nz + sz;   // dense arrays only
  return fa[(long long)i * g.n + src];
}

// ---------------------------------------------------------------------------
// Per-node arithmetic.  Directions come in opposite pairs (i, rev(i)); the
// moments, the forcing term and the equilibrium share their work across the
// pair.  The library is built with -fmad=false and every fused multiply-add
// below is explicit (__fmaf_rn), so each kernel that calls these functions
// produces the same bits whatever its launch shape.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
#define LBM_FMA(a, b, c) ::lbm::fma_rn((a), (b), (c))

// Moments (flow/d3/base.py:116-133): rho = sum f, u = (sum f e + F/2) / rho,
// u := 0 on all six boundary planes whatever their condition.
template <int Q, typename R>
__device__ __forceinline__ void moments(const R f[Q], R fx, R fy, R fz, bool face, R &rho, R &ux,
                                        R &uy, R &uz) {
  using V = VSet<Q>;
  R r = f[0], jx = R(0), jy = R(0), jz = R(0);
  static_for<Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    constexpr int j = V::rev(i);
    if constexpr (i != 0 && i < j) {
      const R s = f[i] + f[j];
      const R d = f[i] - f[j];
      r += s;
      if constexpr (V::ex(i) > 0) jx += d;
      if constexpr (V::ex(i) < 0) jx -= d;
      if constexpr (V::ey(i) > 0) jy += d;
      if constexpr (V::ey(i) < 0) jy -= d;
      if constexpr (V::ez(i) > 0) jz += d;
      if constexpr (V::ez(i) < 0) jz -= d;
    }
  });
  rho = r;
  const R inv = R(1) / r;
  ux = face ? R(0) : LBM_FMA(R(0.5), fx, jx) * inv;
  uy = face ? R(0) : LBM_FMA(R(0.5), fy, jy) * inv;
  uz = face ? R(0) : LBM_FMA(R(0.5), fz, jz) * inv;
}

// e_i . v with e_i in {-1, 0, 1}^3, folded at compile time
template <int Q, int I, typename R>
__device__ __forceinline__ R edot(R vx, R vy, R vz) {
  using V = VSet<Q>;
  R r = R(0);
  bool first = true;
  auto acc = [&](int e, R v) {
    if (e == 0) return;
    if (first) {
      r = e > 0 ? v : -v;
      first = false;
    } else {
      r = e > 0 ? r + v : r - v;
    }
  };
  acc(V::ex(I), vx);
  acc(V::ey(I), vy);
  acc(V::ez(I), vz);
  return r;
}

// Forcing term of FlowD3.cul_equ2 (flow/d3/base.py:103-114):
//   f_i += (1 - 1/(2 tau)) w_i [ (e_i - u)/cs^2 + (u o e_i) o e_i / cs^4 ] . F
// (component-wise u_k e_ik^2, the reference's form).  For the pair (i, j),
// e_j = -e_i: the e.F part flips sign, the rest is shared.
template <int Q, int SH = 0, typename R>
__device__ __forceinline__ void add_force(R f[Q], const Geom &g, R ux, R uy, R uz, R fx, R fy,
                                          R fz) {
  using V = VSet<Q>;
  const R inv_cs2 = Cst<R>::inv_cs2(g), force_c = Cst<R>::force_c(g);
  const R uF = LBM_FMA(ux, fx, LBM_FMA(uy, fy, uz * fz));
  const R ax = ux * fx, ay = uy * fy, az = uz * fz;
  const R base = -uF * inv_cs2;
  static_for<Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    constexpr int j = V::rev(i);
    constexpr R cw = V::template wr<R>(i) * R(1 << SH);     // working units
    if constexpr (i == 0) {
      f[0] = LBM_FMA(force_c * cw, base, f[0]);
    } else if constexpr (i < j) {
      R t2 = R(0);
      if constexpr (V::ex(i) != 0) t2 += ax;
      if constexpr (V::ey(i) != 0) t2 += ay;
      if constexpr (V::ez(i) != 0) t2 += az;
      const R shared = LBM_FMA(t2, Cst<R>::inv_cs4(g), base);
      const R eF = edot<Q, i>(fx, fy, fz) * inv_cs2;
      const R c = force_c * cw;
      f[i] = LBM_FMA(c, shared + eF, f[i]);
      f[j] = LBM_FMA(c, shared - eF, f[j]);
    }
  });
}

// BGK collision of FlowD3.cul_equ (flow/d3/base.py:150-159):
//   feq_i = (1 + t + t^2/2 - |u|^2/(2 cs^2)) rho w_i,  t = e_i.u / cs^2
//   f_i  <- f_i - (f_i - feq_i) / tau = f_i (1 - 1/tau) + feq_i / tau
// With a = rho w (1 - |u|^2/(2cs^2) + t^2/2) and b = rho w t, the pair gets
// feq_i = a + b, feq_rev(i) = a - b.
template <int Q>
__device__ __forceinline__ float feq_of(const Geom &g, int i, float rho, float ux, float uy,
                                        float uz, float u2) {
  using V = VSet<Q>;
  const float t = ((float)V::ex(i) * ux + (float)V::ey(i) * uy + (float)V::ez(i) * uz) * g.inv_cs2;
  return LBM_FMA(0.5f * t, t, (1.f - u2) + t) * (rho * V::w(i));
}

template <int Q, typename R>
__device__ __forceinline__ void collide(R f[Q], const Geom &g, R rho, R ux, R uy, R uz) {
  using V = VSet<Q>;
  const R inv_cs2 = Cst<R>::inv_cs2(g), inv_tau = Cst<R>::inv_tau(g);
  const R u2 = LBM_FMA(ux, ux, LBM_FMA(uy, uy, uz * uz)) * (R(0.5) * inv_cs2);
  const R om = inv_tau, keep = R(1) - inv_tau;
  const R orho = om * rho;
  const R one_u2 = R(1) - u2;
  static_for<Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    constexpr int j = V::rev(i);
    constexpr R w = V::template wr<R>(i);
    if constexpr (i == 0) {
      f[0] = LBM_FMA(f[0], keep, (orho * w) * one_u2);
    } else if constexpr (i < j) {
      const R t = edot<Q, i>(ux, uy, uz) * inv_cs2;
      const R ow = orho * w;
      const R a = ow * LBM_FMA(R(0.5) * t, t, one_u2);
      const R b = ow * t;
      f[i] = LBM_FMA(f[i], keep, a + b);
      f[j] = LBM_FMA(f[j], keep, a - b);
    }
  });
}

// Deviation form, for the shifted storages.  With f_i = w_i + d_i,
// sum w_i = 1 and sum w_i e_i = 0:
//   rho = 1 + sum d_i,   rho u = sum d_i e_i + F/2,
// and the BGK update of FlowD3.cul_equ (flow/d3/base.py:150-159) becomes
//   d_i <- d_i (1 - 1/tau) + (feq_i - w_i) / tau,
//   feq_i - w_i = w_i [ (rho - 1) + rho (t + t^2/2 - |u|^2/(2 cs^2)) ],
// so the pair (i, rev(i)) gets A +- B with
//   A = w (drho - rho |u|^2/(2cs^2)) / tau + (w rho t / (2 tau)) t,  B = w rho t / tau.
// The forcing term (add_force) is additive and applies to d unchanged.
template <int Q, int SH = 0>
__device__ __forceinline__ void dev_moments(const float d[Q], float fx, float fy, float fz,
                                            bool face, float &rho, float &drho, float &ux,
                                            float &uy, float &uz) {
  using V = VSet<Q>;
  float r = d[0], jx = 0.f, jy = 0.f, jz = 0.f;
  static_for<Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    constexpr int j = V::rev(i);
    if constexpr (i != 0 && i < j) {
      const float s = d[i] + d[j];
      const float t = d[i] - d[j];
      r += s;
      if constexpr (V::ex(i) > 0) jx += t;
      if constexpr (V::ex(i) < 0) jx -= t;
      if constexpr (V::ey(i) > 0) jy += t;
      if constexpr (V::ey(i) < 0) jy -= t;
      if constexpr (V::ez(i) > 0) jz += t;
      if constexpr (V::ez(i) < 0) jz -= t;
    }
  });
  constexpr float kUnscale = 1.f / (float)(1 << SH);      // d = working value / 2^SH
  drho = r * kUnscale;
  rho = 1.f + drho;
  const float inv = 1.f / rho;
  ux = face ? 0.f : LBM_FMA(0.5f, fx, jx * kUnscale) * inv;
  uy = face ? 0.f : LBM_FMA(0.5f, fy, jy * kUnscale) * inv;
  uz = face ? 0.f : LBM_FMA(0.5f, fz, jz * kUnscale) * inv;
}

template <int Q, int SH = 0>
__device__ __forceinline__ void collide_dev(float d[Q], const Geom &g, float rho, float drho,
                                            float ux, float uy, float uz) {
  using V = VSet<Q>;
  const float u2 = LBM_FMA(ux, ux, LBM_FMA(uy, uy, uz * uz)) * (0.5f * g.inv_cs2);
  const float vx = ux * g.inv_cs2, vy = uy * g.inv_cs2, vz = uz * g.inv_cs2;
  const float om = g.inv_tau, keep = 1.f - g.inv_tau;
  const float orho = om * rho;
  const float c = om * LBM_FMA(-rho, u2, drho);
  static_for<Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    constexpr int j = V::rev(i);
    constexpr float w = V::w(i) * (float)(1 << SH);         // working units
    if constexpr (i == 0) {
      d[0] = LBM_FMA(d[0], keep, w * c);
    } else if constexpr (i < j) {
      const float t = edot<Q, i>(vx, vy, vz);
      const float a = LBM_FMA((orho * (0.5f * w)) * t, t, w * c);
      const float b = (orho * w) * t;
      d[i] = LBM_FMA(d[i], keep, a + b);
      d[j] = LBM_FMA(d[j], keep, a - b);
    }
  });
}

template <typename R>
__device__ __forceinline__ void flag_bad(unsigned *status, R rho, R ux, R uy, R uz) {
  if (status == nullptr) return;
  if (!(rho > R(0)) || !(rho < R(3.0e38))) atomicOr(status, LBM_STATUS_RHO_BAD);
  if (!(fabs(ux) + fabs(uy) + fabs(uz) < R(3.0e38))) atomicOr(status, LBM_STATUS_U_BAD);
}

}  // namespace lbm
