// Host-side helpers shared by the C-ABI translation units: error reporting,
// lattice validation, Geom construction, fast index division.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "lbm_lattice.cuh"

namespace lbm {

void set_error(const char *fmt, ...);
int fail_cuda(cudaError_t e, const char *where);
int check_lattice(const lbm_lattice *lat);  // LBM_OK or an error code (message set)
Geom make_geom(const lbm_lattice *lat);
// pull-source / face-source / destination plane pointers of a lattice step
void fill_step_planes(const Geom &g, int q, int storage, const void *fa, void *fb, StepPlanes &p);
bool any_face(const lbm_lattice *lat, int code);
// bits of one stored population
inline int storage_bits(int storage) {
  return storage == LBM_STORAGE_FP32 ? 32 : storage == LBM_STORAGE_FP64 ? 64 : 16;
}
// default poll limit of every bounded mbarrier wait in the TMA-staged step
constexpr unsigned kTmaWaitPollsDefault = 1u << 24;
// poll limit of its consumer waits for the next launches (lbm_debug_set_wait_limit)
unsigned tma_wait_polls();

// Bounds-checked build: every translation unit registers a reader of its own
// violation counter (g_lbm_oob) with the library (lbm_debug_bounds_faults).
using OobReader = unsigned long long (*)(bool reset);
void register_oob_reader(OobReader r);
#ifdef LBM_BOUNDS_CHECK
namespace {
unsigned long long read_oob(bool reset) {
  unsigned long long v = 0;
  if (cudaMemcpyFromSymbol(&v, g_lbm_oob, sizeof(v)) != cudaSuccess) return ~0ull;
  if (reset) {
    const unsigned long long z = 0;
    cudaMemcpyToSymbol(g_lbm_oob, &z, sizeof(z));
  }
  return v;
}
struct OobRegistration {
  OobRegistration() { register_oob_reader(read_oob); }
};
const OobRegistration oob_registration;
}  // namespace
#endif

// Launch-error check after a kernel launch.
#define LBM_LAUNCH_CHECK(where)                              \
  do {                                                       \
    cudaError_t e__ = cudaGetLastError();                    \
    if (e__ != cudaSuccess) return ::lbm::fail_cuda(e__, where); \
  } while (0)

// Division of node indices (< 2^31) by a lattice extent d (< 2^31) with one
// high multiply: m = ceil(2^(31+l) / d), l = ceil(log2 d), so that
// floor(n / d) = floor(n * m / 2^(31+l)) for every n < 2^31 (the error term
// n * (m - 2^(31+l)/d) / 2^(31+l) stays below 1/d).
struct FastDiv {
  unsigned d, m, s;  // s = l - 1; d == 1 is special-cased with m == 0
};

inline FastDiv make_fastdiv(unsigned d) {
  FastDiv f{d, 0u, 0u};
  if (d <= 1) return f;
  unsigned l = 0;
  while ((1ull << l) < d) ++l;
  const unsigned long long p = 1ull << (31 + l);
  f.m = (unsigned)((p + d - 1) / d);
  f.s = l - 1;
  return f;
}

__device__ __forceinline__ unsigned fdiv(unsigned n, const FastDiv &f) {
  return f.m == 0 ? n : (__umulhi(n, f.m) >> f.s);
}

// (x, y, z) of node idx
struct NodeDecomp {
  FastDiv dz, dy;
  __device__ __forceinline__ void operator()(unsigned idx, int &x, int &y, int &z) const {
    const unsigned t = fdiv(idx, dz);
    z = (int)(idx - t * dz.d);
    const unsigned xx = fdiv(t, dy);
    y = (int)(t - xx * dy.d);
    x = (int)xx;
  }
};

inline NodeDecomp make_decomp(const Geom &g) {
  return NodeDecomp{make_fastdiv((unsigned)g.nz), make_fastdiv((unsigned)g.ny)};
}

inline unsigned blocks_for(long long n, int threads) {
  return (unsigned)((n + threads - 1) / threads);
}

}  // namespace lbm
