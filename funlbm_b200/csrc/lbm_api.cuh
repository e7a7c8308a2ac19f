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

// Whether the per-step kernels are launched chained (programmatic dependent
// launch, see chain_wait): on unless FUNLBM_B200_CHAIN=0 in the environment
// (read once).
bool chained_launches();

// Launch kernel k with programmatic stream serialization when chained
// launches are on and stream s is not being captured into a CUDA graph; the
// kernel must begin with chain_enter().  Measured on B200 the chained form
// takes the launch gaps out of eagerly issued steps (sphere free fall,
// 161 x 65 x 65: 73 -> 59 us per LBMD3.run_step) and gains nothing inside
// graph replays, where the gaps are already small, while kernels that wait
// on the GPU would hold SM slots that the concurrent graphs of a served
// stream can use -- so captured launches stay plain.  The result is also
// recorded as the thread's last CUDA error, as for <<< >>> launches.
template <typename... P, typename... A>
cudaError_t launch_chained(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                           A &&...args) {
  bool chain = chained_launches();
  if (chain) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
      (void)cudaGetLastError();   // (the query's own error is not the launch's)
      chain = false;
    } else if (cs != cudaStreamCaptureStatusNone) {
      chain = false;
    }
  }
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = chain ? 1 : 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

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
