// Flow kernels: initialisation, the single-function kernels (collide /
// stream / moments / force) of the reference's FlowD3, and the C ABI of the
// fused step (kernels in lbm_step.cuh).
#include "lbm_step.cuh"

namespace lbm {

#define LBM_EXTERN_STEP(Q, S)                                                                 \
  extern template int run_step_qs<Q, S>(const StepArgs &, bool, int, int, cudaStream_t);      \
  extern template int run_step_batch_qs<Q, S>(const StepArgs *, const unsigned *, int, unsigned, \
                                              bool, int, cudaStream_t);                      \
  extern template int run_stats_qs<Q, S>(const StepArgs &, bool, unsigned long long *, cudaStream_t);
LBM_FOR_EACH_QS(LBM_EXTERN_STEP)
#undef LBM_EXTERN_STEP

static int run_step(const StepArgs &a, int q, int storage, bool force, int nodes, int threads,
                    cudaStream_t s) {
#define LBM_CASE_STEP(Q, S) \
  if (q == Q && storage == S) return run_step_qs<Q, S>(a, force, nodes, threads, s);
  LBM_FOR_EACH_QS(LBM_CASE_STEP)
#undef LBM_CASE_STEP
  set_error("Unknown parameter type: D3Q%d", q);
  return LBM_ERR_INVALID;
}

// ---------------------------------------------------------------------------
// Initialisation: f = f0 (or w), moments with FOL = 0 and the face rule,
// then two collisions with those same moments (LBMD3._init's cul_equ and
// step 1's cul_equ, which the reference runs before refreshing the moments).
// ---------------------------------------------------------------------------
// f0 and face_rho hold the storage's arithmetic type (float64 for FP64).
template <int Q, int S>
__global__ void __launch_bounds__(kThreads)
    k_init(const Geom g, const NodeDecomp dec, const void *f0_, void *fa_, void *face_rho_) {
  using V = VSet<Q>;
  using St = Storage<S>;
  using R = typename St::R;
  const unsigned idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= (unsigned)g.n) return;
  int x, y, z;
  dec(idx, x, y, z);
  const bool face = on_any_face(g, x, y, z);
  const R *f0 = static_cast<const R *>(f0_);
  R f[Q];
#pragma unroll
  for (int i = 0; i < Q; ++i) f[i] = f0 ? f0[(long long)i * g.n + idx] : V::template wr<R>(i);
  R rho, ux, uy, uz;
  moments<Q>(f, R(0), R(0), R(0), face, rho, ux, uy, uz);
  collide<Q>(f, g, rho, ux, uy, uz);
  collide<Q>(f, g, rho, ux, uy, uz);
  if (face && face_rho_ != nullptr) write_face_rho<Q>(g, static_cast<R *>(face_rho_), x, y, z, rho);
  typename St::T *fa = static_cast<typename St::T *>(fa_);
  const long long pidx = ((long long)x * g.ny + y) * g.pz + z;
  if (!lbm_in(pidx < g.np)) return;
#pragma unroll
  for (int i = 0; i < Q; ++i) St::store(fa + (long long)i * g.np + pidx, f[i], V::template wr<R>(i));
}

// ---------------------------------------------------------------------------
// Single-function kernels (float32 SoA), one reference method each.
// ---------------------------------------------------------------------------
template <int Q>
__global__ void __launch_bounds__(kThreads)
    k_collide(const Geom g, float *f, const float *rho, const float *u, float *feq) {
  const unsigned idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= (unsigned)g.n) return;
  const float r = rho[idx], ux = u[3ull * idx], uy = u[3ull * idx + 1], uz = u[3ull * idx + 2];
  float fl[Q];
  static_for<Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    fl[i] = f[(long long)i * g.n + idx];
  });
  if (feq != nullptr) {
    const float u2 = LBM_FMA(ux, ux, LBM_FMA(uy, uy, uz * uz)) * (0.5f * g.inv_cs2);
    static_for<Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      feq[(long long)i * g.n + idx] = feq_of<Q>(g, i, r, ux, uy, uz, u2);
    });
  }
  collide<Q>(fl, g, r, ux, uy, uz);
  static_for<Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    f[(long long)i * g.n + idx] = fl[i];
  });
}

// f_stream + f_stream_bound_* with every face code, NON_EQUILIBRIUM included.
template <int Q>
__global__ void __launch_bounds__(kThreads) k_stream(const Geom g, const NodeDecomp dec,
                                                     const float *fin, float *fout,
                                                     const float *rho, const float *feq) {
  using V = VSet<Q>;
  const unsigned idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= (unsigned)g.n) return;
  int x, y, z;
  dec(idx, x, y, z);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    int fc = -1;
    if (x == 0 && (V::ex(i) > 0 || g.face[0] == LBM_BC_NON_EQUILIBRIUM)) fc = 0;
    if (x == g.nx - 1 && (V::ex(i) < 0 || g.face[1] == LBM_BC_NON_EQUILIBRIUM)) fc = 1;
    if (V::ey(i) > 0 && y == 0) fc = 2;
    if (V::ey(i) < 0 && y == g.ny - 1) fc = 3;
    if (V::ez(i) > 0 && z == 0) fc = 4;
    if (V::ez(i) < 0 && z == g.nz - 1) fc = 5;
    float v;
    if (fc < 0) {
      v = fin[(long long)i * g.n + idx - ((long long)V::ex(i) * g.nyz + (long long)V::ey(i) * g.nz +
                                          V::ez(i))];
    } else {
      const int code = g.face[fc];
      if (code == LBM_BC_PERIODICAL) {
        int sx = x, sy = y, sz = z;
        const bool first = (fc & 1) == 0;
        if ((fc >> 1) == 0) sx = first ? g.nx - 1 : 0;
        else if ((fc >> 1) == 1) sy = first ? g.ny - 1 : 0;
        else sz = first ? g.nz - 1 : 0;
        v = fin[(long long)i * g.n + ((long long)sx * g.ny + sy) * g.nz + sz];
      } else if (code == LBM_BC_NON_EQUILIBRIUM) {
        const int nbx = fc == 0 ? 1 : g.nx - 2;
        const long long nb = ((long long)nbx * g.ny + y) * g.nz + z;
        const float rolled = pull_rolled<Q>(fin, g, i, nbx, y, z);
        v = feq[(long long)i * g.n + idx] + (rolled - feq[(long long)i * g.n + nb]);
      } else {
        v = fin[(long long)V::rev(i) * g.n + idx];
        if (code == LBM_BC_WALL_WITH_SPEED) {
          const float eu = (float)V::ex(i) * g.uw[fc][0] + (float)V::ey(i) * g.uw[fc][1] +
                           (float)V::ez(i) * g.uw[fc][2];
          v -= 2.f * (rho[idx] * V::w(i)) * eu * g.inv_cs2;
        }
      }
    }
    fout[(long long)i * g.n + idx] = v;
  }
}

__device__ __forceinline__ void atomic_max_nonneg(float *addr, float v) {
  if (v >= 0.f) atomicMax(reinterpret_cast<int *>(addr), __float_as_int(v));
}

template <int Q>
__global__ void __launch_bounds__(kThreads)
    k_moments(const Geom g, const NodeDecomp dec, const float *f, const float *fol, float *rho,
              float *u, float *p, float *rmax) {
  __shared__ float s_max[kThreads / 32];
  const unsigned idx = blockIdx.x * kThreads + threadIdx.x;
  float r = 0.f;
  if (idx < (unsigned)g.n) {
    int x, y, z;
    dec(idx, x, y, z);
    float fl[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) fl[i] = f[(long long)i * g.n + idx];
    const float fx = fol ? fol[3ull * idx] : 0.f, fy = fol ? fol[3ull * idx + 1] : 0.f,
                fz = fol ? fol[3ull * idx + 2] : 0.f;
    float ux, uy, uz;
    moments<Q>(fl, fx, fy, fz, on_any_face(g, x, y, z), r, ux, uy, uz);
    rho[idx] = r;
    if (p != nullptr) p[idx] = r / 3.0f;
    u[3ull * idx] = ux;
    u[3ull * idx + 1] = uy;
    u[3ull * idx + 2] = uz;
  }
  if (rmax == nullptr) return;  // uniform per launch
  for (int o = 16; o > 0; o >>= 1) r = fmaxf(r, __shfl_xor_sync(0xffffffffu, r, o));
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x < 32) {
    float m = threadIdx.x < kThreads / 32 ? s_max[threadIdx.x] : 0.f;
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) atomic_max_nonneg(rmax, m);
  }
}

// update_u_rou_boundary's NON_EQUILIBRIUM part (flow/d3/base.py:135-148): the
// inlet takes the duct profile scaled by Re mu / max(rho) / min(Y, Z) and the
// density of plane 1; the outlet copies plane X-2.  One thread per (y, z).
__global__ void k_neq_moments(const Geom g, float *rho, float *u, const float *rmax) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.nyz) return;
  const long long plane = g.nyz;
  if (g.face[0] == LBM_BC_NON_EQUILIBRIUM) {
    const float uw = (1.0f / *rmax) * g.re_mu / (float)(g.ny < g.nz ? g.ny : g.nz);
    u[3 * t] = (float)((double)uw * g.neq_profile[t]);
    rho[t] = rho[plane + t];
  }
  if (g.face[1] == LBM_BC_NON_EQUILIBRIUM) {
    const long long last = (long long)(g.nx - 1) * plane + t, prev = last - plane;
    rho[last] = rho[prev];
    for (int k = 0; k < 3; ++k) u[3 * last + k] = u[3 * prev + k];
  }
}

template <int Q>
__global__ void __launch_bounds__(kThreads)
    k_force(const Geom g, float *f, const float *u, const float *fol) {
  const unsigned idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= (unsigned)g.n) return;
  float fl[Q];
#pragma unroll
  for (int i = 0; i < Q; ++i) fl[i] = f[(long long)i * g.n + idx];
  add_force<Q>(fl, g, u[3ull * idx], u[3ull * idx + 1], u[3ull * idx + 2], fol[3ull * idx],
               fol[3ull * idx + 1], fol[3ull * idx + 2]);
#pragma unroll
  for (int i = 0; i < Q; ++i) f[(long long)i * g.n + idx] = fl[i];
}

// ---------------------------------------------------------------------------
// Dispatch helpers
// ---------------------------------------------------------------------------
template <template <int> class F, typename... A>
int dispatch_q(int q, A &&...args) {
  switch (q) {
    case 13: return F<13>::run(args...);
    case 15: return F<15>::run(args...);
    case 19: return F<19>::run(args...);
    case 27: return F<27>::run(args...);
    default: set_error("Unknown parameter type: D3Q%d", q); return LBM_ERR_INVALID;
  }
}

template <int Q>
struct RunInit {
  static int run(const Geom &g, const void *f0, void *fa, void *face_rho, int storage,
                 cudaStream_t s) {
    const unsigned nb = blocks_for(g.n, kThreads);
    const NodeDecomp dec = make_decomp(g);
    switch (storage) {
      case LBM_STORAGE_FP32:
        k_init<Q, LBM_STORAGE_FP32><<<nb, kThreads, 0, s>>>(g, dec, f0, fa, face_rho);
        break;
      case LBM_STORAGE_FP16S:
        k_init<Q, LBM_STORAGE_FP16S><<<nb, kThreads, 0, s>>>(g, dec, f0, fa, face_rho);
        break;
      case LBM_STORAGE_FP64:
        k_init<Q, LBM_STORAGE_FP64><<<nb, kThreads, 0, s>>>(g, dec, f0, fa, face_rho);
        break;
      default:
        k_init<Q, LBM_STORAGE_BF16S><<<nb, kThreads, 0, s>>>(g, dec, f0, fa, face_rho);
        break;
    }
    LBM_LAUNCH_CHECK("lbm_flow_init");
    return LBM_OK;
  }
};

template <int Q>
struct RunCollide {
  static int run(const Geom &g, float *f, const float *rho, const float *u, float *feq,
                 cudaStream_t s) {
    k_collide<Q><<<blocks_for(g.n, kThreads), kThreads, 0, s>>>(g, f, rho, u, feq);
    LBM_LAUNCH_CHECK("lbm_collide");
    return LBM_OK;
  }
};

template <int Q>
struct RunStream {
  static int run(const Geom &g, const float *fin, float *fout, const float *rho, const float *feq,
                 cudaStream_t s) {
    k_stream<Q><<<blocks_for(g.n, kThreads), kThreads, 0, s>>>(g, make_decomp(g), fin, fout, rho,
                                                               feq);
    LBM_LAUNCH_CHECK("lbm_stream");
    return LBM_OK;
  }
};

template <int Q>
struct RunMoments {
  static int run(const Geom &g, const float *f, const float *fol, float *rho, float *u, float *p,
                 float *rmax, cudaStream_t s) {
    k_moments<Q><<<blocks_for(g.n, kThreads), kThreads, 0, s>>>(g, make_decomp(g), f, fol, rho, u,
                                                                p, rmax);
    LBM_LAUNCH_CHECK("lbm_moments");
    return LBM_OK;
  }
};

template <int Q>
struct RunForce {
  static int run(const Geom &g, float *f, const float *u, const float *fol, cudaStream_t s) {
    k_force<Q><<<blocks_for(g.n, kThreads), kThreads, 0, s>>>(g, f, u, fol);
    LBM_LAUNCH_CHECK("lbm_add_force");
    return LBM_OK;
  }
};

// StepArgs of one fused step (shared by lbm_flow_step and lbm_batch_pack).
static int build_step_args(const lbm_lattice *lat, const void *fa, void *fb, const lbm_force *force,
                           const float *face_rho_in, float *face_rho_out, const lbm_observe *obs,
                           uint32_t *status, StepArgs &a, bool &use_force, const char *who) {
  int rc = check_lattice(lat);
  if (rc) return rc;
  if (any_face(lat, LBM_BC_NON_EQUILIBRIUM)) {
    set_error("%s: NON_EQUILIBRIUM faces need the global inlet density; run them "
              "through lbm_collide / lbm_stream / lbm_moments / lbm_add_force", who);
    return LBM_ERR_UNSUPPORTED;
  }
  if (fa == nullptr) {
    set_error("%s: input populations are NULL", who);
    return LBM_ERR_INVALID;
  }
  const bool wws = any_face(lat, LBM_BC_WALL_WITH_SPEED);
  if (wws && face_rho_in == nullptr) {
    set_error("%s: WALL_WITH_SPEED faces need face_rho_in", who);
    return LBM_ERR_INVALID;
  }
  memset(&a, 0, sizeof(a));
  a.g = make_geom(lat);
  a.dec = make_decomp(a.g);
  a.pdec = NodeDecomp{make_fastdiv((unsigned)a.g.pz), make_fastdiv((unsigned)a.g.ny)};
  a.fa = fa;
  a.fb = fb;
  use_force = false;
  if (force != nullptr) {
    for (int k = 0; k < 3; ++k) {
      a.go[k] = force->old_uniform[k];
      a.gn[k] = force->new_uniform[k];
      use_force = use_force || a.go[k] != 0.f || a.gn[k] != 0.f;
    }
    a.fol_old = force->old_field;
    a.fol_new = force->new_field;
    a.ch_old = force->old_chunks;
    a.ch_new = force->new_chunks;
    use_force = use_force || a.fol_old != nullptr || a.fol_new != nullptr;
  }
  a.face_rho_in = face_rho_in;
  a.face_rho_out = wws ? face_rho_out : nullptr;
  if (obs != nullptr) {
    a.obs_f = obs->f;
    a.obs_rho = obs->rho;
    a.obs_u = obs->u;
  }
  a.status = status;
  fill_step_planes(a.g, lat->q, lat->storage, fa, fb, a.p);
  return LBM_OK;
}

}  // namespace lbm

using namespace lbm;

extern "C" {

int lbm_flow_init(const lbm_lattice *lat, const float *f0, void *fa, float *face_rho,
                  void *stream) {
  int rc = check_lattice(lat);
  if (rc) return rc;
  if (fa == nullptr) {
    set_error("lbm_flow_init: population buffer is NULL");
    return LBM_ERR_INVALID;
  }
  if ((any_face(lat, LBM_BC_WALL_WITH_SPEED) || any_face(lat, LBM_BC_NON_EQUILIBRIUM)) &&
      face_rho == nullptr) {
    set_error("lbm_flow_init: WALL_WITH_SPEED / NON_EQUILIBRIUM faces need face_rho");
    return LBM_ERR_INVALID;
  }
  const Geom g = make_geom(lat);
  return dispatch_q<RunInit>(lat->q, g, static_cast<const void *>(f0), fa,
                             static_cast<void *>(face_rho), lat->storage, (cudaStream_t)stream);
}

int lbm_flow_step(const lbm_lattice *lat, const void *fa, void *fb, const lbm_force *force,
                  const float *face_rho_in, float *face_rho_out, const lbm_observe *obs,
                  uint32_t *status, void *stream) {
  StepArgs a;
  bool use_force = false;
  int rc = build_step_args(lat, fa, fb, force, face_rho_in, face_rho_out, obs, status, a,
                           use_force, "lbm_flow_step");
  if (rc) return rc;
  const int bits = storage_bits(lat->storage);
  if (lat->step_nodes != 0 && lat->step_nodes != LBM_STEP_ROWS &&
      !step_shape_legal(lat->step_nodes, a.g.pz, bits)) {
    set_error("lbm_flow_step: %d nodes per thread does not fit rows of pitch %d (%d-bit storage)",
              lat->step_nodes, a.g.pz, bits);
    return LBM_ERR_INVALID;
  }
  if (lat->step_threads != 0 && lat->step_threads != 128 && lat->step_threads != 256) {
    set_error("lbm_flow_step: step_threads must be 128 or 256");
    return LBM_ERR_INVALID;
  }
  return run_step(a, lat->q, lat->storage, use_force, (int)lat->step_nodes,
                  (int)lat->step_threads, (cudaStream_t)stream);
}

int lbm_flow_stats(const lbm_lattice *lat, const void *fa, const lbm_force *force,
                   const float *face_rho_in, double *out, uint32_t *status, void *stream) {
  if (out == nullptr) {
    set_error("lbm_flow_stats: needs an output buffer of 9 doubles");
    return LBM_ERR_INVALID;
  }
  StepArgs a;
  bool use_force = false;
  int rc = build_step_args(lat, fa, nullptr, force, face_rho_in, nullptr, nullptr, status, a,
                           use_force, "lbm_flow_stats");
  if (rc) return rc;
  unsigned long long *slots = reinterpret_cast<unsigned long long *>(out);
  cudaStream_t s = (cudaStream_t)stream;
#define LBM_CASE_STATS(Q, S) \
  if (lat->q == Q && lat->storage == S) return run_stats_qs<Q, S>(a, use_force, slots, s);
  LBM_FOR_EACH_QS(LBM_CASE_STATS)
#undef LBM_CASE_STATS
  set_error("Unknown parameter type: D3Q%d", lat->q);
  return LBM_ERR_INVALID;
}

size_t lbm_batch_entry_bytes(void) { return sizeof(StepArgs); }

int lbm_batch_pack(const lbm_lattice *lat, const void *fa, void *fb, const lbm_force *force,
                   const float *face_rho_in, float *face_rho_out, uint32_t *status, int32_t nodes,
                   void *entry, uint32_t *blocks) {
  if (entry == nullptr || blocks == nullptr) {
    set_error("lbm_batch_pack: entry and blocks are required");
    return LBM_ERR_INVALID;
  }
  if (fb == nullptr) {
    set_error("lbm_batch_pack: a batched step needs an output buffer");
    return LBM_ERR_INVALID;
  }
  StepArgs a;
  bool use_force = false;
  int rc = build_step_args(lat, fa, fb, force, face_rho_in, face_rho_out, nullptr, status, a,
                           use_force, "lbm_batch_pack");
  if (rc) return rc;
  const int bits = storage_bits(lat->storage);
  if (nodes != 1 && !((nodes == 2 || nodes == 4) && step_shape_ok(nodes, a.g.pz, bits))) {
    set_error("lbm_batch_pack: nodes per thread must be 1, or 2 / 4 for rows of a multiple of "
              "that many nodes (at least twice as many)");
    return LBM_ERR_INVALID;
  }
  const long long per_block = (nodes == 1 ? 256 : 128) * (long long)kBatchTiles;
  const long long work = nodes == 1 ? a.g.n : a.g.np / nodes;
  *blocks = (uint32_t)((work + per_block - 1) / per_block);
  memcpy(entry, &a, sizeof(a));
  return LBM_OK;
}

int lbm_flow_step_batch(int32_t q, int32_t storage, int32_t nodes, int32_t force,
                        const void *entries, const uint32_t *block_begin, int32_t count,
                        uint32_t total_blocks, void *stream) {
  if (entries == nullptr || block_begin == nullptr || count <= 0 || total_blocks == 0) {
    set_error("lbm_flow_step_batch: empty batch");
    return LBM_ERR_INVALID;
  }
  if (nodes != 1 && nodes != 2 && nodes != 4) {
    set_error("lbm_flow_step_batch: nodes per thread must be 1, 2 or 4");
    return LBM_ERR_INVALID;
  }
  const StepArgs *e = static_cast<const StepArgs *>(entries);
  cudaStream_t s = (cudaStream_t)stream;
#define LBM_CASE_BATCH(Q, S)                                                             \
  if (q == Q && storage == S)                                                            \
    return run_step_batch_qs<Q, S>(e, block_begin, count, total_blocks, force != 0, nodes, s);
  LBM_FOR_EACH_QS(LBM_CASE_BATCH)
#undef LBM_CASE_BATCH
  set_error("lbm_flow_step_batch: unknown velocity set D3Q%d or storage %d", q, storage);
  return LBM_ERR_INVALID;
}

int lbm_collide(const lbm_lattice *lat, float *f, const float *rho, const float *u, float *feq,
                void *stream) {
  int rc = check_lattice(lat);
  if (rc) return rc;
  if (lat->pz != 0 && lat->pz != lat->nz) {
    set_error("lbm_collide: the single-function calls take dense arrays (pz = 0 or nz)");
    return LBM_ERR_INVALID;
  }
  if (f == nullptr || rho == nullptr || u == nullptr) {
    set_error("lbm_collide: f, rho and u are required");
    return LBM_ERR_INVALID;
  }
  return dispatch_q<RunCollide>(lat->q, make_geom(lat), f, rho, u, feq, (cudaStream_t)stream);
}

int lbm_stream(const lbm_lattice *lat, const float *f_in, float *f_out, const float *rho,
               const float *feq, void *stream) {
  int rc = check_lattice(lat);
  if (rc) return rc;
  if (lat->pz != 0 && lat->pz != lat->nz) {
    set_error("lbm_stream: the single-function calls take dense arrays (pz = 0 or nz)");
    return LBM_ERR_INVALID;
  }
  if (f_in == nullptr || f_out == nullptr || f_in == f_out) {
    set_error("lbm_stream: needs distinct input and output buffers");
    return LBM_ERR_INVALID;
  }
  if (any_face(lat, LBM_BC_WALL_WITH_SPEED) && rho == nullptr) {
    set_error("lbm_stream: WALL_WITH_SPEED faces need rho");
    return LBM_ERR_INVALID;
  }
  if (any_face(lat, LBM_BC_NON_EQUILIBRIUM) && feq == nullptr) {
    set_error("lbm_stream: NON_EQUILIBRIUM faces need feq");
    return LBM_ERR_INVALID;
  }
  return dispatch_q<RunStream>(lat->q, make_geom(lat), f_in, f_out, rho, feq,
                               (cudaStream_t)stream);
}

int lbm_moments(const lbm_lattice *lat, const float *f, const float *fol, float *rho, float *u,
                float *p, float *scratch, void *stream) {
  int rc = check_lattice(lat);
  if (rc) return rc;
  if (lat->pz != 0 && lat->pz != lat->nz) {
    set_error("lbm_moments: the single-function calls take dense arrays (pz = 0 or nz)");
    return LBM_ERR_INVALID;
  }
  if (f == nullptr || rho == nullptr || u == nullptr) {
    set_error("lbm_moments: f, rho and u are required");
    return LBM_ERR_INVALID;
  }
  const bool neq = any_face(lat, LBM_BC_NON_EQUILIBRIUM);
  const bool neq_in = lat->face[0] == LBM_BC_NON_EQUILIBRIUM;
  if (neq_in && scratch == nullptr) {
    set_error("lbm_moments: a NON_EQUILIBRIUM input face needs one float of scratch");
    return LBM_ERR_INVALID;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const Geom g = make_geom(lat);
  if (neq_in) {
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(float), s);
    if (e != cudaSuccess) return fail_cuda(e, "lbm_moments");
  }
  rc = dispatch_q<RunMoments>(lat->q, g, f, fol, rho, u, p, neq_in ? scratch : nullptr, s);
  if (rc || !neq) return rc;
  k_neq_moments<<<blocks_for(g.nyz, 128), 128, 0, s>>>(g, rho, u, scratch);
  LBM_LAUNCH_CHECK("lbm_moments");
  return LBM_OK;
}

int lbm_add_force(const lbm_lattice *lat, float *f, const float *u, const float *fol,
                  void *stream) {
  int rc = check_lattice(lat);
  if (rc) return rc;
  if (lat->pz != 0 && lat->pz != lat->nz) {
    set_error("lbm_add_force: the single-function calls take dense arrays (pz = 0 or nz)");
    return LBM_ERR_INVALID;
  }
  if (f == nullptr || u == nullptr || fol == nullptr) {
    set_error("lbm_add_force: f, u and FOL are required");
    return LBM_ERR_INVALID;
  }
  return dispatch_q<RunForce>(lat->q, make_geom(lat), f, u, fol, (cudaStream_t)stream);
}

}  // extern "C"
