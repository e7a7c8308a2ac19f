// Immersed boundary coupling and rigid particles: interpolation (fused with
// the moment pass it reads), wall spring + Newton-Euler update, spreading,
// and the rotation-vector marker update.
#include <algorithm>
#include <mutex>

#include "lbm_api.cuh"

namespace lbm {

constexpr int kStencil = 64;                // 4 x 4 x 4 nodes per marker
constexpr int kMarkersPerBlock = 4;         // interpolation / spreading blocks
constexpr int kIbmThreads = kStencil * kMarkersPerBlock;
constexpr int kRigidThreads = 512;

// Stencil box of lbm/lbm3d.py:32-44 for marker position `l` on one axis:
// lo = max(floor(l) - 1, 0), hi = min(lo + 4, size) with size = nodes - 1
// (the reference clamps to the configured size, so the last node is never
// part of a stencil).  Computed in float32 like the reference.
// lo is also capped at size (the box is then empty) so that markers far
// outside the domain (or non-finite) never produce an out-of-range index.
// R is the arithmetic type: float, or double for FP64 lattices.
template <typename R>
__device__ __forceinline__ void box_axis(R l, int size, int &lo, int &hi) {
  R rl = floor(l) - R(1);
  rl = fmax(rl, R(0));
  R rr = fmin(rl + R(4), (R)size);
  rl = fmin(rl, (R)size);
  rr = fmax(rr, R(0));
  lo = (int)rl;
  hi = (int)rr;
}

// 4-point cosine delta of lbm/lbm3d.py:46-64, one axis:
// (1 + cos(|r pi / 2|)) / 4, and the |r| <= 2 test of the mask.
template <typename R>
__device__ __forceinline__ R delta_axis(R r, bool &inside) {
  inside = inside && (fabs(r) <= R(2));
  const R arg = fabs(r * R(3.14159265358979323846) / R(2));
  return (R(1) + cos(arg)) / R(4);
}

// Unnormalised weight of stencil slot j of a marker at `l`; false if the slot
// is outside the (clamped) box.
template <typename R>
__device__ __forceinline__ bool stencil_slot(const Geom &g, const R l[3], int j, int &x, int &y,
                                             int &z, R &w) {
  int lo[3], hi[3];
  box_axis(l[0], g.nx - 1, lo[0], hi[0]);
  box_axis(l[1], g.ny - 1, lo[1], hi[1]);
  box_axis(l[2], g.nz - 1, lo[2], hi[2]);
  x = lo[0] + (j >> 4);
  y = lo[1] + ((j >> 2) & 3);
  z = lo[2] + (j & 3);
  if (x >= hi[0] || y >= hi[1] || z >= hi[2]) return false;
  bool in = true;
  const R wx = delta_axis((R)x - l[0], in);
  const R wy = delta_axis((R)y - l[1], in);
  const R wz = delta_axis((R)z - l[2], in);
  w = in ? (wx * wy) * wz : R(0);
  return true;
}

// Sum over the 64 stencil threads of one marker (two warps) via shared memory.
template <int N, typename R>
__device__ __forceinline__ void stencil_sum(R (&v)[N], R (*sh)[kMarkersPerBlock * 2], int slot,
                                            int mk) {
#pragma unroll
  for (int k = 0; k < N; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  const int lane = threadIdx.x & 31;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) sh[k][mk * 2 + (slot >> 5)] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < N; ++k) v[k] = sh[k][mk * 2] + sh[k][mk * 2 + 1];
}

// The particle arrays of an lbm_particles in the arithmetic type R (its
// `float *` members hold float64 when the struct's fp64 flag is set).
template <typename R>
struct PView {
  const int32_t *offset, *owner;
  const R *lagrange, *lm, *mass, *inertia, *rou;
  R *lx, *lu, *lF, *lrou, *cx, *cu, *cw, *cF, *cT, *angle;
};

template <typename R>
__device__ __forceinline__ PView<R> pview(const lbm_particles &p) {
  PView<R> v;
  v.offset = p.marker_offset;
  v.owner = p.marker_owner;
  v.lagrange = reinterpret_cast<const R *>(p.lagrange);
  v.lm = reinterpret_cast<const R *>(p.lm);
  v.mass = reinterpret_cast<const R *>(p.mass);
  v.inertia = reinterpret_cast<const R *>(p.inertia);
  v.rou = reinterpret_cast<const R *>(p.rou);
  v.lx = reinterpret_cast<R *>(p.lx);
  v.lu = reinterpret_cast<R *>(p.lu);
  v.lF = reinterpret_cast<R *>(p.lF);
  v.lrou = reinterpret_cast<R *>(p.lrou);
  v.cx = reinterpret_cast<R *>(p.cx);
  v.cu = reinterpret_cast<R *>(p.cu);
  v.cw = reinterpret_cast<R *>(p.cw);
  v.cF = reinterpret_cast<R *>(p.cF);
  v.cT = reinterpret_cast<R *>(p.cT);
  v.angle = reinterpret_cast<R *>(p.angle);
  return v;
}

// ---------------------------------------------------------------------------
// Interpolation: thread = (marker, stencil slot).
// ---------------------------------------------------------------------------
struct InterpArgs {
  Geom g;
  const void *fa;
  const void *u_field, *rho_field;   // arithmetic type of the lattice
  float go[3];
  const void *fol_old;
  const void *face_rho_in;
  lbm_particles p;
  float dt;
  int step;
  unsigned *status;
  StepPlanes planes;   // pull sources of fa (interior rows)
  int wall;            // apply the wall spring at the extreme markers
  float size[3];       // wall positions: nodes - 1 per axis
  float dx;
  // The first half of reference-mode spreading, fused in (ibm_interpolate_
  // wall_claim; NULL otherwise): every in-box stencil node of every marker is
  // claimed in claim_owner (largest marker index), and the blocks from
  // interp_blocks on clear the chunks of clear_field flagged in clear_chunks
  // (k_spread_clear's work).  interp_blocks: blocks of the interpolation.
  int32_t *claim_owner;
  void *clear_field;
  uint8_t *clear_chunks;
  unsigned interp_blocks;
};

// Wall spring of LBMD3.particle_to_wall (lbm/lbm3d.py:121-167) for marker m
// of particle pi, whose force after interpolation is lf: k0 = 300 times
// (1 - distance / (2 dx)), clamped at 0, along the wall normal, at the six
// extreme markers `ext` (least x, y, z, greatest x, y, z); the reference's
// indexed += reads all six old forces and the last of duplicate entries
// wins; nothing happens when all six distances give 0.
template <typename R>
__device__ __forceinline__ void wall_spring(const PView<R> &P, const int32_t *ext, int m, int pi,
                                            const float size[3], float dx, R lf[3]) {
  const int m0 = P.offset[pi], m1 = P.offset[pi + 1];
  bool valid = m1 > m0;
  for (int k = 0; k < 6; ++k) valid = valid && ext[k] >= m0 && ext[k] < m1;
  if (!valid) return;
  bool mine = false;
  for (int k = 0; k < 6; ++k) mine = mine || ext[k] == m;
  if (!mine) return;
  const R k0 = R(300);
  R d[6], dmax = R(0);
  for (int k = 0; k < 6; ++k) {
    const R c = P.lx[3 * ext[k] + (k % 3)];
    const R b = k < 3 ? R(0) : (R)size[k - 3];
    d[k] = fmax(k0 * (R(1) - fabs(c - b) / (R(2) * (R)dx)), R(0));
    dmax = fmax(dmax, d[k]);
  }
  if (dmax == R(0)) return;
  R out[3] = {lf[0], lf[1], lf[2]};
  for (int k = 0; k < 6; ++k) {
    if (ext[k] != m) continue;
    for (int c = 0; c < 3; ++c) {
      const R nrm = (c == k % 3) ? (k < 3 ? R(1) : R(-1)) : R(0);
      out[c] = lf[c] + nrm * d[k];
    }
  }
  lf[0] = out[0];
  lf[1] = out[1];
  lf[2] = out[2];
}

// Clear the chunks of `field` flagged in `chunks` (the chunks written the last
// time this buffer was used) and reset their flags.  Each lane reads the flag
// of chunk `chunk`; the warp then clears its flagged chunks together (3 values
// per lane per chunk), so a mostly flagged small lattice costs no more than a
// sparse large one.  Called by whole warps.
template <typename R>
__device__ __forceinline__ void clear_flagged_chunks(long long chunk, long long n, R *field,
                                                     uint8_t *chunks) {
  const long long nchunks = (n + 31) >> 5;
  const int lane = threadIdx.x & 31;
  const bool mine = chunk < nchunks && chunks[chunk] != 0;
  unsigned todo = __ballot_sync(0xffffffffu, mine);
  const long long base = chunk - lane;   // first chunk of this warp
  while (todo != 0) {
    const int j = __ffs(todo) - 1;
    todo &= todo - 1;
    const long long first = (base + j) * 32;
    const long long count = 3 * ((first + 32 < n ? first + 32 : n) - first);
    for (long long k = lane; k < count; k += 32) field[3 * first + k] = R(0);
  }
  if (mine) chunks[chunk] = 0;
}

template <int Q, int S>
__global__ void __launch_bounds__(kIbmThreads) k_interp(const InterpArgs a) {
  chain_enter();
  using R = typename Storage<S>::R;
  if (blockIdx.x >= a.interp_blocks) {   // (the grid has such blocks only with clear_chunks)
    clear_flagged_chunks<R>((long long)(blockIdx.x - a.interp_blocks) * blockDim.x + threadIdx.x,
                            a.g.n, static_cast<R *>(a.clear_field), a.clear_chunks);
    return;
  }
  __shared__ R sh[3][kMarkersPerBlock * 2];
  const PView<R> P = pview<R>(a.p);
  const int mk = threadIdx.x / kStencil, slot = threadIdx.x % kStencil;
  const int m = blockIdx.x * kMarkersPerBlock + mk;
  const bool live = m < a.p.n_markers;
  R acc[3] = {R(0), R(0), R(0)};  // sum w, sum w (ux+uy+uz), sum w rho
  R l[3] = {R(0), R(0), R(0)};
  if (live) {
    l[0] = P.lx[3 * m];
    l[1] = P.lx[3 * m + 1];
    l[2] = P.lx[3 * m + 2];
    int x, y, z;
    R w;
    if (stencil_slot(a.g, l, slot, x, y, z, w)) {
      bool node_ok = true;
      if (!lbm_in(x >= 0 && x < a.g.nx && y >= 0 && y < a.g.ny && z >= 0 && z < a.g.nz)) {
        x = 0;
        y = 0;
        z = 0;
        node_ok = false;
      }
      const long long idx = ((long long)x * a.g.ny + y) * a.g.nz + z;
      // (the claim of spreading's pass 0, on the same positions)
      if (a.claim_owner != nullptr && node_ok) atomicMax(a.claim_owner + idx, m);
      R rho, ux, uy, uz;
      if (a.fa != nullptr) {
        const typename Storage<S>::T *fa = static_cast<const typename Storage<S>::T *>(a.fa);
        const R *face_rho = static_cast<const R *>(a.face_rho_in);
        R f[Q];
        const unsigned pidx = (unsigned)(((long long)x * a.g.ny + y) * a.g.pz + z);
        if (x > 0 && x < a.g.nx - 1 && y > 0 && y < a.g.ny - 1)
          pull_row_node<Q, S, false>(a.planes, a.g, face_rho, pidx, x, y, z, f);
        else
          pull_general<Q, S>(fa, a.g, x, y, z, face_rho, f);
        R fx = a.go[0], fy = a.go[1], fz = a.go[2];
        if (a.fol_old != nullptr) {
          const R *fol = static_cast<const R *>(a.fol_old);
          fx += fol[3 * idx];
          fy += fol[3 * idx + 1];
          fz += fol[3 * idx + 2];
        }
        moments<Q>(f, fx, fy, fz, on_any_face(a.g, x, y, z), rho, ux, uy, uz);
      } else {
        const R *rf = static_cast<const R *>(a.rho_field);
        const R *uf = static_cast<const R *>(a.u_field);
        rho = rf[idx];
        ux = uf[3 * idx];
        uy = uf[3 * idx + 1];
        uz = uf[3 * idx + 2];
      }
      acc[0] = w;
      acc[1] = w * ((ux + uy) + uz);
      acc[2] = w * rho;
    }
  }
  stencil_sum<3>(acc, sh, slot, mk);
  if (!live || slot != 0) return;
  const R W = acc[0];
  const R lus = W > R(0) ? acc[1] / W : acc[1];
  const R lrho = W > R(0) ? acc[2] / W : acc[2];
  if (!(W > R(0)) && a.step > 100 && a.status != nullptr) atomicOr(a.status, LBM_STATUS_STENCIL_EMPTY);
  const int pi = P.owner[m];
  const R rx = l[0] - P.cx[3 * pi], ry = l[1] - P.cx[3 * pi + 1], rz = l[2] - P.cx[3 * pi + 2];
  const R wx = P.cw[3 * pi], wy = P.cw[3 * pi + 1], wz = P.cw[3 * pi + 2];
  const R v[3] = {P.cu[3 * pi] + (wy * rz - wz * ry), P.cu[3 * pi + 1] + (wz * rx - wx * rz),
                  P.cu[3 * pi + 2] + (wx * ry - wy * rx)};
  R lf[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    P.lu[3 * m + k] = v[k];
    lf[k] = (R(2) * lrho) * (v[k] - lus) / (R)a.dt;
  }
  if (a.wall) wall_spring<R>(P, a.p.extreme + 6 * pi, m, pi, a.size, a.dx, lf);
#pragma unroll
  for (int k = 0; k < 3; ++k) P.lF[3 * m + k] = lf[k];
  P.lrou[m] = lrho;
}

// ---------------------------------------------------------------------------
// Wall spring (lbm/lbm3d.py:121-167) + update_from_lar
// (particle/base/base.py:120-151).  One block per particle.
// ---------------------------------------------------------------------------
struct RigidArgs {
  lbm_particles p;
  int what;
  float size[3];
  float dt, dx, gl, rouf;
};

template <typename R>
__device__ __forceinline__ void argext_merge(R &v, int &i, R v2, int i2, bool want_min) {
  const bool better = want_min ? (v2 < v || (v2 == v && i2 < i)) : (v2 > v || (v2 == v && i2 < i));
  if (better) {
    v = v2;
    i = i2;
  }
}

// Newton-Euler update of particle pi (update_from_lar, particle/base/
// base.py:120-152), one block: a single pass over the markers gives the
// float64 sums A = sum lF lm and B = sum (lx x lF) lm, then thread 0 writes
// cF = -A + (1 - rho_p / rho_f) mass [gl, 0, 0], cu, cx, and the torque about
// the new centre, cT = -(B - cx x A): the reference's -sum((lx - cx) x lF lm)
// with the centre taken out of the sum, so the torque needs no second pass
// after cx is known.  With s_ang set, also angle += cw (particle/coord.py:
// 107).  Returns with s_cx (and s_ang) filled for every thread.
template <typename R>
__device__ __forceinline__ void rigid_update_block(const RigidArgs &a, const PView<R> &P, int pi,
                                                   int m0, int m1,
                                                   double (*s_sum)[kRigidThreads / 32], R *s_cx,
                                                   R *s_ang) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  // Thread 0's particle state, loaded before the marker sums: the update
  // below interleaves its stores with these reads, which would otherwise
  // each wait out a memory round trip after the barrier.  Nothing in this
  // block writes them before the update.
  R p_mass = R(0), p_rou = R(0), p_cu[3] = {}, p_cx[3] = {}, p_cw[3] = {}, p_in[3] = {},
    p_ang[3] = {};
  if (threadIdx.x == 0) {
    p_mass = P.mass[pi];
    p_rou = P.rou[pi];
    for (int k = 0; k < 3; ++k) {
      p_cu[k] = P.cu[3 * pi + k];
      p_cx[k] = P.cx[3 * pi + k];
      p_cw[k] = P.cw[3 * pi + k];
      p_in[k] = P.inertia[3 * pi + k];
      if (s_ang != nullptr) p_ang[k] = P.angle[3 * pi + k];
    }
  }
  double sm[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  // (unrolled so that the loads of several markers are in flight together;
  // the sums keep their marker order)
#pragma unroll 4
  for (int m = m0 + threadIdx.x; m < m1; m += kRigidThreads) {
    const double lm = P.lm[m];
    const double fx = (double)P.lF[3 * m] * lm, fy = (double)P.lF[3 * m + 1] * lm,
                 fz = (double)P.lF[3 * m + 2] * lm;
    const double x = P.lx[3 * m], y = P.lx[3 * m + 1], z = P.lx[3 * m + 2];
    sm[0] += fx;
    sm[1] += fy;
    sm[2] += fz;
    sm[3] += y * fz - z * fy;
    sm[4] += z * fx - x * fz;
    sm[5] += x * fy - y * fx;
  }
  for (int k = 0; k < 6; ++k) {
    for (int o = 16; o > 0; o >>= 1) sm[k] += __shfl_xor_sync(0xffffffffu, sm[k], o);
    if (lane == 0) s_sum[k][wid] = sm[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double A[3], B[3];
    for (int k = 0; k < 3; ++k) {
      A[k] = 0.0;
      B[k] = 0.0;
      for (int w = 0; w < kRigidThreads / 32; ++w) {
        A[k] += s_sum[k][w];
        B[k] += s_sum[k + 3][w];
      }
    }
    const R mass = p_mass;
    const R buoy = (R)(1.0 - (double)p_rou / (double)a.rouf) * mass;
    double c[3];
    for (int k = 0; k < 3; ++k) {
      const R cf = (R)(-A[k]) + (k == 0 ? buoy * (R)a.gl : R(0));
      P.cF[3 * pi + k] = cf;
      const R cu = p_cu[k] + cf / mass * (R)a.dt;
      P.cu[3 * pi + k] = cu;
      const R cx = p_cx[k] + cu * (R)a.dt;
      P.cx[3 * pi + k] = cx;
      s_cx[k] = cx;
      c[k] = (double)cx;
    }
    const double T[3] = {B[0] - (c[1] * A[2] - c[2] * A[1]), B[1] - (c[2] * A[0] - c[0] * A[2]),
                         B[2] - (c[0] * A[1] - c[1] * A[0])};
    for (int k = 0; k < 3; ++k) {
      const R ct = -(R)T[k];
      P.cT[3 * pi + k] = ct;
      const R cw = p_cw[k] + R(0.1) * ct * (R)a.dt / p_in[k];
      P.cw[3 * pi + k] = cw;
      if (s_ang != nullptr) {
        // shared, so that no thread reads the rotation vector after it is
        // overwritten
        const R ang = p_ang[k] + cw;
        s_ang[k] = ang;
        P.angle[3 * pi + k] = ang;
      }
    }
  }
  __syncthreads();
}

template <typename R>
__global__ void __launch_bounds__(kRigidThreads) k_rigid(const RigidArgs a) {
  const PView<R> P = pview<R>(a.p);
  const int pi = blockIdx.x;
  const int m0 = P.offset[pi], m1 = P.offset[pi + 1];
  __shared__ R s_v[6][kRigidThreads / 32];
  __shared__ int s_i[6][kRigidThreads / 32];
  __shared__ int s_ext[6];
  __shared__ double s_sum[6][kRigidThreads / 32];
  __shared__ R s_cx[3];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;

  // -- extreme markers: argmin x,y,z then argmax x,y,z (first index on ties)
  R v[6];
  int id[6];
  for (int k = 0; k < 3; ++k) {
    v[k] = R(INFINITY);
    v[k + 3] = -R(INFINITY);
    id[k] = id[k + 3] = 0x7fffffff;
  }
  for (int m = m0 + threadIdx.x; m < m1; m += kRigidThreads) {
    for (int k = 0; k < 3; ++k) {
      const R c = P.lx[3 * m + k];
      argext_merge(v[k], id[k], c, m, true);
      argext_merge(v[k + 3], id[k + 3], c, m, false);
    }
  }
  for (int k = 0; k < 6; ++k) {
    for (int o = 16; o > 0; o >>= 1) {
      const R v2 = __shfl_xor_sync(0xffffffffu, v[k], o);
      const int i2 = __shfl_xor_sync(0xffffffffu, id[k], o);
      argext_merge(v[k], id[k], v2, i2, k < 3);
    }
    if (lane == 0) {
      s_v[k][wid] = v[k];
      s_i[k][wid] = id[k];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && (a.what & RIGID_WALL)) {
    for (int k = 0; k < 6; ++k) {
      R bv = s_v[k][0];
      int bi = s_i[k][0];
      for (int w = 1; w < kRigidThreads / 32; ++w) argext_merge(bv, bi, s_v[k][w], s_i[k][w], k < 3);
      s_ext[k] = bi;
    }
    bool valid = m1 > m0;
    for (int k = 0; k < 6; ++k) valid = valid && s_ext[k] >= m0 && s_ext[k] < m1;
    if (valid) {  // (non-finite positions leave no extreme marker: no spring)
      // spring force k0 (1 - |x - wall| / (2 dx)), clamped at 0; the indexed
      // += of the reference reads all six old values and the last write wins
      const R k0 = R(300);
      R d[6], dmax = R(0);
      for (int k = 0; k < 6; ++k) {
        const R c = P.lx[3 * s_ext[k] + (k % 3)];
        const R b = k < 3 ? R(0) : (R)a.size[k - 3];
        d[k] = fmax(k0 * (R(1) - fabs(c - b) / (R(2) * (R)a.dx)), R(0));
        dmax = fmax(dmax, d[k]);
      }
      if (dmax != R(0)) {
        R nv[6][3];
        for (int k = 0; k < 6; ++k)
          for (int c = 0; c < 3; ++c) {
            const R nrm = (c == k % 3) ? (k < 3 ? R(1) : R(-1)) : R(0);
            nv[k][c] = P.lF[3 * s_ext[k] + c] + nrm * d[k];
          }
        for (int k = 0; k < 6; ++k)
          for (int c = 0; c < 3; ++c) P.lF[3 * s_ext[k] + c] = nv[k][c];
      }
    }
  }
  __syncthreads();
  if (!(a.what & RIGID_UPDATE)) return;
  rigid_update_block<R>(a, P, pi, m0, m1, s_sum, s_cx, nullptr);
}

// ---------------------------------------------------------------------------
// Spreading (lbm/lbm3d.py:102-119)
// ---------------------------------------------------------------------------
// Clear the chunks written last time this buffer was used.  Each lane reads
// the flag of one chunk; the warp then clears its flagged chunks together
// (3 floats per lane per chunk), so a mostly flagged small lattice costs no
// more than a sparse large one.
template <typename R>
__global__ void k_spread_clear(long long n, R *field, uint8_t *chunks) {
  chain_enter();
  clear_flagged_chunks<R>((long long)blockIdx.x * blockDim.x + threadIdx.x, n, field, chunks);
}

struct SpreadArgs {
  Geom g;
  lbm_particles p;
  void *field;   // [n][3] in the arithmetic type of the particles
  uint8_t *chunks;
  int *owner;
};

// pass 0: flag chunks and claim nodes (max marker index = last in loop order)
// pass 1: the owning marker writes w lF lm (reference mode) and releases its
//         claim: a thread of another marker that reads the node's claim after
//         the release sees -1, which is not its index either, so it still
//         leaves the node to the owner, and the claim array holds -1 again
//         when the pass ends
// pass 3: accumulate w lF lm (accumulate mode; flags set as in pass 0)
// pass 4: pass 1 after claims made by ibm_interpolate_wall_claim -- the owner
//         also flags the chunk (every claimed node has exactly one owner, so
//         the flagged chunks are pass 0's)
template <int PASS, typename R>
__global__ void __launch_bounds__(kIbmThreads) k_spread(const SpreadArgs a) {
  chain_enter();
  __shared__ R sh[1][kMarkersPerBlock * 2];
  const PView<R> P = pview<R>(a.p);
  R *field = static_cast<R *>(a.field);
  const int mk = threadIdx.x / kStencil, slot = threadIdx.x % kStencil;
  const int m = blockIdx.x * kMarkersPerBlock + mk;
  const bool live = m < a.p.n_markers;
  R l[3] = {R(0), R(0), R(0)};
  int x = 0, y = 0, z = 0;
  R w = R(0);
  bool in_box = false;
  if (live) {
    l[0] = P.lx[3 * m];
    l[1] = P.lx[3 * m + 1];
    l[2] = P.lx[3 * m + 2];
    in_box = stencil_slot(a.g, l, slot, x, y, z, w);
  }
  const long long idx = ((long long)x * a.g.ny + y) * a.g.nz + z;
  if (in_box && !lbm_in(idx >= 0 && idx < a.g.n)) in_box = false;
  if (PASS == 0) {
    if (!in_box) return;
    a.chunks[idx >> 5] = 1;
    atomicMax(a.owner + idx, m);
    return;
  }
  // passes 1 and 3 need the normalised weight: sum over the marker's stencil
  R W[1] = {in_box ? w : R(0)};
  stencil_sum<1>(W, sh, slot, mk);
  if (!in_box) return;
  const R wn = W[0] > R(0) ? w / W[0] : w;
  const R lm = P.lm[m];
  if (PASS == 1 || PASS == 4) {
    if (a.owner[idx] != m) return;
    a.owner[idx] = -1;
    if (PASS == 4) a.chunks[idx >> 5] = 1;
    for (int k = 0; k < 3; ++k) field[3 * idx + k] = (wn * P.lF[3 * m + k]) * lm;
  } else {
    a.chunks[idx >> 5] = 1;
    for (int k = 0; k < 3; ++k) atomicAdd(field + 3 * idx + k, (wn * P.lF[3 * m + k]) * lm);
  }
}

// ---------------------------------------------------------------------------
// Tiled spreading: the lattice is cut into 8 x 8 x 8-node tiles.  k_spread_bin
// (thread = marker x stencil slot, as k_spread) takes each marker's
// normalising weight sum and lists the marker under every tile its stencil
// box touches (at most 8).  k_spread_tile (block = tile) then resolves the
// tile entirely in shared memory: reference mode takes the last writer of
// every node (largest marker index, the reference's loop order) with
// shared-memory atomicMax and writes each claimed node once; accumulate mode
// sums the contributions in shared memory and stores each node once.  No
// global atomics touch the field, and no global claim array is needed.
// ---------------------------------------------------------------------------
constexpr int kTile = 8;
constexpr int kTileNodes = kTile * kTile * kTile;
constexpr int kTileCap = 512;      // markers listed per tile; more: the tile scans all markers

struct TileArgs {
  Geom g;
  lbm_particles p;
  void *field;        // [n][3] in the particles' arithmetic type
  uint8_t *chunks;
  int *tile_count;    // [ntiles], zero between calls
  int *tile_list;     // [ntiles][kTileCap]
  void *wsum;         // [n_markers] normalising weight sums
  int tx, ty, tz;     // tiles per axis
};

template <typename R>
__global__ void __launch_bounds__(kIbmThreads) k_spread_bin(const TileArgs a) {
  __shared__ R sh[1][kMarkersPerBlock * 2];
  const PView<R> P = pview<R>(a.p);
  const int mk = threadIdx.x / kStencil, slot = threadIdx.x % kStencil;
  const int m = blockIdx.x * kMarkersPerBlock + mk;
  const bool live = m < a.p.n_markers;
  R l[3] = {R(0), R(0), R(0)};
  int x = 0, y = 0, z = 0;
  R w = R(0);
  bool in_box = false;
  if (live) {
    l[0] = P.lx[3 * m];
    l[1] = P.lx[3 * m + 1];
    l[2] = P.lx[3 * m + 2];
    in_box = stencil_slot(a.g, l, slot, x, y, z, w);
  }
  R W[1] = {in_box ? w : R(0)};
  stencil_sum<1>(W, sh, slot, mk);
  if (!live || slot != 0) return;
  static_cast<R *>(a.wsum)[m] = W[0];
  int lo[3], hi[3];
  box_axis(l[0], a.g.nx - 1, lo[0], hi[0]);
  box_axis(l[1], a.g.ny - 1, lo[1], hi[1]);
  box_axis(l[2], a.g.nz - 1, lo[2], hi[2]);
  if (hi[0] <= lo[0] || hi[1] <= lo[1] || hi[2] <= lo[2]) return;
  for (int i = lo[0] / kTile; i <= (hi[0] - 1) / kTile; ++i)
    for (int j = lo[1] / kTile; j <= (hi[1] - 1) / kTile; ++j)
      for (int k = lo[2] / kTile; k <= (hi[2] - 1) / kTile; ++k) {
        const int t = (i * a.ty + j) * a.tz + k;
        if (!lbm_in(t >= 0 && t < a.tx * a.ty * a.tz)) continue;
        const int pos = atomicAdd(a.tile_count + t, 1);
        if (pos < kTileCap) a.tile_list[(long long)t * kTileCap + pos] = m;
      }
}

template <typename R, int MODE>
__global__ void __launch_bounds__(kTileNodes) k_spread_tile(const TileArgs a) {
  __shared__ int s_owner[kTileNodes];
  __shared__ R s_acc[MODE == 1 ? kTileNodes * 3 : 1];
  const int t = blockIdx.x;
  const int cnt = a.tile_count[t];
  if (cnt == 0) return;
  const PView<R> P = pview<R>(a.p);
  const R *wsum = static_cast<const R *>(a.wsum);
  R *field = static_cast<R *>(a.field);
  const int ti = t / (a.ty * a.tz), tj = (t / a.tz) % a.ty, tk = t % a.tz;
  const int ox = ti * kTile, oy = tj * kTile, oz = tk * kTile;
  const int tid = threadIdx.x;
  s_owner[tid] = -1;
  if constexpr (MODE == 1) {
    s_acc[3 * tid] = R(0);
    s_acc[3 * tid + 1] = R(0);
    s_acc[3 * tid + 2] = R(0);
  }
  __syncthreads();
  const bool all = cnt > kTileCap;   // list overflowed: scan every marker
  const long long pairs = (long long)(all ? a.p.n_markers : cnt) * kStencil;
  for (long long pr = tid; pr < pairs; pr += kTileNodes) {
    const int li = (int)(pr / kStencil), slot = (int)(pr % kStencil);
    const int m = all ? li : a.tile_list[(long long)t * kTileCap + li];
    const R l[3] = {P.lx[3 * m], P.lx[3 * m + 1], P.lx[3 * m + 2]};
    int x, y, z;
    R w;
    if (!stencil_slot(a.g, l, slot, x, y, z, w)) continue;
    const int dx = x - ox, dy = y - oy, dz = z - oz;
    if (dx < 0 || dx >= kTile || dy < 0 || dy >= kTile || dz < 0 || dz >= kTile) continue;
    const int local = (dx * kTile + dy) * kTile + dz;
    if constexpr (MODE == 0) {
      atomicMax(s_owner + local, m);
    } else {
      const R W = wsum[m];
      const R wn = W > R(0) ? w / W : w;
      const R lm = P.lm[m];
      for (int k = 0; k < 3; ++k) atomicAdd(s_acc + 3 * local + k, (wn * P.lF[3 * m + k]) * lm);
      s_owner[local] = 0;   // touched
    }
  }
  __syncthreads();
  const int x = ox + tid / (kTile * kTile), y = oy + (tid / kTile) % kTile, z = oz + tid % kTile;
  const int m = s_owner[tid];
  if (m >= 0 && lbm_in(x < a.g.nx && y < a.g.ny && z < a.g.nz)) {
    const long long idx = ((long long)x * a.g.ny + y) * a.g.nz + z;
    a.chunks[idx >> 5] = 1;
    if constexpr (MODE == 0) {
      // the winner's weight at this node: its stencil slot of (x, y, z)
      const R l[3] = {P.lx[3 * m], P.lx[3 * m + 1], P.lx[3 * m + 2]};
      int lo[3], hi[3];
      box_axis(l[0], a.g.nx - 1, lo[0], hi[0]);
      box_axis(l[1], a.g.ny - 1, lo[1], hi[1]);
      box_axis(l[2], a.g.nz - 1, lo[2], hi[2]);
      const int slot = ((x - lo[0]) * 4 + (y - lo[1])) * 4 + (z - lo[2]);
      int xs, ys, zs;
      R w;
      stencil_slot(a.g, l, slot, xs, ys, zs, w);
      const R W = wsum[m];
      const R wn = W > R(0) ? w / W : w;
      const R lm = P.lm[m];
      for (int k = 0; k < 3; ++k) field[3 * idx + k] = (wn * P.lF[3 * m + k]) * lm;
    } else {
      for (int k = 0; k < 3; ++k) field[3 * idx + k] = s_acc[3 * tid + k];
    }
  }
  __syncthreads();
  if (tid == 0) a.tile_count[t] = 0;    // ready for the next call
}

static void tile_dims(const Geom &g, int &tx, int &ty, int &tz) {
  tx = (g.nx + kTile - 1) / kTile;
  ty = (g.ny + kTile - 1) / kTile;
  tz = (g.nz + kTile - 1) / kTile;
}

// ---------------------------------------------------------------------------
// Marker update (particle/base/base.py:153-156, particle/coord.py:87-108):
// angle += cw; R from the rotation vector (float64, through the unit
// quaternion); lx = float32(R X0) + cx.  One block per particle.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(kRigidThreads) k_markers(const lbm_particles pt) {
  const PView<R> p = pview<R>(pt);
  const int pi = blockIdx.x;
  const int m0 = p.offset[pi], m1 = p.offset[pi + 1];
  // the first marker of this thread is loaded before the rotation is built,
  // so the load latency overlaps it
  int m = m0 + (int)threadIdx.x;
  double X = 0.0, Y = 0.0, Z = 0.0;
  if (m < m1) {
    X = p.lagrange[3 * m];
    Y = p.lagrange[3 * m + 1];
    Z = p.lagrange[3 * m + 2];
  }
  // every thread builds the same rotation (no shared-memory broadcast)
  double v[3];
  R ang[3], c[3];
  for (int k = 0; k < 3; ++k) {
    ang[k] = p.angle[3 * pi + k] + p.cw[3 * pi + k];
    v[k] = ang[k];
    c[k] = p.cx[3 * pi + k];
  }
  const double th = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  double s;
  if (th <= 1e-3) {
    const double t2 = th * th;
    s = 0.5 - t2 / 48.0 + t2 * t2 / 3840.0;
  } else {
    s = sin(0.5 * th) / th;
  }
  double x = s * v[0], y = s * v[1], z = s * v[2], w = cos(0.5 * th);
  const double nq = sqrt(x * x + y * y + z * z + w * w);
  x /= nq;
  y /= nq;
  z /= nq;
  w /= nq;
  const double M[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - z * w),     2 * (x * z + y * w),
                       2 * (x * y + z * w),     1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                       2 * (x * z - y * w),     2 * (y * z + x * w),     1 - 2 * (x * x + y * y)};
  for (; m < m1; m += kRigidThreads) {
    for (int k = 0; k < 3; ++k) {
      const double r = M[3 * k] * X + M[3 * k + 1] * Y + M[3 * k + 2] * Z;
      p.lx[3 * m + k] = (R)r + c[k];
    }
    const int mn = m + kRigidThreads;
    if (mn < m1) {
      X = p.lagrange[3 * mn];
      Y = p.lagrange[3 * mn + 1];
      Z = p.lagrange[3 * mn + 2];
    }
  }
  __syncthreads();   // every thread has read the old angle
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) p.angle[3 * pi + k] = ang[k];
}

// ---------------------------------------------------------------------------
// The six extreme markers of one particle (block per particle, kRigidThreads
// threads): argmin x, y, z then argmax x, y, z of lx, first index on ties --
// the markers LBMD3.particle_to_wall acts on (lbm/lbm3d.py:121-167).
// Thread 0 receives them in ext.
// ---------------------------------------------------------------------------
// Block-wide argmin / argmax (first index on ties) of the per-thread
// candidates v / id (argmin x, y, z then argmax x, y, z); thread 0 gets ext.
template <typename R>
__device__ __forceinline__ void extremes_reduce(R v[6], int id[6], R (*s_v)[kRigidThreads / 32],
                                                int (*s_i)[kRigidThreads / 32], int ext[6]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int k = 0; k < 6; ++k) {
    for (int o = 16; o > 0; o >>= 1) {
      const R v2 = __shfl_xor_sync(0xffffffffu, v[k], o);
      const int i2 = __shfl_xor_sync(0xffffffffu, id[k], o);
      argext_merge(v[k], id[k], v2, i2, k < 3);
    }
    if (lane == 0) {
      s_v[k][wid] = v[k];
      s_i[k][wid] = id[k];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < 6; ++k) {
      R bv = s_v[k][0];
      int bi = s_i[k][0];
      for (int w = 1; w < kRigidThreads / 32; ++w) argext_merge(bv, bi, s_v[k][w], s_i[k][w], k < 3);
      ext[k] = bi;
    }
  }
  __syncthreads();
}

// The six extreme markers of particle markers m0..m1 (one block).
template <typename R>
__device__ __forceinline__ void block_extremes(const PView<R> &P, int m0, int m1,
                                               R (*s_v)[kRigidThreads / 32],
                                               int (*s_i)[kRigidThreads / 32], int ext[6]) {
  R v[6];
  int id[6];
  for (int k = 0; k < 3; ++k) {
    v[k] = R(INFINITY);
    v[k + 3] = -R(INFINITY);
    id[k] = id[k + 3] = 0x7fffffff;
  }
  for (int m = m0 + threadIdx.x; m < m1; m += kRigidThreads) {
    for (int k = 0; k < 3; ++k) {
      const R c = P.lx[3 * m + k];
      argext_merge(v[k], id[k], c, m, true);
      argext_merge(v[k + 3], id[k + 3], c, m, false);
    }
  }
  extremes_reduce<R>(v, id, s_v, s_i, ext);
}

template <typename R>
__global__ void __launch_bounds__(kRigidThreads) k_extremes(const lbm_particles pt) {
  const PView<R> P = pview<R>(pt);
  const int pi = blockIdx.x;
  __shared__ R s_v[6][kRigidThreads / 32];
  __shared__ int s_i[6][kRigidThreads / 32];
  int ext[6];
  block_extremes<R>(P, P.offset[pi], P.offset[pi + 1], s_v, s_i, ext);
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; ++k) pt.extreme[6 * pi + k] = ext[k];
}

// Rigid update + marker transform + extremes of the new positions, one block
// per particle: rigid_update_block (as k_rigid's RIGID_UPDATE), then
// k_markers' rotation with the extreme markers of the new positions found
// in the same pass -- the same arithmetic and order, so the same results.
template <typename R>
__global__ void __launch_bounds__(kRigidThreads) k_rigid_step(const RigidArgs a) {
  chain_enter();
  const PView<R> P = pview<R>(a.p);
  const int pi = blockIdx.x;
  const int m0 = P.offset[pi], m1 = P.offset[pi + 1];
  __shared__ double s_sum[6][kRigidThreads / 32];
  __shared__ R s_cx[3], s_ang[3];
  __shared__ R s_v[6][kRigidThreads / 32];
  __shared__ int s_i[6][kRigidThreads / 32];
  // the body-frame coordinates of this thread's first marker are loaded
  // before the update, so their latency overlaps it (nothing writes them)
  int m = m0 + (int)threadIdx.x;
  double X = 0.0, Y = 0.0, Z = 0.0;
  if (m < m1) {
    X = P.lagrange[3 * m];
    Y = P.lagrange[3 * m + 1];
    Z = P.lagrange[3 * m + 2];
  }
  rigid_update_block<R>(a, P, pi, m0, m1, s_sum, s_cx, s_ang);
  // (every thread has read lx for the sums; cw and angle are final)

  // -- lx = R(angle) X0 + cx   (particle/coord.py:87-108)
  double v[3];
  R c[3];
  for (int k = 0; k < 3; ++k) {
    v[k] = s_ang[k];
    c[k] = s_cx[k];
  }
  const double th = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  double sc;
  if (th <= 1e-3) {
    const double t2 = th * th;
    sc = 0.5 - t2 / 48.0 + t2 * t2 / 3840.0;
  } else {
    sc = sin(0.5 * th) / th;
  }
  double x = sc * v[0], y = sc * v[1], z = sc * v[2], w = cos(0.5 * th);
  const double nq = sqrt(x * x + y * y + z * z + w * w);
  x /= nq;
  y /= nq;
  z /= nq;
  w /= nq;
  const double M[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - z * w),     2 * (x * z + y * w),
                       2 * (x * y + z * w),     1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                       2 * (x * z - y * w),     2 * (y * z + x * w),     1 - 2 * (x * x + y * y)};
  const bool ext_on = a.p.extreme != nullptr;
  R ev[6];
  int eid[6];
  for (int k = 0; k < 3; ++k) {
    ev[k] = R(INFINITY);
    ev[k + 3] = -R(INFINITY);
    eid[k] = eid[k + 3] = 0x7fffffff;
  }
  for (; m < m1; m += kRigidThreads) {
    // the next marker's coordinates are loaded before this one's stores
    const int mn = m + kRigidThreads;
    double Xn = 0.0, Yn = 0.0, Zn = 0.0;
    if (mn < m1) {
      Xn = P.lagrange[3 * mn];
      Yn = P.lagrange[3 * mn + 1];
      Zn = P.lagrange[3 * mn + 2];
    }
    for (int k = 0; k < 3; ++k) {
      const double r = M[3 * k] * X + M[3 * k + 1] * Y + M[3 * k + 2] * Z;
      const R nx = (R)r + c[k];
      P.lx[3 * m + k] = nx;
      argext_merge(ev[k], eid[k], nx, m, true);
      argext_merge(ev[k + 3], eid[k + 3], nx, m, false);
    }
    X = Xn;
    Y = Yn;
    Z = Zn;
  }
  if (!ext_on) return;
  int ext[6];
  extremes_reduce<R>(ev, eid, s_v, s_i, ext);
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; ++k) a.p.extreme[6 * pi + k] = ext[k];
}

template <int Q>
struct RunInterp {
  static int run(InterpArgs a, int storage, cudaStream_t s) {
    const unsigned nb = (unsigned)((a.p.n_markers + kMarkersPerBlock - 1) / kMarkersPerBlock);
    a.interp_blocks = nb;
    // (clearing blocks after the interpolation's: one thread per 32-node chunk)
    const unsigned grid =
        nb + (a.clear_chunks != nullptr ? blocks_for((a.g.n + 31) >> 5, kIbmThreads) : 0u);
    switch (storage) {
      case LBM_STORAGE_FP32: launch_chained(k_interp<Q, LBM_STORAGE_FP32>, grid, kIbmThreads, 0, s, a); break;
      case LBM_STORAGE_FP16S: launch_chained(k_interp<Q, LBM_STORAGE_FP16S>, grid, kIbmThreads, 0, s, a); break;
      case LBM_STORAGE_FP64: launch_chained(k_interp<Q, LBM_STORAGE_FP64>, grid, kIbmThreads, 0, s, a); break;
      default: launch_chained(k_interp<Q, LBM_STORAGE_BF16S>, grid, kIbmThreads, 0, s, a); break;
    }
    LBM_LAUNCH_CHECK("ibm_interpolate");
    return LBM_OK;
  }
};

static int check_particles(const lbm_particles *pt, const char *who) {
  if (pt == nullptr || pt->n_particles < 0 || pt->n_markers < 0 ||
      (pt->fp64 != 0 && pt->fp64 != 1)) {
    set_error("%s: bad particle description", who);
    return LBM_ERR_INVALID;
  }
  return LBM_OK;
}

// particle arrays must be float64 exactly when the lattice stores FP64
static int check_precision(const lbm_lattice *lat, const lbm_particles *pt, const char *who) {
  const bool any = pt->n_particles > 0 || pt->n_markers > 0;
  if (any && (lat->storage == LBM_STORAGE_FP64) != (pt->fp64 == 1)) {
    set_error("%s: particles of an FP64 lattice are float64 (fp64 = 1), otherwise float32", who);
    return LBM_ERR_INVALID;
  }
  return LBM_OK;
}

// spreading launches (clear, then the claim pass and the write pass that
// releases the claims, or the accumulation) in the particles' arithmetic type
template <typename R>
static int spread_launch(const SpreadArgs &a, int mode, long long n_markers, cudaStream_t s,
                         const char *who) {
  const long long nchunks = (a.g.n + 31) >> 5;
  launch_chained(k_spread_clear<R>, blocks_for(nchunks, 256), 256, 0, s, a.g.n, static_cast<R *>(a.field),
                                                             a.chunks);
  LBM_LAUNCH_CHECK(who);
  if (n_markers == 0) return LBM_OK;
  const unsigned nb = (unsigned)((n_markers + kMarkersPerBlock - 1) / kMarkersPerBlock);
  if (mode == 0) {
    launch_chained(k_spread<0, R>, nb, kIbmThreads, 0, s, a);
    launch_chained(k_spread<1, R>, nb, kIbmThreads, 0, s, a);
  } else {
    launch_chained(k_spread<3, R>, nb, kIbmThreads, 0, s, a);
  }
  LBM_LAUNCH_CHECK(who);
  return LBM_OK;
}

// ---------------------------------------------------------------------------
// Claim array of ibm_spread_noalloc.  It lives in the library's own device
// memory (one copy per GPU that loads the library, kept until exit), so
// that entry point needs no buffer from the caller and allocates nothing.
// Host code must not use the symbol itself -- only the device address that
// cudaGetSymbolAddress returns for the current device.
// ---------------------------------------------------------------------------
static __device__ __align__(256) int32_t g_spread_owner[LBM_SPREAD_NOALLOC_MAX_NODES];

__global__ void k_owner_reset(int32_t *owner, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    owner[i] = -1;
}

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_owner_mu;
int32_t *g_owner_addr[kMaxDevices] = {};
// whether the array on a device holds -1 everywhere between calls: false
// until the first reference-mode call resets it (__device__ memory starts at
// 0), and again after a call whose launches failed part-way
bool g_owner_clean[kMaxDevices] = {};
}  // namespace

// Device address of g_spread_owner on the current device, looked up once per
// device (the first call on a device does this set-up), and whether the
// array still needs its one-time reset to -1.  The cached address belongs to
// the device's current primary context: after cudaDeviceReset it is stale.
static int owner_scratch(int32_t **out, int *dev_out, bool *clean) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_cuda(e, "ibm_spread_noalloc");
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("ibm_spread_noalloc: device index %d out of range", dev);
    return LBM_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_owner_mu);
  if (g_owner_addr[dev] == nullptr) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_spread_owner);
    if (e != cudaSuccess) return fail_cuda(e, "ibm_spread_noalloc: cudaGetSymbolAddress");
    g_owner_addr[dev] = static_cast<int32_t *>(p);
  }
  *out = g_owner_addr[dev];
  *dev_out = dev;
  *clean = g_owner_clean[dev];
  return LBM_OK;
}

static void owner_mark(int dev, bool clean) {
  std::lock_guard<std::mutex> lock(g_owner_mu);
  g_owner_clean[dev] = clean;
}

}  // namespace lbm

using namespace lbm;

extern "C" {

int ibm_interpolate(const lbm_lattice *lat, const void *fa, const lbm_force *force,
                    const float *face_rho_in, const float *u_field, const float *rho_field,
                    const lbm_particles *pt, float dt, int32_t step, uint32_t *status,
                    void *stream) {
  int rc = check_lattice(lat);
  if (rc) return rc;
  if ((rc = check_particles(pt, "ibm_interpolate"))) return rc;
  if (!(dt > 0.f)) {
    set_error("ibm_interpolate: dt must be positive");
    return LBM_ERR_INVALID;
  }
  if (fa == nullptr && (u_field == nullptr || rho_field == nullptr)) {
    set_error("ibm_interpolate: needs populations or the u / rho fields");
    return LBM_ERR_INVALID;
  }
  if (fa != nullptr && any_face(lat, LBM_BC_NON_EQUILIBRIUM)) {
    set_error("ibm_interpolate: NON_EQUILIBRIUM faces need the u / rho fields");
    return LBM_ERR_UNSUPPORTED;
  }
  if (fa != nullptr && any_face(lat, LBM_BC_WALL_WITH_SPEED) && face_rho_in == nullptr) {
    set_error("ibm_interpolate: WALL_WITH_SPEED faces need face_rho_in");
    return LBM_ERR_INVALID;
  }
  if ((rc = check_precision(lat, pt, "ibm_interpolate"))) return rc;
  if (pt->n_markers == 0) return LBM_OK;
  InterpArgs a;
  memset(&a, 0, sizeof(a));
  a.g = make_geom(lat);
  a.fa = fa;
  if (fa != nullptr) fill_step_planes(a.g, lat->q, lat->storage, fa, nullptr, a.planes);
  a.u_field = u_field;
  a.rho_field = rho_field;
  if (force != nullptr) {
    for (int k = 0; k < 3; ++k) a.go[k] = force->old_uniform[k];
    a.fol_old = force->old_field;
  }
  a.face_rho_in = face_rho_in;
  a.p = *pt;
  a.dt = dt;
  a.step = step;
  a.status = status;
  switch (lat->q) {
    case 13: return RunInterp<13>::run(a, lat->storage, (cudaStream_t)stream);
    case 15: return RunInterp<15>::run(a, lat->storage, (cudaStream_t)stream);
    case 19: return RunInterp<19>::run(a, lat->storage, (cudaStream_t)stream);
    default: return RunInterp<27>::run(a, lat->storage, (cudaStream_t)stream);
  }
}

int rigid_wall_and_update(const lbm_lattice *lat, const lbm_particles *pt, int32_t what, float dt,
                          float dx, float gl, float rouf, void *stream) {
  int rc = LBM_OK;
  if ((what & RIGID_WALL) && (rc = check_lattice(lat))) return rc;
  if ((rc = check_particles(pt, "rigid_wall_and_update"))) return rc;
  if (!(dt > 0.f)) {
    set_error("Time step must be positive");
    return LBM_ERR_INVALID;
  }
  if (!(rouf > 0.f)) {
    set_error("Fluid density must be positive");
    return LBM_ERR_INVALID;
  }
  if (pt->n_particles == 0) return LBM_OK;
  if (what < 1 || what > 3) {
    set_error("rigid_wall_and_update: what must be RIGID_WALL, RIGID_UPDATE or both");
    return LBM_ERR_INVALID;
  }
  RigidArgs a;
  a.p = *pt;
  a.what = what;
  for (int k = 0; k < 3; ++k) a.size[k] = 0.f;
  if (lat != nullptr) {
    a.size[0] = (float)(lat->nx - 1);
    a.size[1] = (float)(lat->ny - 1);
    a.size[2] = (float)(lat->nz - 1);
  }
  a.dt = dt;
  a.dx = dx;
  a.gl = gl;
  a.rouf = rouf;
  if (pt->fp64)
    k_rigid<double><<<pt->n_particles, kRigidThreads, 0, (cudaStream_t)stream>>>(a);
  else
    k_rigid<float><<<pt->n_particles, kRigidThreads, 0, (cudaStream_t)stream>>>(a);
  LBM_LAUNCH_CHECK("rigid_wall_and_update");
  return LBM_OK;
}

int ibm_spread(const lbm_lattice *lat, const lbm_particles *pt, int32_t mode, float *field,
               uint8_t *chunks, int32_t *owner, void *stream) {
  int rc = check_lattice(lat);
  if (rc) return rc;
  if ((rc = check_particles(pt, "ibm_spread"))) return rc;
  if (mode != 0 && mode != 1) {
    set_error("ibm_spread: mode must be 0 (reference) or 1 (accumulate)");
    return LBM_ERR_INVALID;
  }
  if (field == nullptr || chunks == nullptr || (mode == 0 && owner == nullptr)) {
    set_error("ibm_spread: field, chunks (and owner in reference mode) are required");
    return LBM_ERR_INVALID;
  }
  if ((rc = check_precision(lat, pt, "ibm_spread"))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  SpreadArgs a;
  a.g = make_geom(lat);
  a.p = *pt;
  a.field = field;
  a.chunks = chunks;
  a.owner = owner;
  return lat->storage == LBM_STORAGE_FP64
             ? spread_launch<double>(a, mode, pt->n_markers, s, "ibm_spread")
             : spread_launch<float>(a, mode, pt->n_markers, s, "ibm_spread");
}

}  // extern "C"

namespace lbm {
// ibm_interpolate_wall, and with field / chunks / owner set
// ibm_interpolate_wall_claim (the claims and the chunk clearing of reference-
// mode spreading in the same launch).
static int interp_wall(const lbm_lattice *lat, const void *fa, const lbm_force *force,
                       const float *face_rho_in, const lbm_particles *pt, float dt, float dx,
                       int32_t step, uint32_t *status, float *field, uint8_t *chunks,
                       int32_t *owner, void *stream, const char *who) {
  int rc = check_lattice(lat);
  if (rc) return rc;
  if ((rc = check_particles(pt, who))) return rc;
  if (!(dt > 0.f)) {
    set_error("%s: dt must be positive", who);
    return LBM_ERR_INVALID;
  }
  if (fa == nullptr) {
    set_error("%s: needs the post-collision populations", who);
    return LBM_ERR_INVALID;
  }
  if (any_face(lat, LBM_BC_NON_EQUILIBRIUM)) {
    set_error("%s: NON_EQUILIBRIUM faces need the u / rho fields", who);
    return LBM_ERR_UNSUPPORTED;
  }
  if (any_face(lat, LBM_BC_WALL_WITH_SPEED) && face_rho_in == nullptr) {
    set_error("%s: WALL_WITH_SPEED faces need face_rho_in", who);
    return LBM_ERR_INVALID;
  }
  const bool claim = chunks != nullptr;
  if (claim && (field == nullptr || owner == nullptr)) {
    set_error("%s: field, chunks and owner are required", who);
    return LBM_ERR_INVALID;
  }
  if ((rc = check_precision(lat, pt, who))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (pt->n_markers == 0) {
    if (!claim) return LBM_OK;
    // nothing to interpolate or claim: only the clearing
    const unsigned nb = blocks_for((make_geom(lat).n + 31) >> 5, 256);
    if (lat->storage == LBM_STORAGE_FP64)
      launch_chained(k_spread_clear<double>, nb, 256, 0, s, make_geom(lat).n, (double *)field, chunks);
    else
      launch_chained(k_spread_clear<float>, nb, 256, 0, s, make_geom(lat).n, field, chunks);
    LBM_LAUNCH_CHECK(who);
    return LBM_OK;
  }
  if (pt->extreme == nullptr) {
    set_error("%s: the particles' extreme markers are required", who);
    return LBM_ERR_INVALID;
  }
  InterpArgs a;
  memset(&a, 0, sizeof(a));
  a.g = make_geom(lat);
  a.fa = fa;
  fill_step_planes(a.g, lat->q, lat->storage, fa, nullptr, a.planes);
  if (force != nullptr) {
    for (int k = 0; k < 3; ++k) a.go[k] = force->old_uniform[k];
    a.fol_old = force->old_field;
  }
  a.face_rho_in = face_rho_in;
  a.p = *pt;
  a.dt = dt;
  a.step = step;
  a.status = status;
  a.wall = 1;
  a.size[0] = (float)(lat->nx - 1);
  a.size[1] = (float)(lat->ny - 1);
  a.size[2] = (float)(lat->nz - 1);
  a.dx = dx;
  if (claim) {
    a.claim_owner = owner;
    a.clear_field = field;
    a.clear_chunks = chunks;
  }
  switch (lat->q) {
    case 13: return RunInterp<13>::run(a, lat->storage, s);
    case 15: return RunInterp<15>::run(a, lat->storage, s);
    case 19: return RunInterp<19>::run(a, lat->storage, s);
    default: return RunInterp<27>::run(a, lat->storage, s);
  }
}
}  // namespace lbm

extern "C" {

int ibm_interpolate_wall(const lbm_lattice *lat, const void *fa, const lbm_force *force,
                         const float *face_rho_in, const lbm_particles *pt, float dt, float dx,
                         int32_t step, uint32_t *status, void *stream) {
  return interp_wall(lat, fa, force, face_rho_in, pt, dt, dx, step, status, nullptr, nullptr,
                     nullptr, stream, "ibm_interpolate_wall");
}

int ibm_interpolate_wall_claim(const lbm_lattice *lat, const void *fa, const lbm_force *force,
                               const float *face_rho_in, const lbm_particles *pt, float dt,
                               float dx, int32_t step, uint32_t *status, float *field,
                               uint8_t *chunks, int32_t *owner, void *stream) {
  if (chunks == nullptr) {
    set_error("ibm_interpolate_wall_claim: field, chunks and owner are required");
    return LBM_ERR_INVALID;
  }
  return interp_wall(lat, fa, force, face_rho_in, pt, dt, dx, step, status, field, chunks, owner,
                     stream, "ibm_interpolate_wall_claim");
}

int ibm_spread_claimed(const lbm_lattice *lat, const lbm_particles *pt, float *field,
                       uint8_t *chunks, int32_t *owner, void *stream) {
  int rc = check_lattice(lat);
  if (rc) return rc;
  if ((rc = check_particles(pt, "ibm_spread_claimed"))) return rc;
  if (field == nullptr || chunks == nullptr || owner == nullptr) {
    set_error("ibm_spread_claimed: field, chunks and owner are required");
    return LBM_ERR_INVALID;
  }
  if ((rc = check_precision(lat, pt, "ibm_spread_claimed"))) return rc;
  if (pt->n_markers == 0) return LBM_OK;
  cudaStream_t s = (cudaStream_t)stream;
  SpreadArgs a;
  a.g = make_geom(lat);
  a.p = *pt;
  a.field = field;
  a.chunks = chunks;
  a.owner = owner;
  const unsigned nb = (unsigned)((pt->n_markers + kMarkersPerBlock - 1) / kMarkersPerBlock);
  if (lat->storage == LBM_STORAGE_FP64)
    launch_chained(k_spread<4, double>, nb, kIbmThreads, 0, s, a);
  else
    launch_chained(k_spread<4, float>, nb, kIbmThreads, 0, s, a);
  LBM_LAUNCH_CHECK("ibm_spread_claimed");
  return LBM_OK;
}

int rigid_step(const lbm_particles *pt, float dt, float gl, float rouf, void *stream) {
  int rc = check_particles(pt, "rigid_step");
  if (rc) return rc;
  if (!(dt > 0.f)) {
    set_error("Time step must be positive");
    return LBM_ERR_INVALID;
  }
  if (!(rouf > 0.f)) {
    set_error("Fluid density must be positive");
    return LBM_ERR_INVALID;
  }
  if (pt->n_particles == 0) return LBM_OK;
  RigidArgs a;
  memset(&a, 0, sizeof(a));
  a.p = *pt;
  a.what = RIGID_UPDATE;
  a.dt = dt;
  a.dx = 1.f;
  a.gl = gl;
  a.rouf = rouf;
  if (pt->fp64)
    launch_chained(k_rigid_step<double>, pt->n_particles, kRigidThreads, 0, (cudaStream_t)stream, a);
  else
    launch_chained(k_rigid_step<float>, pt->n_particles, kRigidThreads, 0, (cudaStream_t)stream, a);
  LBM_LAUNCH_CHECK("rigid_step");
  return LBM_OK;
}

int rigid_extremes(const lbm_particles *pt, void *stream) {
  int rc = check_particles(pt, "rigid_extremes");
  if (rc) return rc;
  if (pt->n_particles == 0) return LBM_OK;
  if (pt->extreme == nullptr) {
    set_error("rigid_extremes: no output array (extreme)");
    return LBM_ERR_INVALID;
  }
  if (pt->fp64)
    k_extremes<double><<<pt->n_particles, kRigidThreads, 0, (cudaStream_t)stream>>>(*pt);
  else
    k_extremes<float><<<pt->n_particles, kRigidThreads, 0, (cudaStream_t)stream>>>(*pt);
  LBM_LAUNCH_CHECK("rigid_extremes");
  return LBM_OK;
}

size_t ibm_spread_tiled_scratch_bytes(const lbm_lattice *lat, int32_t n_markers) {
  if (lat == nullptr || n_markers < 0) return 0;
  const Geom g = make_geom(lat);
  int tx, ty, tz;
  tile_dims(g, tx, ty, tz);
  const size_t ntiles = (size_t)tx * ty * tz;
  const size_t real = lat->storage == LBM_STORAGE_FP64 ? 8 : 4;
  return ntiles * 4 + ntiles * kTileCap * 4 + (size_t)n_markers * real + 256;
}

int ibm_spread_tiled(const lbm_lattice *lat, const lbm_particles *pt, int32_t mode, float *field,
                     uint8_t *chunks, void *scratch, size_t scratch_bytes, void *stream) {
  int rc = check_lattice(lat);
  if (rc) return rc;
  if ((rc = check_particles(pt, "ibm_spread_tiled"))) return rc;
  if (mode != 0 && mode != 1) {
    set_error("ibm_spread_tiled: mode must be 0 (reference) or 1 (accumulate)");
    return LBM_ERR_INVALID;
  }
  if (field == nullptr || chunks == nullptr || scratch == nullptr) {
    set_error("ibm_spread_tiled: field, chunks and scratch are required");
    return LBM_ERR_INVALID;
  }
  if (scratch_bytes < ibm_spread_tiled_scratch_bytes(lat, pt->n_markers)) {
    set_error("ibm_spread_tiled: scratch of %zu bytes, %zu needed", scratch_bytes,
              ibm_spread_tiled_scratch_bytes(lat, pt->n_markers));
    return LBM_ERR_INVALID;
  }
  if ((rc = check_precision(lat, pt, "ibm_spread_tiled"))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  TileArgs a;
  memset(&a, 0, sizeof(a));
  a.g = make_geom(lat);
  a.p = *pt;
  a.field = field;
  a.chunks = chunks;
  tile_dims(a.g, a.tx, a.ty, a.tz);
  const long long ntiles = (long long)a.tx * a.ty * a.tz;
  char *base = static_cast<char *>(scratch);
  a.tile_count = reinterpret_cast<int *>(base);
  a.tile_list = a.tile_count + ntiles;
  const size_t off = ((size_t)(ntiles + ntiles * kTileCap) * 4 + 255) / 256 * 256;
  a.wsum = base + off;
  const bool fp64 = lat->storage == LBM_STORAGE_FP64;
  const long long nchunks = (a.g.n + 31) >> 5;
  if (fp64)
    launch_chained(k_spread_clear<double>, blocks_for(nchunks, 256), 256, 0, s, a.g.n, (double *)field, chunks);
  else
    launch_chained(k_spread_clear<float>, blocks_for(nchunks, 256), 256, 0, s, a.g.n, field, chunks);
  LBM_LAUNCH_CHECK("ibm_spread_tiled");
  if (pt->n_markers == 0) return LBM_OK;
  const unsigned nb = (unsigned)((pt->n_markers + kMarkersPerBlock - 1) / kMarkersPerBlock);
  if (fp64) {
    k_spread_bin<double><<<nb, kIbmThreads, 0, s>>>(a);
    if (mode == 0)
      k_spread_tile<double, 0><<<(unsigned)ntiles, kTileNodes, 0, s>>>(a);
    else
      k_spread_tile<double, 1><<<(unsigned)ntiles, kTileNodes, 0, s>>>(a);
  } else {
    k_spread_bin<float><<<nb, kIbmThreads, 0, s>>>(a);
    if (mode == 0)
      k_spread_tile<float, 0><<<(unsigned)ntiles, kTileNodes, 0, s>>>(a);
    else
      k_spread_tile<float, 1><<<(unsigned)ntiles, kTileNodes, 0, s>>>(a);
  }
  LBM_LAUNCH_CHECK("ibm_spread_tiled");
  return LBM_OK;
}

int rigid_update_markers(const lbm_particles *pt, void *stream) {
  int rc = check_particles(pt, "rigid_update_markers");
  if (rc) return rc;
  if (pt->n_particles == 0) return LBM_OK;
  if (pt->fp64)
    k_markers<double><<<pt->n_particles, kRigidThreads, 0, (cudaStream_t)stream>>>(*pt);
  else
    k_markers<float><<<pt->n_particles, kRigidThreads, 0, (cudaStream_t)stream>>>(*pt);
  LBM_LAUNCH_CHECK("rigid_update_markers");
  return LBM_OK;
}

// Same spreading as ibm_spread, with the per-node claim array taken from the
// library's static device array instead of from the caller.
int ibm_spread_noalloc(const lbm_lattice *lat, const lbm_particles *pt, int32_t mode, float *field,
                       uint8_t *chunks, void *stream) {
  int rc = check_lattice(lat);
  if (rc) return rc;
  if ((rc = check_particles(pt, "ibm_spread_noalloc"))) return rc;
  if (mode != 0 && mode != 1) {
    set_error("ibm_spread_noalloc: mode must be 0 (reference) or 1 (accumulate)");
    return LBM_ERR_INVALID;
  }
  if (field == nullptr || chunks == nullptr) {
    set_error("ibm_spread_noalloc: field and chunks are required");
    return LBM_ERR_INVALID;
  }
  const long long n = (long long)lat->nx * lat->ny * lat->nz;
  if (n > LBM_SPREAD_NOALLOC_MAX_NODES) {
    set_error("ibm_spread_noalloc: the lattice has %lld nodes, more than the %d nodes its "
              "built-in claim array holds; use ibm_spread with a caller-owned array",
              n, (int)LBM_SPREAD_NOALLOC_MAX_NODES);
    return LBM_ERR_INVALID;
  }
  if ((rc = check_precision(lat, pt, "ibm_spread_noalloc"))) return rc;
  int32_t *owner = nullptr;
  int dev = 0;
  bool clean = false;
  if ((rc = owner_scratch(&owner, &dev, &clean))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  SpreadArgs a;
  a.g = make_geom(lat);
  a.p = *pt;
  a.field = field;
  a.chunks = chunks;
  a.owner = owner;
  const bool claims = mode == 0 && pt->n_markers > 0;
  if (claims) {
    // the claim pass needs -1 in every slot it touches; the write pass
    // restores it, so only the first reference-mode call on a device (or
    // one after a failed call) resets the whole array
    owner_mark(dev, false);
    if (!clean) {
      k_owner_reset<<<(unsigned)std::min<long long>(
                          (LBM_SPREAD_NOALLOC_MAX_NODES + 255) / 256, 4096),
                      256, 0, s>>>(owner, LBM_SPREAD_NOALLOC_MAX_NODES);
      LBM_LAUNCH_CHECK("ibm_spread_noalloc");
    }
  }
  rc = lat->storage == LBM_STORAGE_FP64
           ? spread_launch<double>(a, mode, pt->n_markers, s, "ibm_spread_noalloc")
           : spread_launch<float>(a, mode, pt->n_markers, s, "ibm_spread_noalloc");
  if (rc == LBM_OK && claims) owner_mark(dev, true);
  return rc;
}

}  // extern "C"
