// Error reporting, lattice validation and Geom construction for the C ABI.
#include <atomic>
#include <cmath>
#include <mutex>
#include <vector>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "lbm_api.cuh"

namespace lbm {

namespace {
thread_local char g_msg[512] = "";
std::atomic<unsigned> g_tma_wait_polls{kTmaWaitPollsDefault};
}

unsigned tma_wait_polls() { return g_tma_wait_polls.load(std::memory_order_relaxed); }

namespace {
std::mutex g_oob_mu;
std::vector<OobReader> &oob_readers() {
  static std::vector<OobReader> v;
  return v;
}
}  // namespace

void register_oob_reader(OobReader r) {
  std::lock_guard<std::mutex> lock(g_oob_mu);
  oob_readers().push_back(r);
}

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
}

bool chained_launches() {
  static const bool on = [] {
    const char *v = std::getenv("FUNLBM_B200_CHAIN");
    return v == nullptr || std::strcmp(v, "0") != 0;
  }();
  return on;
}

int fail_cuda(cudaError_t e, const char *where) {
  set_error("%s: CUDA error %d (%s)", where, (int)e, cudaGetErrorString(e));
  return LBM_ERR_CUDA;
}

bool any_face(const lbm_lattice *lat, int code) {
  for (int i = 0; i < LBM_NFACES; ++i)
    if (lat->face[i] == code) return true;
  return false;
}

static const char *kFaceName[LBM_NFACES] = {"input", "output", "back", "forward", "bottom", "top"};

int check_lattice(const lbm_lattice *lat) {
  if (lat == nullptr) {
    set_error("lattice description is NULL");
    return LBM_ERR_INVALID;
  }
  if (lat->q != 13 && lat->q != 15 && lat->q != 19 && lat->q != 27) {
    set_error("Unknown parameter type: D3Q%d", lat->q);
    return LBM_ERR_INVALID;
  }
  if (lat->nx < 2 || lat->ny < 2 || lat->nz < 2) {
    set_error("lattice needs at least 2 nodes per axis (got %d x %d x %d)", lat->nx, lat->ny,
              lat->nz);
    return LBM_ERR_INVALID;
  }
  const long long n = (long long)lat->nx * lat->ny * lat->nz;
  if (n >= (1ll << 31)) {
    set_error("lattice of %lld nodes exceeds the 2^31 node limit of one lattice", n);
    return LBM_ERR_INVALID;
  }
  if (!(lat->tau > 0.5f) || !std::isfinite(lat->tau)) {
    set_error("relaxation time tau=%g must exceed 0.5", (double)lat->tau);
    return LBM_ERR_INVALID;
  }
  if (lat->pz != 0 && (lat->pz < lat->nz ||
                       (long long)lat->nx * lat->ny * lat->pz >= (1ll << 31))) {
    set_error("row pitch %d must be 0 or at least nz = %d (and the pitched lattice under "
              "2^31 elements per direction)", lat->pz, lat->nz);
    return LBM_ERR_INVALID;
  }
  if (lat->storage < LBM_STORAGE_FP32 || lat->storage > LBM_STORAGE_FP64) {
    set_error("unknown population storage %d", lat->storage);
    return LBM_ERR_INVALID;
  }
  for (int fc = 0; fc < LBM_NFACES; ++fc) {
    const int c = lat->face[fc];
    const bool plain = c == LBM_BC_PERIODICAL || c == LBM_BC_WALL || c == LBM_BC_WALL_WITH_SPEED;
    const bool neq_ok = fc < 2 && c == LBM_BC_NON_EQUILIBRIUM;
    if (!plain && !neq_ok) {
      set_error("boundary code %d is not implemented on face '%s'", c, kFaceName[fc]);
      return LBM_ERR_UNSUPPORTED;
    }
  }
  if (any_face(lat, LBM_BC_NON_EQUILIBRIUM) && lat->nx < 3) {
    set_error("NON_EQUILIBRIUM faces need at least 3 nodes along x");
    return LBM_ERR_INVALID;
  }
  if (lat->face[0] == LBM_BC_NON_EQUILIBRIUM && lat->neq_profile == nullptr) {
    set_error("NON_EQUILIBRIUM input face needs the inlet profile");
    return LBM_ERR_INVALID;
  }
  return LBM_OK;
}

Geom make_geom(const lbm_lattice *lat) {
  Geom g;
  std::memset(&g, 0, sizeof(g));
  g.nx = lat->nx;
  g.ny = lat->ny;
  g.nz = lat->nz;
  g.nyz = (long long)lat->ny * lat->nz;
  g.n = g.nyz * lat->nx;
  g.pz = lat->pz > 0 ? lat->pz : lat->nz;
  g.nyzp = (long long)lat->ny * g.pz;
  g.np = g.nyzp * lat->nx;
  for (int i = 0; i < LBM_NFACES; ++i) {
    g.face[i] = lat->face[i];
    for (int k = 0; k < 3; ++k) g.uw[i][k] = lat->face_uw[i][k];
  }
  const long long yz = (long long)g.ny * g.nz, xz = (long long)g.nx * g.nz,
                  xy = (long long)g.nx * g.ny;
  g.plane_off[0] = 0;
  g.plane_off[1] = yz;
  g.plane_off[2] = 2 * yz;
  g.plane_off[3] = 2 * yz + xz;
  g.plane_off[4] = 2 * yz + 2 * xz;
  g.plane_off[5] = 2 * yz + 2 * xz + xy;
  g.tau = lat->tau;
  g.inv_tau = 1.0f / lat->tau;
  g.cs2 = lat->cs2;
  g.inv_cs2 = 1.0f / lat->cs2;
  const float cs4 = lat->cs2 * lat->cs2;
  g.inv_cs4 = 1.0f / cs4;
  g.force_c = 1.0f - 1.0f / (2.0f * lat->tau);
  g.re_mu = lat->re_mu;
  g.neq_profile = lat->neq_profile;
  const double tau = (double)lat->tau;
  const double cs = std::sqrt(1.0 / 3.0);
  const double cs2 = cs * cs;
  g.inv_tau_d = 1.0 / tau;
  g.inv_cs2_d = 1.0 / cs2;
  g.inv_cs4_d = 1.0 / (cs2 * cs2);
  g.force_c_d = 1.0 - 1.0 / (2.0 * tau);
  for (int i = 0; i < LBM_NFACES; ++i)
    for (int k = 0; k < 3; ++k) g.uw_d[i][k] = (double)lat->face_uw[i][k];
  return g;
}

// Plane pointers (StepPlanes) for velocity set q, elements
// of `elem` bytes.  Pure address arithmetic: nothing is dereferenced here.
template <int Q>
static void fill_planes_q(const Geom &g, const void *fa, void *fb, int elem, StepPlanes &p) {
  using V = VSet<Q>;
  const uintptr_t a = (uintptr_t)fa, b = (uintptr_t)fb;
  auto at = [&](uintptr_t base, long long e) { return base + (uintptr_t)(e * elem); };
  for (int i = 0; i < Q; ++i) {
    const long long plane = (long long)i * g.np, rplane = (long long)V::rev(i) * g.np;
    p.src[i] = (const void *)at(a, plane - (long long)V::ex(i) * g.nyzp - (long long)V::ey(i) * g.pz);
    p.zlo[i] = nullptr;
    p.zhi[i] = nullptr;
    if (V::ez(i) > 0)
      p.zlo[i] = (const void *)(g.face[4] == LBM_BC_PERIODICAL ? at(a, plane + g.nz - 1)
                                                               : at(a, rplane));
    if (V::ez(i) < 0)
      p.zhi[i] = (const void *)(g.face[5] == LBM_BC_PERIODICAL ? at(a, plane - (g.nz - 1))
                                                               : at(a, rplane));
    p.dst[i] = fb == nullptr ? nullptr : (void *)at(b, plane);
  }
}

void fill_step_planes(const Geom &g, int q, int storage, const void *fa, void *fb,
                             StepPlanes &p) {
  const int elem = storage_bits(storage) / 8;
  switch (q) {
    case 13: fill_planes_q<13>(g, fa, fb, elem, p); break;
    case 15: fill_planes_q<15>(g, fa, fb, elem, p); break;
    case 19: fill_planes_q<19>(g, fa, fb, elem, p); break;
    default: fill_planes_q<27>(g, fa, fb, elem, p); break;
  }
}

}  // namespace lbm

extern "C" {

const char *lbm_last_error(void) { return lbm::g_msg; }

const char *lbm_version(void) { return "funlbm_b200 0.1.0 (sm_100a)"; }

size_t lbm_face_plane_floats(const lbm_lattice *lat) {
  if (lat == nullptr) return 0;
  const size_t yz = (size_t)lat->ny * lat->nz, xz = (size_t)lat->nx * lat->nz,
               xy = (size_t)lat->nx * lat->ny;
  return 2 * (yz + xz + xy);
}

int lbm_lattice_check(const lbm_lattice *lat) { return lbm::check_lattice(lat); }

int64_t lbm_debug_bounds_faults(int32_t reset) {
#ifdef LBM_BOUNDS_CHECK
  std::lock_guard<std::mutex> lock(lbm::g_oob_mu);
  unsigned long long total = 0;
  for (auto r : lbm::oob_readers()) {
    const unsigned long long v = r(reset != 0);
    if (v == ~0ull) return -2;
    total += v;
  }
  return (int64_t)total;
#else
  (void)reset;
  return -1;
#endif
}

void lbm_debug_set_wait_limit(int64_t polls) {
  const unsigned v = polls < 0 ? lbm::kTmaWaitPollsDefault
                     : polls > (int64_t)lbm::kTmaWaitPollsDefault ? lbm::kTmaWaitPollsDefault
                                                                   : (unsigned)polls;
  lbm::g_tma_wait_polls.store(v, std::memory_order_relaxed);
}

}  // extern "C"
