// grhd2_gpu.cu -- C-ABI of the B200 per-stage path (include/grhd2_gpu.h).
//
// One handle = one grid on the current device, one CUDA stream.  Device state:
//   P      primitives, SoA interior planes (double, or float under the mixed policy)
//   U, UP  conserved u and up of grhd2.f90:232-249, SoA interior planes (double)
//   F[d]   face fluxes of direction d (double, or float under the mixed policy)
//   tables k-invariant metric tables per (i,j) and per face (see state.cuh)
// A step is 3 x (face_flux per active direction, cell_update); the first stage also
// performs u = up.  Ghost cells are evaluated on load (state.cuh), so no boundary pass
// runs between stages.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "grhd2_gpu.h"
#include "frame.h"
#include "kernels.cuh"

using namespace grhd;

struct grhd2_gpu {
  grhd2_gpu_config cfg{};
  Phys phys{};
  GridDev G{};
  int device = 0;
  bool mixed = false;
  cudaStream_t stream = nullptr;
  // device buffers
  void *P = nullptr;
  double *U = nullptr, *UP = nullptr, *RHS = nullptr;
  void *F[3] = {nullptr, nullptr, nullptr};
  double *centre = nullptr, *face[3] = {nullptr, nullptr, nullptr};
  double *inj = nullptr, *dust = nullptr, *xc = nullptr, *frozen[3] = {nullptr, nullptr, nullptr};
  unsigned long long *cnt = nullptr, *red = nullptr;
  double *staging = nullptr;
  size_t n_ghosted = 0, n_interior = 0;
  bool metric_set = false, bc_set = false, prims_set = false, cons_set = false;
  double dt_cache = 0.0;
  bool dt_valid = false;
  std::string err;
  // per-launch timing (grhd2_gpu_profile_step): events recorded after every launch
  std::vector<cudaEvent_t> prof_ev;
  std::vector<const char *> prof_names;
  bool profiling = false;
};

namespace {

int fail(grhd2_gpu *h, int code, const char *fmt, ...) {
  if (h) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    h->err = buf;
  }
  return code;
}

#define CUDA_TRY(h, call)                                                                        \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) return fail((h), GRHD2_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

template <class T>
int dalloc(grhd2_gpu *h, T **p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
  if (e != cudaSuccess) return fail(h, GRHD2_ERR_NOMEM, "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
  return 0;
}

inline unsigned nblocks(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

bool bit_equal(double a, double b) { return std::memcmp(&a, &b, sizeof a) == 0; }

int launch_check(grhd2_gpu *h, const char *name = nullptr) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(h, GRHD2_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
  if (h->profiling && name) {
    cudaEvent_t ev;
    if (cudaEventCreate(&ev) != cudaSuccess) return fail(h, GRHD2_ERR_CUDA, "cudaEventCreate failed");
    cudaEventRecord(ev, h->stream);
    h->prof_ev.push_back(ev);
    h->prof_names.push_back(name);
  }
  return 0;
}

// ---- kernel dispatch ---------------------------------------------------------------
template <class R, class PT>
int launch_fluxes(grhd2_gpu *h) {
  const GridDev &G = h->G;
  const PT *P = (const PT *)h->P;
  int rc;
  k_face_flux<1, R, PT><<<nblocks(G.nface[0] * G.nz, 128), 128, 0, h->stream>>>(G, h->phys, P, (R *)h->F[0], h->cnt);
  if ((rc = launch_check(h, "face_flux_x"))) return rc;
  if (G.ny > 1) {
    k_face_flux<2, R, PT><<<nblocks((long long)G.nx * (G.ny + 1) * G.nz, 128), 128, 0, h->stream>>>(G, h->phys, P, (R *)h->F[1], h->cnt);
    if ((rc = launch_check(h, "face_flux_y"))) return rc;
  }
  if (G.nz > 1) {
    k_face_flux<3, R, PT><<<nblocks((long long)G.nx * G.ny * (G.nz + 1), 128), 128, 0, h->stream>>>(G, h->phys, P, (R *)h->F[2], h->cnt);
    if ((rc = launch_check(h, "face_flux_z"))) return rc;
  }
  return 0;
}

template <int MODE, class R, class PT>
int launch_update(grhd2_gpu *h, double dt) {
  const GridDev &G = h->G;
  k_cell_update<MODE, R, PT><<<nblocks(G.ncell, 128), 128, 0, h->stream>>>(
      G, h->phys, (PT *)h->P, (const R *)h->F[0], (const R *)h->F[1], (const R *)h->F[2], h->U, h->UP, h->RHS, dt,
      h->cfg.dx, h->cfg.dy, h->cfg.dz, h->cnt);
  return launch_check(h, MODE == 0 ? "cell_rhs" : "cell_update");
}

template <class R, class PT>
int do_step(grhd2_gpu *h, double dt) {
  int rc;
  if ((rc = launch_fluxes<R, PT>(h))) return rc;
  if ((rc = launch_update<1, R, PT>(h, dt))) return rc;
  if ((rc = launch_fluxes<R, PT>(h))) return rc;
  if ((rc = launch_update<2, R, PT>(h, dt))) return rc;
  if ((rc = launch_fluxes<R, PT>(h))) return rc;
  return launch_update<3, R, PT>(h, dt);
}

int step_dispatch(grhd2_gpu *h, double dt) {
  return h->mixed ? do_step<float, float>(h, dt) : do_step<double, double>(h, dt);
}

int ready(grhd2_gpu *h, bool need_state) {
  if (!h) return GRHD2_ERR_ARG;
  if (!h->metric_set) return fail(h, GRHD2_ERR_STATE, "metric tables not set (call grhd2_gpu_set_metric first)");
  const int cs = h->cfg.case_id;
  if ((cs == 7 || cs == 8 || cs == 5) && !h->bc_set)
    return fail(h, GRHD2_ERR_STATE, "boundary data not set for case %d (call grhd2_gpu_set_bc_data)", cs);
  if (need_state && !(h->prims_set && h->cons_set)) return fail(h, GRHD2_ERR_STATE, "state not uploaded");
  CUDA_TRY(h, cudaSetDevice(h->device));
  return 0;
}

// face table for n faces of direction dir from Fortran-order face-cache slices
int build_face_table(grhd2_gpu *h, std::vector<double> &T, size_t n, int dir, const double *alpha,
                     const double *beta, const double *gamma, const double *sqg, const std::vector<uint8_t> &zero) {
  T.assign((size_t)NFF * n, 0.0);
  for (size_t f = 0; f < n; ++f) {
    const double *g = &gamma[9 * f];
    if (!bit_equal(g[1], g[3]) || !bit_equal(g[2], g[6]) || !bit_equal(g[5], g[7]))
      return fail(h, GRHD2_ERR_ARG, "face metric of direction %d is not exactly symmetric at face %zu", dir, f);
    T[FF_ALPHA * n + f] = alpha[f];
    T[FF_BETA_N * n + f] = beta[3 * f + (dir - 1)];
    T[FF_G11 * n + f] = g[0]; T[FF_G12 * n + f] = g[3]; T[FF_G13 * n + f] = g[6];
    T[FF_G22 * n + f] = g[4]; T[FF_G23 * n + f] = g[7]; T[FF_G33 * n + f] = g[8];
    T[FF_SQG * n + f] = sqg[f];
    T[FF_GUP * n + f] = gamma_up_dd(g, dir);
    double cof[9], gup;
    const bool ok = face_frame(g, dir, cof, &gup);
    for (int q = 0; q < 9; ++q) T[(FF_COF + q) * n + f] = cof[q];
    if (ok && !bit_equal(gup, T[FF_GUP * n + f]))
      return fail(h, GRHD2_ERR_ARG, "internal: frame gamma^dd differs from the wavespeed gamma^dd");
    T[FF_FRAME_OK * n + f] = ok ? 1.0 : 0.0;
    T[FF_ZERO * n + f] = zero.empty() ? 0.0 : (double)zero[f];
  }
  return 0;
}

}  // namespace

// ======================================================================================
extern "C" {

int grhd2_gpu_abi_version(void) { return GRHD2_GPU_ABI_VERSION; }

int grhd2_gpu_create(const grhd2_gpu_config *cfg, grhd2_gpu **out) {
  if (!cfg || !out) return GRHD2_ERR_ARG;
  *out = nullptr;
  grhd2_gpu *h = new (std::nothrow) grhd2_gpu();
  if (!h) return GRHD2_ERR_NOMEM;
  *out = h;  // the caller can read last_error even on failure; destroy() frees it
  h->cfg = *cfg;
  const grhd2_gpu_config &c = *cfg;
  if (c.neq != 5) return fail(h, GRHD2_ERR_ARG, "neq must be 5 (got %d)", c.neq);
  if (c.nx < 2 || c.ny < 1 || c.nz < 1) return fail(h, GRHD2_ERR_ARG, "grid %dx%dx%d unsupported (nx >= 2 required)", c.nx, c.ny, c.nz);
  if (c.rec_method < 1 || c.rec_method > 5) return fail(h, GRHD2_ERR_ARG, "invalid reconstruction id %d", c.rec_method);
  const int ng_need = c.rec_method == 1 ? 1 : (c.rec_method <= 3 ? 2 : 3);
  if (c.nghost != ng_need) return fail(h, GRHD2_ERR_ARG, "nghost %d does not match the reconstruction (%d)", c.nghost, ng_need);
  if (c.riemann != 1 && c.riemann != 2) return fail(h, GRHD2_ERR_ARG, "riemann solver id %d unsupported (1 HLLE, 2 HLLC)", c.riemann);
  if (c.case_id < 1 || c.case_id > 12) return fail(h, GRHD2_ERR_ARG, "invalid case id %d", c.case_id);
  if (c.metric_kind < 0 || c.metric_kind > 2 || c.geom_kind < 0 || c.geom_kind > 3) return fail(h, GRHD2_ERR_ARG, "invalid metric/geometry id");
  if (c.precision_policy != GRHD2_PREC_FP64 && c.precision_policy != GRHD2_PREC_MIXED)
    return fail(h, GRHD2_ERR_ARG, "invalid precision policy %d", c.precision_policy);
  if (c.case_id == 12 && (c.nz % 2) != 0) return fail(h, GRHD2_ERR_BOUNDARY, "nz must be even for 3D trans-polar boundary conditions");
  if ((c.case_id == 11 || c.case_id == 12) && c.ny < c.nghost)
    return fail(h, GRHD2_ERR_ARG, "reflecting/trans-polar boundaries need ny >= nghost");
  if (c.case_id == 5 && (c.nx < c.nghost || c.nz < c.nghost))
    return fail(h, GRHD2_ERR_ARG, "the jet's reflecting boundaries need nx, nz >= nghost");
  if (!(c.dx > 0) || (c.ny > 1 && !(c.dy > 0)) || (c.nz > 1 && !(c.dz > 0))) return fail(h, GRHD2_ERR_ARG, "grid spacing must be positive");

  h->mixed = c.precision_policy == GRHD2_PREC_MIXED;
  h->phys.rec = c.rec_method; h->phys.lim = c.tvd_limiter; h->phys.rs = c.riemann; h->phys.sensor = c.shock_sensor ? 1 : 0;
  h->phys.nonmink = c.metric_kind != GRHD2_METRIC_MINKOWSKI;
  h->phys.srhd = c.metric_kind == GRHD2_METRIC_MINKOWSKI && c.geom_kind == GRHD2_GEOM_CARTESIAN;
  h->phys.adb = c.adb_idx; h->phys.g1 = c.g1; h->phys.rho_floor = c.rho_floor; h->phys.p_floor = c.p_floor; h->phys.v_max = c.v_max;

  GridDev &G = h->G;
  G.nx = c.nx; G.ny = c.ny; G.nz = c.nz; G.ng = c.nghost; G.case_id = c.case_id;
  G.ncell = (long long)c.nx * c.ny * c.nz;
  G.pplane = (G.ncell + 31) / 32 * 32;
  G.nij = (long long)c.nx * c.ny;
  G.nface[0] = (long long)(c.nx + 1) * c.ny;
  G.nface[1] = (long long)c.nx * (c.ny + 1);
  G.nface[2] = G.nij;
  G.rho_floor = c.rho_floor; G.p_floor = c.p_floor;

  CUDA_TRY(h, cudaGetDevice(&h->device));
  CUDA_TRY(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  int rc;
  const size_t es = h->mixed ? sizeof(float) : sizeof(double);
  if ((rc = dalloc(h, (char **)&h->P, 5 * G.pplane * es))) return rc;
  if ((rc = dalloc(h, &h->U, 5 * G.pplane))) return rc;
  if ((rc = dalloc(h, &h->UP, 5 * G.pplane))) return rc;
  const long long nfx = (long long)(c.nx + 1) * c.ny * c.nz;
  if ((rc = dalloc(h, (char **)&h->F[0], 5 * nfx * es))) return rc;
  if (c.ny > 1 && (rc = dalloc(h, (char **)&h->F[1], 5 * (long long)c.nx * (c.ny + 1) * c.nz * es))) return rc;
  if (c.nz > 1 && (rc = dalloc(h, (char **)&h->F[2], 5 * (long long)c.nx * c.ny * (c.nz + 1) * es))) return rc;
  if ((rc = dalloc(h, &h->cnt, NCNT))) return rc;
  if ((rc = dalloc(h, &h->red, 4))) return rc;
  CUDA_TRY(h, cudaMemsetAsync(h->cnt, 0, NCNT * sizeof(unsigned long long), h->stream));
  h->n_ghosted = (size_t)5 * (c.nx + 2 * c.nghost + 1) * (c.ny + 2 * c.nghost + 1) * (c.nz + 2 * c.nghost + 1);
  h->n_interior = (size_t)5 * G.ncell;
  if ((rc = dalloc(h, &h->staging, h->n_ghosted))) return rc;
  if (c.nghost == 2) {
    if ((rc = dalloc(h, &h->frozen[0], 5 * (size_t)c.ny * c.nz))) return rc;
    if ((rc = dalloc(h, &h->frozen[1], 5 * (size_t)c.nx * c.nz))) return rc;
    if ((rc = dalloc(h, &h->frozen[2], 5 * (size_t)c.nx * c.ny))) return rc;
    for (int d = 0; d < 3; ++d) G.frozen[d] = h->frozen[d];
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  h->err.clear();
  return GRHD2_OK;
}

int grhd2_gpu_set_metric(grhd2_gpu *h, const grhd2_gpu_metric_view *m) {
  if (!h || !m) return GRHD2_ERR_ARG;
  const grhd2_gpu_config &c = h->cfg;
  if (!m->alpha_c || !m->beta_c || !m->gamma_c || !m->gamma_inv_c || !m->gmunu_c || !m->sqrt_gamma_c || !m->chris_c ||
      !m->dg_c || !m->dlna_c || !m->alpha_f_x || !m->beta_f_x || !m->gamma_f_x || !m->sqrt_gamma_f_x || !m->x_face)
    return fail(h, GRHD2_ERR_ARG, "metric view has NULL centre or x-face arrays");
  if (c.ny > 1 && (!m->alpha_f_y || !m->beta_f_y || !m->gamma_f_y || !m->sqrt_gamma_f_y || !m->y_face))
    return fail(h, GRHD2_ERR_ARG, "metric view has NULL y-face arrays (ny > 1)");
  if (c.nz > 1 && (!m->alpha_f_z || !m->beta_f_z || !m->gamma_f_z || !m->sqrt_gamma_f_z))
    return fail(h, GRHD2_ERR_ARG, "metric view has NULL z-face arrays (nz > 1)");
  CUDA_TRY(h, cudaSetDevice(h->device));
  const size_t nij = (size_t)c.nx * c.ny;
  std::vector<double> C((size_t)NCF * nij, 0.0);
  for (size_t q = 0; q < nij; ++q) {
    const double *g = &m->gamma_c[9 * q], *gi = &m->gamma_inv_c[9 * q], *gm = &m->gmunu_c[16 * q];
    const double *ch = &m->chris_c[64 * q], *dg = &m->dg_c[48 * q];
    if (!bit_equal(g[1], g[3]) || !bit_equal(g[2], g[6]) || !bit_equal(g[5], g[7]) || !bit_equal(gi[1], gi[3]) ||
        !bit_equal(gi[2], gi[6]) || !bit_equal(gi[5], gi[7]))
      return fail(h, GRHD2_ERR_ARG, "gamma_c / gamma_inv_c not exactly symmetric at cell %zu", q);
    C[CF_ALPHA * nij + q] = m->alpha_c[q];
    for (int d = 0; d < 3; ++d) C[(CF_B1 + d) * nij + q] = m->beta_c[3 * q + d];
    const int sidx[6] = {0, 3, 6, 4, 7, 8};  // (1,1) (1,2) (1,3) (2,2) (2,3) (3,3)
    for (int s = 0; s < 6; ++s) { C[(CF_G11 + s) * nij + q] = g[sidx[s]]; C[(CF_I11 + s) * nij + q] = gi[sidx[s]]; }
    C[CF_SQG * nij + q] = m->sqrt_gamma_c[q];
    for (int mu = 0; mu < 4; ++mu)
      for (int nu = mu; nu < 4; ++nu) {
        if (!bit_equal(gm[mu + 4 * nu], gm[nu + 4 * mu]) || !bit_equal(ch[4 * mu + 16 * nu], ch[4 * nu + 16 * mu]))
          return fail(h, GRHD2_ERR_ARG, "gmunu_c / chris_c(0,:,:) not exactly symmetric at cell %zu", q);
        C[(CF_GM + sym4(mu, nu)) * nij + q] = gm[mu + 4 * nu];
        C[(CF_CH0 + sym4(mu, nu)) * nij + q] = ch[0 + 4 * mu + 16 * nu];
        for (int d = 0; d < 3; ++d) {
          if (!bit_equal(dg[mu + 4 * nu + 16 * d], dg[nu + 4 * mu + 16 * d]))
            return fail(h, GRHD2_ERR_ARG, "dg_c not exactly symmetric at cell %zu", q);
          C[(CF_DG + 10 * d + sym4(mu, nu)) * nij + q] = dg[mu + 4 * nu + 16 * d];
        }
      }
    for (int mu = 0; mu < 4; ++mu) C[(CF_DLNA + mu) * nij + q] = m->dlna_c[4 * q + mu];
    C[CF_VA * nij + q] = m->beta_c[3 * q] / m->alpha_c[q];
  }
  // faces
  const double eps64 = 64.0 * DBL_EPSILON;
  std::vector<double> T[3];
  int rc;
  {
    const size_t n = (size_t)(c.nx + 1) * c.ny;
    std::vector<uint8_t> zero(n, 0);
    if (c.geom_kind == GRHD2_GEOM_CYLINDRICAL)  // evolution.f90:69-71
      for (size_t f = 0; f < n; ++f) zero[f] = std::fabs(m->x_face[f % (c.nx + 1)]) <= eps64;
    if ((rc = build_face_table(h, T[0], n, 1, m->alpha_f_x, m->beta_f_x, m->gamma_f_x, m->sqrt_gamma_f_x, zero))) return rc;
  }
  if (c.ny > 1) {
    const size_t n = (size_t)c.nx * (c.ny + 1);
    std::vector<uint8_t> zero(n, 0);
    if (c.geom_kind == GRHD2_GEOM_SPHERICAL || c.geom_kind == GRHD2_GEOM_SPHEROIDAL)  // evolution.f90:122-124
      for (size_t f = 0; f < n; ++f) zero[f] = std::fabs(std::sin(m->y_face[f / c.nx])) <= eps64;
    if ((rc = build_face_table(h, T[1], n, 2, m->alpha_f_y, m->beta_f_y, m->gamma_f_y, m->sqrt_gamma_f_y, zero))) return rc;
  }
  if (c.nz > 1) {
    const size_t n = nij;
    if ((rc = build_face_table(h, T[2], n, 3, m->alpha_f_z, m->beta_f_z, m->gamma_f_z, m->sqrt_gamma_f_z, {}))) return rc;
  }
  if (!h->centre && (rc = dalloc(h, &h->centre, C.size()))) return rc;
  CUDA_TRY(h, cudaMemcpyAsync(h->centre, C.data(), C.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  for (int d = 0; d < 3; ++d) {
    if (T[d].empty()) continue;
    if (!h->face[d] && (rc = dalloc(h, &h->face[d], T[d].size()))) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(h->face[d], T[d].data(), T[d].size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));  // host vectors go out of scope
  h->G.centre = h->centre;
  for (int d = 0; d < 3; ++d) h->G.face[d] = h->face[d];
  h->metric_set = true;
  h->dt_valid = false;
  return GRHD2_OK;
}

int grhd2_gpu_set_bc_data(grhd2_gpu *h, const grhd2_gpu_bc_view *b) {
  if (!h || !b) return GRHD2_ERR_ARG;
  const grhd2_gpu_config &c = h->cfg;
  CUDA_TRY(h, cudaSetDevice(h->device));
  int rc;
  if (c.case_id == 7) {
    if (!b->michel_injector) return fail(h, GRHD2_ERR_ARG, "Michel case needs michel_injector");
    const size_t n = (size_t)5 * c.nghost * c.ny * c.nz;
    std::vector<double> t(n);
    for (size_t q = 0; q < n / 5; ++q)
      for (int v = 0; v < 5; ++v) t[v * (n / 5) + q] = b->michel_injector[5 * q + v];
    if (!h->inj && (rc = dalloc(h, &h->inj, n))) return rc;
    CUDA_TRY(h, cudaMemcpy(h->inj, t.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    h->G.inj = h->inj;
  }
  if (c.case_id == 8) {
    if (!b->dust_outer) return fail(h, GRHD2_ERR_ARG, "dust case needs dust_outer");
    const size_t n = (size_t)5 * c.nghost;
    std::vector<double> t(n);
    for (int g = 0; g < c.nghost; ++g)
      for (int v = 0; v < 5; ++v) t[v * c.nghost + g] = b->dust_outer[5 * g + v];
    if (!h->dust && (rc = dalloc(h, &h->dust, n))) return rc;
    CUDA_TRY(h, cudaMemcpy(h->dust, t.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    h->G.dust = h->dust;
  }
  if (c.case_id == 5) {
    if (!b->x_c) return fail(h, GRHD2_ERR_ARG, "jet case needs x_c");
    const size_t n = (size_t)c.nx + 2 * c.nghost + 1;
    if (!h->xc && (rc = dalloc(h, &h->xc, n))) return rc;
    CUDA_TRY(h, cudaMemcpy(h->xc, b->x_c, n * sizeof(double), cudaMemcpyHostToDevice));
    h->G.xc = h->xc;
  }
  for (int q = 0; q < 7; ++q) h->G.jet[q] = b->jet[q];
  h->bc_set = true;
  return GRHD2_OK;
}

int grhd2_gpu_upload(grhd2_gpu *h, const double *up, const double *p) {
  if (!h) return GRHD2_ERR_ARG;
  CUDA_TRY(h, cudaSetDevice(h->device));
  const GridDev &G = h->G;
  if (p) {
    CUDA_TRY(h, cudaMemcpyAsync(h->staging, p, h->n_ghosted * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (h->mixed)
      k_prims_in<float><<<nblocks(G.ncell, 256), 256, 0, h->stream>>>(G, h->staging, (float *)h->P, h->frozen[0],
                                                                     G.ny > 0 ? h->frozen[1] : nullptr, h->frozen[2]);
    else
      k_prims_in<double><<<nblocks(G.ncell, 256), 256, 0, h->stream>>>(G, h->staging, (double *)h->P, h->frozen[0],
                                                                      h->frozen[1], h->frozen[2]);
    if (int rc = launch_check(h)) return rc;
    h->prims_set = true;
  }
  if (up) {
    CUDA_TRY(h, cudaMemcpyAsync(h->staging, up, h->n_interior * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    k_cons_in<<<nblocks(G.ncell, 256), 256, 0, h->stream>>>(G, h->staging, h->UP);
    if (int rc = launch_check(h)) return rc;
    h->cons_set = true;
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return GRHD2_OK;
}

int grhd2_gpu_prim_to_cons_all(grhd2_gpu *h) {
  if (int rc = ready(h, false)) return rc;
  if (!h->prims_set) return fail(h, GRHD2_ERR_STATE, "primitives not uploaded");
  const GridDev &G = h->G;
  if (h->mixed) k_p2c_all<float><<<nblocks(G.ncell, 128), 128, 0, h->stream>>>(G, h->phys, (const float *)h->P, h->UP);
  else k_p2c_all<double><<<nblocks(G.ncell, 128), 128, 0, h->stream>>>(G, h->phys, (const double *)h->P, h->UP);
  if (int rc = launch_check(h)) return rc;
  h->cons_set = true;
  return GRHD2_OK;
}

int grhd2_gpu_cfl(grhd2_gpu *h, double *dt_out) {
  if (!dt_out) return fail(h, GRHD2_ERR_ARG, "dt_out is NULL");
  if (int rc = ready(h, false)) return rc;
  const grhd2_gpu_config &c = h->cfg;
  if (!std::isfinite(c.dx) || c.dx <= 0.0 || (c.ny > 1 && (!std::isfinite(c.dy) || c.dy <= 0.0)) ||
      (c.nz > 1 && (!std::isfinite(c.dz) || c.dz <= 0.0)))
    return fail(h, GRHD2_ERR_CFL, "CRITICAL ERROR: invalid grid spacing in multidimensional CFL condition.");
  if (h->dt_valid) { *dt_out = h->dt_cache; return GRHD2_OK; }
  CUDA_TRY(h, cudaMemsetAsync(h->red, 0, 4 * sizeof(unsigned long long), h->stream));
  k_cfl_reduce<<<148 * 4, 256, 0, h->stream>>>(h->G, h->red);
  if (int rc = launch_check(h)) return rc;
  unsigned long long r[4];
  CUDA_TRY(h, cudaMemcpyAsync(r, h->red, sizeof r, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (r[3] > 0) return fail(h, GRHD2_ERR_CFL, "CRITICAL ERROR: invalid metric data in CFL cells: %llu", r[3]);
  double mx, my, mz;
  std::memcpy(&mx, &r[0], 8); std::memcpy(&my, &r[1], 8); std::memcpy(&mz, &r[2], 8);
  double inv = mx / c.dx;
  if (c.ny > 1) inv = inv + my / c.dy;
  if (c.nz > 1) inv = inv + mz / c.dz;
  if (!std::isfinite(inv) || inv <= 0.0) return fail(h, GRHD2_ERR_CFL, "CRITICAL ERROR: invalid multidimensional CFL propagation rate.");
  h->dt_cache = c.cfl / inv;
  h->dt_valid = true;
  *dt_out = h->dt_cache;
  return GRHD2_OK;
}

int grhd2_gpu_step(grhd2_gpu *h, double dt) {
  if (int rc = ready(h, true)) return rc;
  return step_dispatch(h, dt);
}

int grhd2_gpu_run(grhd2_gpu *h, double t0, double final_time, int64_t max_steps, double *t_out, int64_t *steps_out) {
  if (int rc = ready(h, true)) return rc;
  double dt;
  if (int rc = grhd2_gpu_cfl(h, &dt)) return rc;
  double t = t0;
  int64_t n = 0;
  while (t < final_time && (max_steps < 0 || n < max_steps)) {
    double d = dt;
    if (t + d > final_time) d = final_time - t;  // grhd2.f90:182-184
    ++n;
    t = t + d;
    if (int rc = step_dispatch(h, d)) return rc;
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (t_out) *t_out = t;
  if (steps_out) *steps_out = n;
  return GRHD2_OK;
}

int grhd2_gpu_calc_rhs(grhd2_gpu *h, double *rhs_host) {
  if (int rc = ready(h, false)) return rc;
  if (!h->prims_set) return fail(h, GRHD2_ERR_STATE, "primitives not uploaded");
  int rc;
  if (!h->RHS && (rc = dalloc(h, &h->RHS, 5 * h->G.pplane))) return rc;
  if ((rc = h->mixed ? launch_fluxes<float, float>(h) : launch_fluxes<double, double>(h))) return rc;
  if ((rc = h->mixed ? launch_update<0, float, float>(h, 0.0) : launch_update<0, double, double>(h, 0.0))) return rc;
  if (rhs_host) {
    k_cons_out<<<nblocks(h->G.ncell, 256), 256, 0, h->stream>>>(h->G, h->RHS, h->staging);
    if ((rc = launch_check(h))) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(rhs_host, h->staging, h->n_interior * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return GRHD2_OK;
}

int grhd2_gpu_cons_to_prim_all(grhd2_gpu *h) {
  if (int rc = ready(h, false)) return rc;
  if (!h->cons_set) return fail(h, GRHD2_ERR_STATE, "conserved state not uploaded");
  const GridDev &G = h->G;
  if (h->mixed) k_c2p_all<float><<<nblocks(G.ncell, 128), 128, 0, h->stream>>>(G, h->phys, (float *)h->P, h->UP, h->cnt);
  else k_c2p_all<double><<<nblocks(G.ncell, 128), 128, 0, h->stream>>>(G, h->phys, (double *)h->P, h->UP, h->cnt);
  if (int rc = launch_check(h)) return rc;
  h->prims_set = true;
  return GRHD2_OK;
}

int grhd2_gpu_set_boundary(grhd2_gpu *h) {
  if (int rc = ready(h, false)) return rc;
  if (h->cfg.case_id == 12 && (h->cfg.nz % 2) != 0)
    return fail(h, GRHD2_ERR_BOUNDARY, "CRITICAL ERROR: nz must be even for 3D Trans-Polar boundary conditions.");
  return GRHD2_OK;
}

int grhd2_gpu_download(grhd2_gpu *h, double *up, double *p) {
  if (int rc = ready(h, false)) return rc;
  const GridDev &G = h->G;
  if (p) {
    if (!h->prims_set) return fail(h, GRHD2_ERR_STATE, "primitives not uploaded");
    CUDA_TRY(h, cudaMemcpyAsync(h->staging, p, h->n_ghosted * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    const long long n = (long long)(G.nx + 2 * G.ng + 1) * (G.ny + 2 * G.ng + 1) * (G.nz + 2 * G.ng + 1);
    if (h->mixed) k_prims_out<float><<<nblocks(n, 256), 256, 0, h->stream>>>(G, (const float *)h->P, h->staging);
    else k_prims_out<double><<<nblocks(n, 256), 256, 0, h->stream>>>(G, (const double *)h->P, h->staging);
    if (int rc = launch_check(h)) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(p, h->staging, h->n_ghosted * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  }
  if (up) {
    if (!h->cons_set) return fail(h, GRHD2_ERR_STATE, "conserved state not uploaded");
    k_cons_out<<<nblocks(G.ncell, 256), 256, 0, h->stream>>>(G, h->UP, h->staging);
    if (int rc = launch_check(h)) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(up, h->staging, h->n_interior * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return GRHD2_OK;
}

int grhd2_gpu_get_counters(grhd2_gpu *h, grhd2_gpu_counters *out) {
  if (!h || !out) return GRHD2_ERR_ARG;
  CUDA_TRY(h, cudaSetDevice(h->device));
  unsigned long long c[NCNT];
  CUDA_TRY(h, cudaMemcpyAsync(c, h->cnt, sizeof c, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  out->c2p_floor_pre = (int64_t)c[CNT_FLOOR_PRE];
  out->c2p_causal_rescale = (int64_t)c[CNT_CAUSAL];
  out->c2p_brent_used = (int64_t)c[CNT_BRENT];
  out->c2p_root_fail = (int64_t)c[CNT_ROOT_FAIL];
  out->c2p_bad_V = (int64_t)c[CNT_BAD_V];
  out->c2p_final_sanitise = (int64_t)c[CNT_SANITISE];
  out->recon_floor_clamps = (int64_t)c[CNT_RECON_CLAMP];
  out->hllc_fallbacks = (int64_t)c[CNT_HLLC_FALLBACK];
  return GRHD2_OK;
}

int grhd2_gpu_reset_counters(grhd2_gpu *h) {
  if (!h) return GRHD2_ERR_ARG;
  CUDA_TRY(h, cudaSetDevice(h->device));
  CUDA_TRY(h, cudaMemsetAsync(h->cnt, 0, NCNT * sizeof(unsigned long long), h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return GRHD2_OK;
}

static int faces_common(grhd2_gpu *h, int n, int dir, const double *qL, const double *qR, const double *alpha,
                        const double *beta, const double *gamma, const double *sqg, double *flux, int physical_only) {
  if (!h || n < 0 || dir < 1 || dir > 3 || !qL || (!physical_only && !qR) || !alpha || !beta || !gamma || !sqg || !flux)
    return fail(h, GRHD2_ERR_ARG, "invalid arguments to the face-flux entry point");
  if (n == 0) return GRHD2_OK;
  CUDA_TRY(h, cudaSetDevice(h->device));
  std::vector<double> T;
  if (int rc = build_face_table(h, T, (size_t)n, dir, alpha, beta, gamma, sqg, {})) return rc;
  double *dT = nullptr, *dq = nullptr;
  int rc;
  if ((rc = dalloc(h, &dT, T.size()))) return rc;
  if ((rc = dalloc(h, &dq, (size_t)15 * n))) { cudaFree(dT); return rc; }
  cudaMemcpy(dT, T.data(), T.size() * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(dq, qL, (size_t)5 * n * sizeof(double), cudaMemcpyHostToDevice);
  if (qR) cudaMemcpy(dq + 5 * n, qR, (size_t)5 * n * sizeof(double), cudaMemcpyHostToDevice);
  if (h->mixed)
    k_riemann_faces<float><<<nblocks(n, 128), 128>>>(h->phys, n, dir, dq, dq + 5 * n, dT, dq + 10 * n, physical_only);
  else
    k_riemann_faces<double><<<nblocks(n, 128), 128>>>(h->phys, n, dir, dq, dq + 5 * n, dT, dq + 10 * n, physical_only);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(flux, dq + 10 * n, (size_t)5 * n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(dT);
  cudaFree(dq);
  if (e != cudaSuccess) return fail(h, GRHD2_ERR_CUDA, "face-flux kernel: %s", cudaGetErrorString(e));
  return GRHD2_OK;
}

int grhd2_gpu_riemann_faces(grhd2_gpu *h, int n, int dir, const double *qL, const double *qR, const double *alpha,
                            const double *beta, const double *gamma, const double *sqg, double *flux) {
  return faces_common(h, n, dir, qL, qR, alpha, beta, gamma, sqg, flux, 0);
}

int grhd2_gpu_physical_flux(grhd2_gpu *h, int n, int dir, const double *q, const double *alpha, const double *beta,
                            const double *gamma, const double *sqg, double *flux) {
  return faces_common(h, n, dir, q, nullptr, alpha, beta, gamma, sqg, flux, 1);
}

int grhd2_gpu_get_stream(grhd2_gpu *h, void **stream_out) {
  if (!h || !stream_out) return GRHD2_ERR_ARG;
  *stream_out = (void *)h->stream;
  return GRHD2_OK;
}

int grhd2_gpu_profile_step(grhd2_gpu *h, double dt, float *ms, const char **names, int cap, int *n_out) {
  if (int rc = ready(h, true)) return rc;
  cudaEvent_t start;
  CUDA_TRY(h, cudaEventCreate(&start));
  CUDA_TRY(h, cudaEventRecord(start, h->stream));
  h->profiling = true;
  int rc = step_dispatch(h, dt);
  h->profiling = false;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  const int n = (int)h->prof_ev.size();
  for (int k = 0; k < n; ++k) {
    float t = 0.0f;
    cudaEventElapsedTime(&t, k == 0 ? start : h->prof_ev[k - 1], h->prof_ev[k]);
    if (k < cap) {
      if (ms) ms[k] = t;
      if (names) names[k] = h->prof_names[k];
    }
  }
  for (auto ev : h->prof_ev) cudaEventDestroy(ev);
  cudaEventDestroy(start);
  h->prof_ev.clear();
  h->prof_names.clear();
  if (n_out) *n_out = n;
  if (rc) return rc;
  if (e != cudaSuccess) return fail(h, GRHD2_ERR_CUDA, "profile step: %s", cudaGetErrorString(e));
  return GRHD2_OK;
}

int grhd2_gpu_synchronize(grhd2_gpu *h) {
  if (!h) return GRHD2_ERR_ARG;
  CUDA_TRY(h, cudaSetDevice(h->device));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return GRHD2_OK;
}

const char *grhd2_gpu_last_error(const grhd2_gpu *h) { return h ? h->err.c_str() : "NULL handle"; }

void grhd2_gpu_destroy(grhd2_gpu *h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  void *bufs[] = {h->P, h->U, h->UP, h->RHS, h->F[0], h->F[1], h->F[2], h->centre, h->face[0], h->face[1], h->face[2],
                  h->inj, h->dust, h->xc, h->frozen[0], h->frozen[1], h->frozen[2], h->cnt, h->red, h->staging};
  for (void *b : bufs) if (b) cudaFree(b);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

}  // extern "C"
