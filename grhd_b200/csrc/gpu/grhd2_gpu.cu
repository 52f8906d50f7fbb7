// grhd2_gpu.cu -- C-ABI of the B200 per-stage path (include/grhd2_gpu.h).
//
// One handle = one grid on one device and CUDA stream.  Device state of a grid:
//   P      primitives, SoA interior planes (double, or float under the mixed policy)
//   U, UP  conserved u and up of grhd2.f90:232-249, SoA interior planes (double)
//   Q      interface states q_L, q_R of the direction being processed
//   F[d]   face fluxes of direction d
//   tables k-invariant metric tables per (i,j) and per face (state.cuh)
//   clock  t, final time, CFL dt, step count (state.cuh GridClock)
// A step is, three times: for each active direction recon + riemann, then cell_update
// (RHS, RK stage, con2prim; stage 1 also performs u = up); then the clocks advance.
// Ghost cells are evaluated on load (state.cuh), so no boundary pass runs.
//
// Every stage launch is batched: a device array of grid descriptors plus a block map
// (grid, first item) per kernel kind.  A handle steps as a batch of one; a
// grhd2_gpu_batch steps many grids with one launch per kernel kind and scheme group, and
// can replay the whole step as one CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <new>
#include <string>
#include <vector>

#include "grhd2_gpu.h"
#include "flux_launch.h"
#include "frame.h"
#include "diag.cuh"
#include "kernels.cuh"
#include "metric_build.cuh"

using namespace grhd;

namespace {

int vfail(std::string &err, int code, const char *fmt, va_list ap) {
  char buf[512];
  vsnprintf(buf, sizeof buf, fmt, ap);
  err = buf;
  return code;
}

// kernel kinds of a step and their items-per-block
enum Kind {
  K_RECON_X = 0, K_RIEMANN_X, K_RECON_Y, K_RIEMANN_Y, K_RECON_Z, K_RIEMANN_Z, K_CELL, K_FLUX_X, K_FLUX_Y, K_FLUX_Z,
  K_STAGE, NKIND
};
const int KIND_BS[NKIND] = {RECON_BS, RIEMANN_BS, RECON_BS, RIEMANN_BS, RECON_BS, RIEMANN_BS, CELL_BS,
                            FUSED_FLUX_BS, FUSED_FLUX_BS, FUSED_FLUX_BS, STAGE_BLOCK};
const char *KIND_NAME[NKIND] = {"recon_x", "riemann_x", "recon_y", "riemann_y", "recon_z", "riemann_z",
                                "cell_update", "flux_x", "flux_y", "flux_z", "stage"};

// ---- block tiles ------------------------------------------------------------------------
unsigned ilog2(unsigned x) {
  unsigned l = 0;
  while ((1u << (l + 1)) <= x) ++l;
  return l;
}
// extents of the index space of a tile kind (cells, or faces of direction dir)
void space_of(const GridDev &G, int dir, unsigned &nI, unsigned &nJ, unsigned &nK) {
  nI = (unsigned)G.nx + (dir == 1); nJ = (unsigned)G.ny + (dir == 2); nK = (unsigned)G.nz + (dir == 3);
}
// tile of 2^lb threads: tx along i (the whole block for 1D grids), the rest along k, or
// along j when the grid has no k extent
Tile make_tile(unsigned nI, unsigned nJ, unsigned nK, unsigned lb, unsigned tx) {
  Tile T;
  T.lx = std::min(ilog2(std::max(tx, 1u)), lb);
  if (nJ == 1 && nK == 1) T.lx = lb;
  T.ly = nK == 1 ? lb - T.lx : 0;
  T.nti = make_fastdiv((nI + (1u << T.lx) - 1) >> T.lx);
  T.ntj = make_fastdiv((nJ + (1u << T.ly) - 1) >> T.ly);
  return T;
}
long long tile_count(const Tile &T, unsigned lb, unsigned nK) {
  const unsigned lz = lb - T.lx - T.ly;
  return (long long)T.nti.d * T.ntj.d * ((nK + (1u << lz) - 1) >> lz);
}
constexpr unsigned LB_RECON = 8, LB_FACE = 7, LB_CELL = 7;  // log2 of RECON_BS, RIEMANN_BS = FUSED_FLUX_BS, CELL_BS
static_assert((1 << LB_RECON) == RECON_BS && (1 << LB_FACE) == RIEMANN_BS && (1 << LB_FACE) == FUSED_FLUX_BS &&
                  (1 << LB_CELL) == CELL_BS, "block sizes are the tile sizes");
constexpr unsigned DEFAULT_TX = 32;

void set_face_tiles(GridDev &G, int dir, unsigned tx) {
  unsigned nI, nJ, nK;
  space_of(G, dir, nI, nJ, nK);
  G.tiles[TILE_RECON + dir - 1] = make_tile(nI, nJ, nK, LB_RECON, tx);
  G.tiles[TILE_FACE + dir - 1] = make_tile(nI, nJ, nK, LB_FACE, tx);
}
void set_cell_tile(GridDev &G, unsigned tx) {
  G.tiles[TILE_CELL] = make_tile((unsigned)G.nx, (unsigned)G.ny, (unsigned)G.nz, LB_CELL, tx);
}

bool dir_active(const GridDev &G, int dir) { return !((dir == 2 && G.ny == 1) || (dir == 3 && G.nz == 1)); }
long long face_count(const GridDev &G, int dir) {
  unsigned nI, nJ, nK;
  space_of(G, dir, nI, nJ, nK);
  return (long long)nI * nJ * nK;
}

// Tile shape of the stage kernel (stage.cuh) for a grid: 0 for a 1D grid (tiles of 256
// cells along i), 2 for an x-y grid and 3 for an x-z grid (tiles of 32 x 8 cells); -1 for a
// 3D grid, which the stage kernel does not cover.
int stage_sd_of(int ny, int nz) { return ny == 1 ? (nz == 1 ? 0 : 3) : (nz == 1 ? 2 : -1); }
int stage_sd(const GridDev &G) { return stage_sd_of(G.ny, G.nz); }
long long stage_tiles(const GridDev &G) {
  const int sd = stage_sd(G);
  if (sd < 0) return 0;
  const int tx = sd == 0 ? STAGE_TILE_CELLS : 32, tr = sd == 0 ? 1 : STAGE_TILE_CELLS / 32;
  const int nr = sd == 2 ? G.ny : (sd == 3 ? G.nz : 1);
  return (long long)((G.nx + tx - 1) / tx) * ((nr + tr - 1) / tr);
}

// threads (tiles x block size) a kernel kind launches for one grid
long long kind_items(const GridDev &G, int k) {
  if (k == K_CELL) return tile_count(G.tiles[TILE_CELL], LB_CELL, (unsigned)G.nz) * CELL_BS;
  if (k == K_STAGE) return stage_tiles(G) * STAGE_BLOCK;
  const int dir = k >= K_FLUX_X ? k - K_FLUX_X + 1 : k / 2 + 1;
  if (!dir_active(G, dir)) return 0;
  unsigned nI, nJ, nK;
  space_of(G, dir, nI, nJ, nK);
  if (k < K_CELL && (k % 2) == 0) return tile_count(G.tiles[TILE_RECON + dir - 1], LB_RECON, nK) * RECON_BS;
  return tile_count(G.tiles[TILE_FACE + dir - 1], LB_FACE, nK) * RIEMANN_BS;
}

inline unsigned nblocks(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }
bool bit_equal(double a, double b) { return std::memcmp(&a, &b, sizeof a) == 0; }

}  // namespace

struct grhd2_gpu_batch;

struct grhd2_gpu {
  grhd2_gpu_config cfg{};
  GridDev G{};  // host copy of the device descriptor (device pointers inside)
  int device = 0;
  bool mixed = false, own_stream = false;
  cudaStream_t stream = nullptr;
  // owned device buffers (their addresses are also in G)
  double *centre = nullptr, *face[3] = {nullptr, nullptr, nullptr};
  float *centre_f = nullptr, *face_f[3] = {nullptr, nullptr, nullptr};  // mixed policy only
  double *inj = nullptr, *dust = nullptr, *xc = nullptr, *frozen[3] = {nullptr, nullptr, nullptr};
  unsigned long long *red = nullptr;
  double *staging = nullptr;
  char *diag = nullptr;  // diagnostics scratch: block partials, results, per-k sums
  double *vtk = nullptr;  // VTK cell fields (big-endian) and radial scale factors
  // checkpoint snapshot: up in the reference layout, copied out on its own stream
  double *snap = nullptr;
  cudaStream_t snap_stream = nullptr;
  cudaEvent_t snap_taken = nullptr, snap_done = nullptr;
  bool snap_pending = false;
  bool u_valid = false;  // u has been written by a step (the mass monitor sums u)
  size_t n_ghosted = 0, n_interior = 0;
  GridClock hclock{};  // host mirror of the device clock
  int version = 0;     // bumped whenever G changes (batches refresh their device copies)
  bool metric_set = false, bc_set = false, prims_set = false, cons_set = false;
  double dt_cache = 0.0;
  bool dt_valid = false;
  grhd2_gpu_batch *self = nullptr;  // batch of one used by step/run/calc_rhs
  std::string err;
};

struct Group {
  bool mixed;
  int rec, rs;
  int sd;  // stage-kernel tile shape of the members (stage_sd_of; -1: 3D grids)
  std::vector<int> members;
  BlockMap *d_map = nullptr;
  int off[NKIND], nb[NKIND];
  int variant[3];  // per direction: GRHD2_FLUX_SPLIT or GRHD2_FLUX_FUSED
  unsigned tx[3];  // per direction: tile extent along i of the face kernels
  // persistent step kernel: member list and the item segments of its two phases
  int *d_members = nullptr;
  Segment *d_seg = nullptr;  // face segments, then cell segments
  int nseg_face = 0, nseg_cell = 0;
  long long n_face = 0, n_cell = 0;
  int max_blocks = 0;  // resident blocks of the group's persistent instantiation
  int max_blocks_stage = 0;  // resident blocks of its persistent stage kernel (stage groups of 1D grids)
  int cell_dirs = 1;   // the most active directions of a member grid (cell kernel staging)
  bool stage = false;  // steps run the stage kernel (one launch per stage) instead of face and cell kernels
};

struct FluxChoice {
  int variant;
  unsigned tx;
};

struct grhd2_gpu_batch {
  std::vector<grhd2_gpu *> m;
  std::vector<int> versions;
  int device = 0;
  cudaStream_t stream = nullptr;
  GridDev *d_grids = nullptr;
  GridClock *d_clocks = nullptr;  // gathered clocks of every member (grhd2_gpu_batch_clocks)
  std::vector<Group> groups;
  int variant_request = GRHD2_FLUX_AUTO;  // GRHD2_FLUX_AUTO: tuned choice if cached, else the default
  int stage_request = GRHD2_STAGE_AUTO;   // the stage kernel for groups of 1D and 2D grids
  unsigned tile_request = 0;              // 0: tuned tile if cached, else DEFAULT_TX
  int step_request = GRHD2_STEP_AUTO;     // stage kernels in a graph, or the persistent kernel
  bool persistent = false;                // the mode in use
  unsigned *d_bar = nullptr;              // persistent kernel barrier words and status
  std::map<std::pair<int, int>, FluxChoice> forced;  // (group, direction) -> choice, while tuning
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // a captured step runs the scheme groups as parallel branches of its graph: group 0 on
  // the batch stream, group g on lanes[g - 1] (forked from and joined back into it)
  std::vector<cudaStream_t> lanes;
  std::vector<cudaEvent_t> lane_done;
  cudaEvent_t fork = nullptr;
  bool profiling = false;
  std::vector<cudaEvent_t> prof_ev;
  std::vector<const char *> prof_names;
  std::string err;
};

namespace {

int fail(grhd2_gpu *h, int code, const char *fmt, ...) {
  if (!h) return code;
  va_list ap;
  va_start(ap, fmt);
  vfail(h->err, code, fmt, ap);
  va_end(ap);
  return code;
}
int bfail(grhd2_gpu_batch *b, int code, const char *fmt, ...) {
  if (!b) return code;
  va_list ap;
  va_start(ap, fmt);
  vfail(b->err, code, fmt, ap);
  va_end(ap);
  return code;
}

#define CUDA_TRY(h, call)                                                                             \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) return fail((h), GRHD2_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)
#define BCUDA_TRY(b, call)                                                                             \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess) return bfail((b), GRHD2_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

// Handle buffers come from the device's stream-ordered memory pool, allocated and freed
// in the order of the handle's stream: creating and destroying grids (a solve server does
// this all the time) neither synchronises the device nor returns memory to the driver.
// The pool keeps up to POOL_KEEP_BYTES of freed memory for reuse.  Every entry point that
// allocates synchronises the handle's stream before it returns, so the buffers are ready
// for any stream afterwards.
constexpr unsigned long long POOL_KEEP_BYTES = 8ull << 30;
static void keep_pool_memory(int device) {
  static std::mutex mu;
  static std::vector<int> done;
  std::lock_guard<std::mutex> lock(mu);
  if (std::find(done.begin(), done.end(), device) != done.end()) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    unsigned long long keep = POOL_KEEP_BYTES;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  done.push_back(device);
}

template <class T>
int dalloc(grhd2_gpu *h, T **p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMallocAsync((void **)p, n * sizeof(T), h->stream);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(h, GRHD2_ERR_NOMEM, "cudaMallocAsync(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
  }
  return 0;
}

int launch_check(grhd2_gpu *h) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(h, GRHD2_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
  return 0;
}
int blaunch_check(grhd2_gpu_batch *b, const char *name) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return bfail(b, GRHD2_ERR_CUDA, "kernel launch (%s): %s", name, cudaGetErrorString(e));
  if (b->profiling) {
    cudaEvent_t ev;
    if (cudaEventCreate(&ev) != cudaSuccess) return bfail(b, GRHD2_ERR_CUDA, "cudaEventCreate failed");
    cudaEventRecord(ev, b->stream);
    b->prof_ev.push_back(ev);
    b->prof_names.push_back(name);
  }
  return 0;
}

// Descriptor buffers of a batch live in the stream-ordered pool too, released in the
// order of the batch's stream: a rebuild (grids joining or leaving) frees the old ones
// after the steps already enqueued and never synchronises the device.
void destroy_batch_resources(grhd2_gpu_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  auto release = [b](void *p) { if (p) cudaFreeAsync(p, b->stream); };
  for (auto &g : b->groups) {
    release(g.d_map);
    release(g.d_members);
    release(g.d_seg);
  }
  release(b->d_bar);
  b->d_bar = nullptr;
  b->groups.clear();
  release(b->d_grids);
  b->d_grids = nullptr;
  release(b->d_clocks);
  b->d_clocks = nullptr;
}

// ---- flux variant choice --------------------------------------------------------------
// Tuned choices are cached per process, keyed by what decides the winner: precision,
// scheme, Riemann solver, shock sensor, direction and the size class of the launch
// (log2 of the faces in the group).
struct TuneKey {
  int mixed, rec, rs, sensor, dir, size_class;
  bool operator<(const TuneKey &o) const {
    return std::tie(mixed, rec, rs, sensor, dir, size_class) <
           std::tie(o.mixed, o.rec, o.rs, o.sensor, o.dir, o.size_class);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, FluxChoice> g_tune;

TuneKey tune_key(const Group &grp, const std::vector<GridDev> &hg, int dir) {
  long long faces = 0;
  for (int g : grp.members) faces += face_count(hg[g], dir);
  int cls = 0;
  while ((1LL << (cls + 1)) <= faces) ++cls;
  return TuneKey{grp.mixed ? 1 : 0, grp.rec, grp.rs, hg[grp.members[0]].phys.sensor, dir, cls};
}

// default without tuning: the split kernels (recon at high occupancy, lean Riemann)
constexpr int DEFAULT_VARIANT = GRHD2_FLUX_SPLIT;
constexpr long long SPLIT_VAR_BELOW_FACES = 4LL * 148 * 4 * RECON_BS;  // four waves of per-face blocks
// Automatic step mode: the graph of stage kernels.  Measured on one B200 with 1024-cell 1D
// grids, a graph replay takes 83-88 us per step and the persistent kernel 127-135 us: a
// small grid is bound by the dependent arithmetic chain of one item per thread, not by
// launch latency (graph replays hide the gaps), and the persistent kernel's fused face
// phase reconstructs the five variables of a face in one thread, one after the other.

FluxChoice choose_flux(const grhd2_gpu_batch *b, int gi, const Group &grp, const std::vector<GridDev> &hg, int dir) {
  auto f = b->forced.find({gi, dir});
  if (f != b->forced.end()) return f->second;
  // untuned: one thread per (face, variable) for launches that one thread per face would
  // leave short of the resident threads of the GPU
  long long faces = 0;
  for (int g : grp.members) faces += face_count(hg[g], dir);
  FluxChoice c{faces < SPLIT_VAR_BELOW_FACES ? GRHD2_FLUX_SPLIT_VAR : DEFAULT_VARIANT, DEFAULT_TX};
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find(tune_key(grp, hg, dir));
    if (it != g_tune.end()) c = it->second;
  }
  if (b->variant_request != GRHD2_FLUX_AUTO) c.variant = b->variant_request;
  if (b->tile_request > 0) c.tx = b->tile_request;
  return c;
}

// Whether a group's steps run the stage kernel: its grids are 1D or 2D and the request
// asks for it; AUTO takes it for 1D grids.  Measured on one B200 (the face and cell kernels
// autotuned or forced to the tuned variant): 64 Michel grids of 1024 cells (MP5 + HLLE,
// FP64) 5.85e8 zone-updates/s against 4.50e8; 32 tori of 400 x 1 x 200 (WENO5 + HLLE)
// 5.86e8 against 7.29e8 in FP64 and 1.57e9 against 1.68e9 mixed.  On a 2D tile the stage
// kernel computes 552 faces for 256 cells (the split kernels 514) at 27 resident warps
// per SM; on a 1D tile 257 faces, and it saves the launches and the interface-state and
// flux round trips that dominate small grids.
bool use_stage(const grhd2_gpu_batch *b, const Group &grp) {
  if (grp.sd < 0 || b->stage_request == GRHD2_STAGE_OFF) return false;
  return b->stage_request == GRHD2_STAGE_ON || grp.sd == 0;
}

// A scheme group of at least SPLIT_GROUP_CELLS cells over two or more grids runs as two
// groups of about half the cells each, which a captured step runs as parallel branches of
// its graph: each half's interface states stay closer to L2 and one half's kernel tails
// overlap the other's work.  Measured on 32 tori of 400x1x200 run as 1, 2, 4 or 8
// independent parts on parallel streams: two parts fastest (mixed +3.9 %, FP64 +0.9 %).
constexpr long long SPLIT_GROUP_CELLS = 2000000;
void split_large_groups(grhd2_gpu_batch *b, const std::vector<GridDev> &hg) {
  std::vector<Group> out;
  for (const Group &grp : b->groups) {
    long long cells = 0;
    for (int g : grp.members) cells += hg[g].ncell;
    if (grp.members.size() < 2 || cells < SPLIT_GROUP_CELLS) {
      out.push_back(grp);
      continue;
    }
    Group lo = grp, hi = grp;
    lo.members.clear();
    hi.members.clear();
    long long acc = 0;
    for (int g : grp.members) {  // the first half takes grids until it holds half the cells
      const bool first = lo.members.empty() || (acc < cells / 2 && grp.members.back() != g);
      (first ? lo : hi).members.push_back(g);
      if (first) acc += hg[g].ncell;
    }
    out.push_back(lo);
    out.push_back(hi);
  }
  b->groups.swap(out);
}

// (re)build device descriptors and block maps of a batch
int build_batch(grhd2_gpu_batch *b) {
  destroy_batch_resources(b);
  const int n = (int)b->m.size();
  std::vector<GridDev> hg(n);
  b->versions.resize(n);
  for (int g = 0; g < n; ++g) { hg[g] = b->m[g]->G; b->versions[g] = b->m[g]->version; }
  for (int g = 0; g < n; ++g) {
    const grhd2_gpu *h = b->m[g];
    Group *grp = nullptr;
    const int sd = stage_sd_of(h->cfg.ny, h->cfg.nz);
    for (auto &x : b->groups)
      if (x.mixed == h->mixed && x.rec == h->cfg.rec_method && x.rs == h->cfg.riemann && x.sd == sd) grp = &x;
    if (!grp) {
      b->groups.push_back(Group{h->mixed, h->cfg.rec_method, h->cfg.riemann, sd, {}, nullptr, {}, {}, {0, 0, 0},
                                {DEFAULT_TX, DEFAULT_TX, DEFAULT_TX}});
      grp = &b->groups.back();
    }
    grp->members.push_back(g);
    grp->cell_dirs = std::max(grp->cell_dirs, 1 + (h->cfg.ny > 1 ? 1 : 0) + (h->cfg.nz > 1 ? 1 : 0));
  }
  split_large_groups(b, hg);
  // flux variant and tile per scheme group and direction; the tiles go into the batch's
  // copies of the descriptors
  for (int gi = 0; gi < (int)b->groups.size(); ++gi) {
    Group &grp = b->groups[gi];
    for (int d = 1; d <= 3; ++d) {
      const FluxChoice ch = choose_flux(b, gi, grp, hg, d);
      grp.variant[d - 1] = ch.variant;
      grp.tx[d - 1] = ch.tx;
      for (int g : grp.members) set_face_tiles(hg[g], d, ch.tx);
    }
    grp.stage = use_stage(b, grp);
    if (grp.stage) {
      cudaError_t e = grp.mixed ? stage_setup<float, float>(grp.sd, grp.rec, grp.rs)
                                : stage_setup<double, double>(grp.sd, grp.rec, grp.rs);
      if (e != cudaSuccess) return bfail(b, GRHD2_ERR_CUDA, "stage kernel set-up: %s", cudaGetErrorString(e));
    }
  }
  BCUDA_TRY(b, cudaMallocAsync((void **)&b->d_grids, sizeof(GridDev) * n, b->stream));
  BCUDA_TRY(b, cudaMallocAsync((void **)&b->d_clocks, sizeof(GridClock) * n, b->stream));
  BCUDA_TRY(b, cudaMemcpyAsync(b->d_grids, hg.data(), sizeof(GridDev) * n, cudaMemcpyHostToDevice, b->stream));
  for (auto &grp : b->groups) {
    std::vector<BlockMap> map;
    for (int k = 0; k < NKIND; ++k) {
      grp.off[k] = (int)map.size();
      for (int g : grp.members) {
        const long long items = kind_items(hg[g], k);
        for (long long first = 0; first < items; first += KIND_BS[k]) map.push_back(BlockMap{g, (int)first});
      }
      grp.nb[k] = (int)map.size() - grp.off[k];
    }
    BCUDA_TRY(b, cudaMallocAsync((void **)&grp.d_map, sizeof(BlockMap) * std::max<size_t>(1, map.size()), b->stream));
    BCUDA_TRY(b, cudaMemcpyAsync(grp.d_map, map.data(), sizeof(BlockMap) * map.size(), cudaMemcpyHostToDevice, b->stream));
    // persistent kernel: flattened item spaces (faces of every active direction; cells)
    std::vector<Segment> seg;
    long long first = 0;
    for (int g : grp.members)
      for (int d = 1; d <= 3; ++d)
        if (dir_active(hg[g], d)) {
          seg.push_back(Segment{g, d, first, face_count(hg[g], d)});
          first += face_count(hg[g], d);
        }
    grp.nseg_face = (int)seg.size();
    grp.n_face = first;
    first = 0;
    for (int g : grp.members) {
      seg.push_back(Segment{g, 0, first, hg[g].ncell});
      first += hg[g].ncell;
    }
    grp.nseg_cell = (int)seg.size() - grp.nseg_face;
    grp.n_cell = first;
    BCUDA_TRY(b, cudaMallocAsync((void **)&grp.d_seg, sizeof(Segment) * seg.size(), b->stream));
    BCUDA_TRY(b, cudaMemcpyAsync(grp.d_seg, seg.data(), sizeof(Segment) * seg.size(), cudaMemcpyHostToDevice, b->stream));
    BCUDA_TRY(b, cudaMallocAsync((void **)&grp.d_members, sizeof(int) * grp.members.size(), b->stream));
    BCUDA_TRY(b, cudaMemcpyAsync(grp.d_members, grp.members.data(), sizeof(int) * grp.members.size(),
                                 cudaMemcpyHostToDevice, b->stream));
    cudaError_t e = grp.mixed ? run_persistent<float, float>(grp.rec, grp.rs, true, &grp.max_blocks, {}, 0, 0, b->stream)
                              : run_persistent<double, double>(grp.rec, grp.rs, true, &grp.max_blocks, {}, 0, 0, b->stream);
    if (e != cudaSuccess) return bfail(b, GRHD2_ERR_CUDA, "persistent kernel occupancy: %s", cudaGetErrorString(e));
    if (grp.stage && grp.sd == 0) {
      e = grp.mixed ? run_persistent_stage<float, float>(grp.rec, grp.rs, true, &grp.max_blocks_stage, {}, 0, 0, b->stream)
                    : run_persistent_stage<double, double>(grp.rec, grp.rs, true, &grp.max_blocks_stage, {}, 0, 0,
                                                           b->stream);
      if (e != cudaSuccess) return bfail(b, GRHD2_ERR_CUDA, "persistent stage kernel occupancy: %s", cudaGetErrorString(e));
    }
  }
  BCUDA_TRY(b, cudaMallocAsync((void **)&b->d_bar, 4 * sizeof(unsigned), b->stream));
  BCUDA_TRY(b, cudaMemsetAsync(b->d_bar, 0, 4 * sizeof(unsigned), b->stream));
  // step mode
  b->persistent = b->step_request == GRHD2_STEP_PERSISTENT;
  if (b->persistent)
    for (const auto &grp : b->groups)
      if (grp.max_blocks <= 0 || (grp.stage && grp.sd == 0 && grp.max_blocks_stage <= 0))
        return bfail(b, GRHD2_ERR_CUDA, "the persistent step kernel cannot be resident");
  BCUDA_TRY(b, cudaStreamSynchronize(b->stream));  // host vectors go out of scope
  return 0;
}

int refresh_batch(grhd2_gpu_batch *b) {
  for (size_t g = 0; g < b->m.size(); ++g)
    if (b->versions[g] != b->m[g]->version) return build_batch(b);
  return 0;
}

// kind 0..5 for directions, then the cell kernel in MODE (0 rhs, 1..3 stages)
template <class R, class PT>
int enqueue_dir(grhd2_gpu_batch *b, const Group &grp, int d, int variant, cudaStream_t st) {
  const int kr = 2 * (d - 1), ks = kr + 1, kf = K_FLUX_X + d - 1;
  if (variant == GRHD2_FLUX_FUSED) {
    if (grp.nb[kf] > 0) {
      launch_flux<R, PT>(d, grp.rec, grp.rs, b->d_grids, grp.d_map + grp.off[kf], grp.nb[kf], st);
      if (int rc = blaunch_check(b, KIND_NAME[kf])) return rc;
    }
    return 0;
  }
  if (grp.nb[kr] > 0) {
    launch_recon<R, PT>(d, grp.rec, variant == GRHD2_FLUX_SPLIT_VAR, b->d_grids, grp.d_map + grp.off[kr], grp.nb[kr], st);
    if (int rc = blaunch_check(b, KIND_NAME[kr])) return rc;
  }
  if (grp.nb[ks] > 0) {
    launch_riemann<R>(d, grp.rs, b->d_grids, grp.d_map + grp.off[ks], grp.nb[ks], st);
    if (int rc = blaunch_check(b, KIND_NAME[ks])) return rc;
  }
  return 0;
}

template <class R, class PT>
int enqueue_fluxes(grhd2_gpu_batch *b, const Group &grp, cudaStream_t st) {
  for (int d = 1; d <= 3; ++d)
    if (int rc = enqueue_dir<R, PT>(b, grp, d, grp.variant[d - 1], st)) return rc;
  return 0;
}

template <int MODE, class R, class PT>
int enqueue_cells(grhd2_gpu_batch *b, const Group &grp, cudaStream_t st) {
  if (grp.nb[K_CELL] <= 0) return 0;
  launch_cell<R, PT>(MODE, b->d_grids, grp.d_map + grp.off[K_CELL], grp.nb[K_CELL], grp.cell_dirs, st);
  return blaunch_check(b, MODE == 0 ? "cell_rhs" : "cell_update");
}

// the three SSP-RK3 stages of one scheme group (its grids depend on no other group's)
int enqueue_group_step(grhd2_gpu_batch *b, const Group &grp, cudaStream_t st) {
  int rc;
  if (grp.stage) {
    if (grp.nb[K_STAGE] <= 0) return 0;
    for (int mode = 1; mode <= 3; ++mode) {
      if (grp.mixed)
        launch_stage<float, float>(grp.sd, grp.rec, grp.rs, mode, b->d_grids, grp.d_map + grp.off[K_STAGE],
                                   grp.nb[K_STAGE], st);
      else
        launch_stage<double, double>(grp.sd, grp.rec, grp.rs, mode, b->d_grids, grp.d_map + grp.off[K_STAGE],
                                     grp.nb[K_STAGE], st);
      if ((rc = blaunch_check(b, KIND_NAME[K_STAGE]))) return rc;
    }
    return 0;
  }
  if (grp.mixed) {
    if ((rc = enqueue_fluxes<float, float>(b, grp, st)) || (rc = enqueue_cells<1, float, float>(b, grp, st)) ||
        (rc = enqueue_fluxes<float, float>(b, grp, st)) || (rc = enqueue_cells<2, float, float>(b, grp, st)) ||
        (rc = enqueue_fluxes<float, float>(b, grp, st)) || (rc = enqueue_cells<3, float, float>(b, grp, st)))
      return rc;
  } else {
    if ((rc = enqueue_fluxes<double, double>(b, grp, st)) || (rc = enqueue_cells<1, double, double>(b, grp, st)) ||
        (rc = enqueue_fluxes<double, double>(b, grp, st)) || (rc = enqueue_cells<2, double, double>(b, grp, st)) ||
        (rc = enqueue_fluxes<double, double>(b, grp, st)) || (rc = enqueue_cells<3, double, double>(b, grp, st)))
      return rc;
  }
  return 0;
}

// streams and events for the branches of a captured step (created before the capture)
int ensure_lanes(grhd2_gpu_batch *b) {
  const size_t need = b->groups.empty() ? 0 : b->groups.size() - 1;
  if (need > 0 && !b->fork) BCUDA_TRY(b, cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
  while (b->lanes.size() < need) {
    cudaStream_t s;
    cudaEvent_t e;
    BCUDA_TRY(b, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    b->lanes.push_back(s);
    BCUDA_TRY(b, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->lane_done.push_back(e);
  }
  return 0;
}

void destroy_lanes(grhd2_gpu_batch *b) {
  for (cudaStream_t s : b->lanes) cudaStreamDestroy(s);
  for (cudaEvent_t e : b->lane_done) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  b->lanes.clear();
  b->lane_done.clear();
  b->fork = nullptr;
}

// One step of every grid.  branches: the scheme groups fork off the batch stream and join
// before the clocks advance (used while capturing the step's graph, where the groups
// become parallel branches); otherwise they run one after another on the batch stream.
int enqueue_step(grhd2_gpu_batch *b, bool branches = false) {
  const int ng = (int)b->groups.size();
  branches = branches && ng > 1 && (int)b->lanes.size() >= ng - 1;
  if (branches) {
    BCUDA_TRY(b, cudaEventRecord(b->fork, b->stream));
    for (int g = 1; g < ng; ++g) BCUDA_TRY(b, cudaStreamWaitEvent(b->lanes[g - 1], b->fork, 0));
  }
  for (int g = 0; g < ng; ++g)
    if (int rc = enqueue_group_step(b, b->groups[g], branches && g > 0 ? b->lanes[g - 1] : b->stream)) return rc;
  if (branches)
    for (int g = 1; g < ng; ++g) {
      BCUDA_TRY(b, cudaEventRecord(b->lane_done[g - 1], b->lanes[g - 1]));
      BCUDA_TRY(b, cudaStreamWaitEvent(b->stream, b->lane_done[g - 1], 0));
    }
  const int n = (int)b->m.size();
  k_advance_clocks<<<nblocks(n, 128), 128, 0, b->stream>>>(b->d_grids, n);
  return blaunch_check(b, "advance_clocks");
}

// nsteps whole steps of every scheme group, each group one cooperative launch of the
// persistent kernel (groups run one after the other on the batch stream)
int enqueue_persistent(grhd2_gpu_batch *b, long long nsteps) {
  for (const auto &grp : b->groups) {
    if (grp.stage && grp.sd == 0) {  // 1D grids: the persistent form of the stage kernel
      if (grp.nb[K_STAGE] <= 0) continue;
      const PersistentStageArgs a{b->d_grids, grp.d_map + grp.off[K_STAGE], grp.nb[K_STAGE], grp.d_members,
                                  (int)grp.members.size(), b->d_bar, b->d_bar + 2};
      const int blocks = std::max(1, std::min(grp.max_blocks_stage, grp.nb[K_STAGE]));
      for (long long done = 0; done < nsteps;) {
        const int chunk = (int)std::min<long long>(nsteps - done, 1 << 30);
        BCUDA_TRY(b, cudaMemsetAsync(b->d_bar, 0, 2 * sizeof(unsigned), b->stream));  // arrivals, generation
        cudaError_t e = grp.mixed ? run_persistent_stage<float, float>(grp.rec, grp.rs, false, nullptr, a, chunk, blocks, b->stream)
                                  : run_persistent_stage<double, double>(grp.rec, grp.rs, false, nullptr, a, chunk, blocks,
                                                                         b->stream);
        if (e != cudaSuccess) return bfail(b, GRHD2_ERR_CUDA, "persistent stage kernel launch: %s", cudaGetErrorString(e));
        if (int rc = blaunch_check(b, "persistent_stage")) return rc;
        done += chunk;
      }
      continue;
    }
    const PersistentArgs a{b->d_grids, grp.d_members, (int)grp.members.size(), grp.d_seg, grp.nseg_face, grp.n_face,
                           grp.d_seg + grp.nseg_face, grp.nseg_cell, grp.n_cell, b->d_bar, b->d_bar + 2};
    const long long need = std::max(std::max(grp.n_face, grp.n_cell), (long long)grp.members.size());
    const int blocks = (int)std::max(1LL, std::min<long long>(grp.max_blocks, (need + FUSED_FLUX_BS - 1) / FUSED_FLUX_BS));
    for (long long done = 0; done < nsteps;) {
      const int chunk = (int)std::min<long long>(nsteps - done, 1 << 30);
      BCUDA_TRY(b, cudaMemsetAsync(b->d_bar, 0, 2 * sizeof(unsigned), b->stream));  // arrivals, generation
      cudaError_t e = grp.mixed ? run_persistent<float, float>(grp.rec, grp.rs, false, nullptr, a, chunk, blocks, b->stream)
                                : run_persistent<double, double>(grp.rec, grp.rs, false, nullptr, a, chunk, blocks, b->stream);
      if (e != cudaSuccess) return bfail(b, GRHD2_ERR_CUDA, "persistent step kernel launch: %s", cudaGetErrorString(e));
      if (int rc = blaunch_check(b, "persistent_step")) return rc;
      done += chunk;
    }
  }
  return 0;
}

// the persistent kernel's status word (nonzero: a grid barrier timed out); synchronises
int check_persistent(grhd2_gpu_batch *b) {
  if (!b->d_bar) return 0;
  unsigned st = 0;
  BCUDA_TRY(b, cudaMemcpyAsync(&st, b->d_bar + 2, sizeof st, cudaMemcpyDeviceToHost, b->stream));
  BCUDA_TRY(b, cudaStreamSynchronize(b->stream));
  if (st) return bfail(b, GRHD2_ERR_CUDA, "persistent step kernel: a grid barrier timed out (status %u)", st);
  return 0;
}

int batch_steps(grhd2_gpu_batch *b, long long nsteps, bool use_graph) {
  for (size_t g = 0; g < b->m.size(); ++g)
    if (b->m[g]->stream != b->stream)
      return bfail(b, GRHD2_ERR_STATE, "grid %zu moved to another stream after the batch was created", g);
  if (int rc = refresh_batch(b)) return rc;
  if (nsteps <= 0) return 0;
  for (auto *m : b->m) m->u_valid = true;
  if (b->persistent) return enqueue_persistent(b, nsteps);
  if (!use_graph) {
    for (long long s = 0; s < nsteps; ++s)
      if (int rc = enqueue_step(b)) return rc;
    return 0;
  }
  if (!b->exec) {
    if (int rc = ensure_lanes(b)) return rc;
    BCUDA_TRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_step(b, true);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return bfail(b, GRHD2_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    b->graph = g;
    BCUDA_TRY(b, cudaGraphInstantiate(&b->exec, b->graph, 0));
  }
  for (long long s = 0; s < nsteps; ++s) BCUDA_TRY(b, cudaGraphLaunch(b->exec, b->stream));
  return 0;
}

int ready(grhd2_gpu *h, bool need_state) {
  if (!h) return GRHD2_ERR_ARG;
  if (!h->metric_set) return fail(h, GRHD2_ERR_STATE, "metric tables not set (call grhd2_gpu_set_metric or grhd2_gpu_set_metric_analytic first)");
  const int cs = h->cfg.case_id;
  if ((cs == 7 || cs == 8 || cs == 5) && !h->bc_set)
    return fail(h, GRHD2_ERR_STATE, "boundary data not set for case %d (call grhd2_gpu_set_bc_data)", cs);
  if (need_state && !(h->prims_set && h->cons_set)) return fail(h, GRHD2_ERR_STATE, "state not uploaded");
  CUDA_TRY(h, cudaSetDevice(h->device));
  return 0;
}

int self_batch(grhd2_gpu *h) {
  if (h->self) {
    if (int rc = refresh_batch(h->self)) return fail(h, rc, "%s", h->self->err.c_str());
    return 0;
  }
  grhd2_gpu_batch *b = new (std::nothrow) grhd2_gpu_batch();
  if (!b) return fail(h, GRHD2_ERR_NOMEM, "out of host memory");
  b->m.push_back(h);
  b->device = h->device;
  b->stream = h->stream;
  h->self = b;
  if (int rc = build_batch(b)) return fail(h, rc, "%s", b->err.c_str());
  return 0;
}

// The compensated accumulation's carries restart at zero whenever up is written outside a
// step (upload, prim_to_cons, cons_to_prim's floors): the state is then up alone.
int clear_carries(grhd2_gpu *h, cudaStream_t st) {
  if (!h->G.carry) return 0;
  const size_t cb = (h->G.carry == 1 ? sizeof(double) : sizeof(float)) * 5 * (size_t)h->G.pplane;
  CUDA_TRY(h, cudaMemsetAsync(h->G.Uc, 0, cb, st));
  CUDA_TRY(h, cudaMemsetAsync(h->G.UPc, 0, cb, st));
  return 0;
}

int write_clock(grhd2_gpu *h) {
  CUDA_TRY(h, cudaMemcpyAsync(h->G.clock, &h->hclock, sizeof(GridClock), cudaMemcpyHostToDevice, h->stream));
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

int profile_common(grhd2_gpu_batch *b, float *ms, const char **names, int cap, int *n_out) {
  cudaEvent_t start;
  BCUDA_TRY(b, cudaEventCreate(&start));
  BCUDA_TRY(b, cudaEventRecord(start, b->stream));
  b->profiling = true;
  int rc = refresh_batch(b);
  if (!rc) rc = b->persistent ? enqueue_persistent(b, 1) : enqueue_step(b);
  b->profiling = false;
  cudaError_t e = cudaStreamSynchronize(b->stream);
  const int n = (int)b->prof_ev.size();
  for (int k = 0; k < n; ++k) {
    float t = 0.0f;
    cudaEventElapsedTime(&t, k == 0 ? start : b->prof_ev[k - 1], b->prof_ev[k]);
    if (k < cap) {
      if (ms) ms[k] = t;
      if (names) names[k] = b->prof_names[k];
    }
  }
  for (auto ev : b->prof_ev) cudaEventDestroy(ev);
  cudaEventDestroy(start);
  b->prof_ev.clear();
  b->prof_names.clear();
  if (n_out) *n_out = n;
  if (rc) return rc;
  if (e != cudaSuccess) return bfail(b, GRHD2_ERR_CUDA, "profile step: %s", cudaGetErrorString(e));
  return GRHD2_OK;
}

}  // namespace

// diagnostics scratch: DIAG_BLOCKS partials, one result, nz per-plane sums
// diagnostics scratch: DIAG_BLOCKS partials and one result (global), DIAG_BLOCKS + 1 sums,
// nz per-plane sums, 3 (DIAG_BLOCKS + 1) quadrupole sums, coordinate tables nx + 2 ny + 2 nz
size_t diag_bytes(int nx, int ny, int nz) {
  return (size_t)(DIAG_BLOCKS + 1) * sizeof(DiagGlobal) +
         (size_t)(DIAG_BLOCKS + 1 + nz + 3 * (DIAG_BLOCKS + 1) + nx + 2 * ny + 2 * nz) * sizeof(double);
}

// device bytes a handle of this configuration allocates (create + set_metric + set_bc_data;
// the calc_rhs scratch is not counted), each allocation rounded up to 4 KB
long long handle_bytes(const grhd2_gpu_config &c) {
  const long long es = c.precision_policy != GRHD2_PREC_FP64 ? 4 : 8;
  const long long ncell = (long long)c.nx * c.ny * c.nz, pplane = (ncell + 31) / 32 * 32;
  const long long nf[3] = {(long long)(c.nx + 1) * c.ny * c.nz, (long long)c.nx * (c.ny + 1) * c.nz,
                           (long long)c.nx * c.ny * (c.nz + 1)};
  std::vector<long long> a;
  a.push_back(5 * pplane * es);
  if (stage_sd_of(c.ny, c.nz) >= 0) {  // P2, P3 of the stage kernel
    a.push_back(5 * pplane * es);
    a.push_back(5 * pplane * es);
  }
  a.push_back(5 * pplane * 8);
  a.push_back(5 * pplane * 8);
  if (c.precision_policy == GRHD2_PREC_MIXED_COMP64 || c.precision_policy == GRHD2_PREC_MIXED_COMP32) {
    const long long cb = c.precision_policy == GRHD2_PREC_MIXED_COMP64 ? 8 : 4;  // carries of u and up
    a.push_back(5 * pplane * cb);
    a.push_back(5 * pplane * cb);
  }
  long long nq = nf[0];
  for (int d = 0; d < 3; ++d) {
    if ((d == 1 && c.ny == 1) || (d == 2 && c.nz == 1)) continue;
    nq = std::max(nq, nf[d]);
    a.push_back(5 * nf[d] * es);
  }
  a.push_back(10 * nq * es);
  a.push_back(NCNT * 8);
  a.push_back((long long)sizeof(GridClock));
  a.push_back(32);
  a.push_back((long long)diag_bytes(c.nx, c.ny, c.nz));
  a.push_back(5LL * (c.nx + 2 * c.nghost + 1) * (c.ny + 2 * c.nghost + 1) * (c.nz + 2 * c.nghost + 1) * 8);
  if (c.nghost == 2) {
    a.push_back(5LL * c.ny * c.nz * 8);
    a.push_back(5LL * c.nx * c.nz * 8);
    a.push_back(5LL * c.nx * c.ny * 8);
  }
  for (long long tb : {8LL, c.precision_policy != GRHD2_PREC_FP64 ? 4LL : 0LL}) {  // tables (+ FP32 copies)
    if (tb == 0) continue;
    a.push_back((long long)NCF * c.nx * c.ny * tb);
    a.push_back((long long)NFF * (c.nx + 1) * c.ny * tb);
    if (c.ny > 1) a.push_back((long long)NFF * c.nx * (c.ny + 1) * tb);
    if (c.nz > 1) a.push_back((long long)NFF * c.nx * c.ny * tb);
  }
  if (c.case_id == 7) a.push_back(5LL * c.nghost * c.ny * c.nz * 8);
  if (c.case_id == 8) a.push_back(5LL * c.nghost * 8);
  if (c.case_id == 5) a.push_back((long long)(c.nx + 2 * c.nghost + 1) * 8);
  long long tot = 0;
  for (long long x : a) tot += (std::max(x, 1LL) + 4095) / 4096 * 4096;
  return tot;
}

__global__ void k_gather_clocks(const GridDev *__restrict__ grids, int n, GridClock *__restrict__ out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < n) out[g] = *grids[g].clock;
}

// ======================================================================================
extern "C" {

int64_t grhd2_gpu_device_bytes(const grhd2_gpu_config *cfg) {
  if (!cfg || cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1 || cfg->nghost < 1) return -1;
  return handle_bytes(*cfg);
}

int grhd2_gpu_set_stream(grhd2_gpu *h, void *stream) {
  if (!h) return GRHD2_ERR_ARG;
  CUDA_TRY(h, cudaSetDevice(h->device));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (h->self) {  // the batch of one follows the handle; its graph was captured for the old stream
    destroy_batch_resources(h->self);  // released in the old stream's order: before it goes
    destroy_lanes(h->self);
    delete h->self;
    h->self = nullptr;
  }
  if (h->own_stream) CUDA_TRY(h, cudaStreamDestroy(h->stream));
  h->own_stream = false;
  h->stream = nullptr;
  if (stream) {
    h->stream = (cudaStream_t)stream;
  } else {
    CUDA_TRY(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
  }
  return GRHD2_OK;
}

int grhd2_gpu_abi_version(void) { return GRHD2_GPU_ABI_VERSION; }

int grhd2_gpu_create_on_stream(const grhd2_gpu_config *cfg, void *stream, grhd2_gpu **out) {
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
  if (c.precision_policy < GRHD2_PREC_FP64 || c.precision_policy > GRHD2_PREC_MIXED_COMP32)
    return fail(h, GRHD2_ERR_ARG, "invalid precision policy %d", c.precision_policy);
  if (c.case_id == 12 && (c.nz % 2) != 0) return fail(h, GRHD2_ERR_BOUNDARY, "nz must be even for 3D trans-polar boundary conditions");
  if ((c.case_id == 11 || c.case_id == 12) && c.ny < c.nghost)
    return fail(h, GRHD2_ERR_ARG, "reflecting/trans-polar boundaries need ny >= nghost");
  if (c.case_id == 5 && (c.nx < c.nghost || c.nz < c.nghost))
    return fail(h, GRHD2_ERR_ARG, "the jet's reflecting boundaries need nx, nz >= nghost");
  if (!(c.dx > 0) || (c.ny > 1 && !(c.dy > 0)) || (c.nz > 1 && !(c.dz > 0))) return fail(h, GRHD2_ERR_ARG, "grid spacing must be positive");
  if ((long long)(c.nx + 1) * c.ny * c.nz > 2000000000LL || (long long)c.nx * (c.ny + 1) * c.nz > 2000000000LL ||
      (long long)c.nx * c.ny * (c.nz + 1) > 2000000000LL)
    return fail(h, GRHD2_ERR_ARG, "grid too large (face count must stay below 2e9)");

  h->mixed = c.precision_policy != GRHD2_PREC_FP64;
  GridDev &G = h->G;
  Phys &ph = G.phys;
  ph.rec = c.rec_method; ph.lim = c.tvd_limiter; ph.rs = c.riemann; ph.sensor = c.shock_sensor ? 1 : 0;
  ph.nonmink = c.metric_kind != GRHD2_METRIC_MINKOWSKI;
  ph.srhd = c.metric_kind == GRHD2_METRIC_MINKOWSKI && c.geom_kind == GRHD2_GEOM_CARTESIAN;
  ph.adb = c.adb_idx; ph.g1 = c.g1; ph.rho_floor = c.rho_floor; ph.p_floor = c.p_floor; ph.v_max = c.v_max;
  G.nx = c.nx; G.ny = c.ny; G.nz = c.nz; G.ng = c.nghost; G.case_id = c.case_id;
  G.div_nx = make_fastdiv((unsigned)c.nx); G.div_ny = make_fastdiv((unsigned)c.ny);
  G.div_nx1 = make_fastdiv((unsigned)c.nx + 1); G.div_ny1 = make_fastdiv((unsigned)c.ny + 1);
  set_cell_tile(G, DEFAULT_TX);
  for (int d = 1; d <= 3; ++d) set_face_tiles(G, d, DEFAULT_TX);
  G.ncell = (long long)c.nx * c.ny * c.nz;
  G.pplane = (G.ncell + 31) / 32 * 32;
  G.nij = (long long)c.nx * c.ny;
  G.nface[0] = (long long)(c.nx + 1) * c.ny;
  G.nface[1] = (long long)c.nx * (c.ny + 1);
  G.nface[2] = G.nij;
  G.rho_floor = c.rho_floor; G.p_floor = c.p_floor;
  G.dx = c.dx; G.dy = c.dy; G.dz = c.dz;

  CUDA_TRY(h, cudaGetDevice(&h->device));
  keep_pool_memory(h->device);
  if (stream) {
    h->stream = (cudaStream_t)stream;
  } else {
    CUDA_TRY(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
  }
  int rc;
  const size_t es = h->mixed ? sizeof(float) : sizeof(double);
  char *p = nullptr;
  if ((rc = dalloc(h, &p, 5 * G.pplane * es))) return rc;
  G.P = p;
  if (stage_sd_of(c.ny, c.nz) >= 0) {  // the stage kernel's primitive rotation (stage.cuh)
    for (int r = 0; r < 2; ++r) {
      if ((rc = dalloc(h, &p, 5 * G.pplane * es))) return rc;
      G.Prot[r] = p;
    }
    const int sd = stage_sd_of(c.ny, c.nz);
    const int tx = sd == 0 ? STAGE_TILE_CELLS : 32;
    G.stage_ntx = make_fastdiv((unsigned)((c.nx + tx - 1) / tx));
  }
  if ((rc = dalloc(h, &G.U, 5 * G.pplane))) return rc;
  if ((rc = dalloc(h, &G.UP, 5 * G.pplane))) return rc;
  G.carry = c.precision_policy == GRHD2_PREC_MIXED_COMP64 ? 1 : (c.precision_policy == GRHD2_PREC_MIXED_COMP32 ? 2 : 0);
  if (G.carry) {  // carries of u and up, starting at zero
    const size_t cb = G.carry == 1 ? sizeof(double) : sizeof(float);
    for (void **cp : {&G.Uc, &G.UPc}) {
      if ((rc = dalloc(h, &p, 5 * G.pplane * cb))) return rc;
      CUDA_TRY(h, cudaMemsetAsync(p, 0, 5 * G.pplane * cb, h->stream));
      *cp = p;
    }
  }
  const long long nf[3] = {(long long)(c.nx + 1) * c.ny * c.nz, (long long)c.nx * (c.ny + 1) * c.nz,
                           (long long)c.nx * c.ny * (c.nz + 1)};
  long long nq = nf[0];
  for (int d = 0; d < 3; ++d) {
    if ((d == 1 && c.ny == 1) || (d == 2 && c.nz == 1)) continue;
    nq = std::max(nq, nf[d]);
    if ((rc = dalloc(h, &p, 5 * nf[d] * es))) return rc;
    G.F[d] = p;
  }
  if ((rc = dalloc(h, &p, 10 * nq * es))) return rc;
  G.Q = p;
  if ((rc = dalloc(h, &G.cnt, NCNT))) return rc;
  if ((rc = dalloc(h, &G.clock, 1))) return rc;
  if ((rc = dalloc(h, &h->red, 4))) return rc;
  if ((rc = dalloc(h, &h->diag, diag_bytes(c.nx, c.ny, c.nz)))) return rc;
  CUDA_TRY(h, cudaMemsetAsync(G.cnt, 0, NCNT * sizeof(unsigned long long), h->stream));
  h->hclock = GridClock{0.0, 0.0, 0.0, 0.0, 0, -1, 0, 1};
  if ((rc = write_clock(h))) return rc;
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

int grhd2_gpu_create(const grhd2_gpu_config *cfg, grhd2_gpu **out) { return grhd2_gpu_create_on_stream(cfg, nullptr, out); }

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
    for (int d = 0; d < 3; ++d) C[(CF_VA + d) * nij + q] = m->beta_c[3 * q + d] / m->alpha_c[q];
  }
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
    if ((rc = build_face_table(h, T[2], nij, 3, m->alpha_f_z, m->beta_f_z, m->gamma_f_z, m->sqrt_gamma_f_z, {}))) return rc;
  }
  if (!h->centre && (rc = dalloc(h, &h->centre, C.size()))) return rc;
  CUDA_TRY(h, cudaMemcpyAsync(h->centre, C.data(), C.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  for (int d = 0; d < 3; ++d) {
    if (T[d].empty()) continue;
    if (!h->face[d] && (rc = dalloc(h, &h->face[d], T[d].size()))) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(h->face[d], T[d].data(), T[d].size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  }
  std::vector<float> Cf, Tf[3];
  if (h->mixed) {  // FP32 copies for the FP32 arithmetic of the mixed policy
    Cf.assign(C.begin(), C.end());
    if (!h->centre_f && (rc = dalloc(h, &h->centre_f, Cf.size()))) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(h->centre_f, Cf.data(), Cf.size() * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    for (int d = 0; d < 3; ++d) {
      if (T[d].empty()) continue;
      Tf[d].assign(T[d].begin(), T[d].end());
      if (!h->face_f[d] && (rc = dalloc(h, &h->face_f[d], Tf[d].size()))) return rc;
      CUDA_TRY(h, cudaMemcpyAsync(h->face_f[d], Tf[d].data(), Tf[d].size() * sizeof(float), cudaMemcpyHostToDevice,
                                  h->stream));
    }
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));  // host vectors go out of scope
  h->G.centre = h->centre;
  for (int d = 0; d < 3; ++d) h->G.face[d] = h->face[d];
  h->G.centre_f = h->centre_f;
  for (int d = 0; d < 3; ++d) h->G.face_f[d] = h->face_f[d];
  h->metric_set = true;
  h->dt_valid = false;
  ++h->version;
  return GRHD2_OK;
}

// face counts of the three directions' tables (0: no table), as grhd2_gpu_set_metric sizes them
static void face_counts(const grhd2_gpu_config &c, size_t nf[3]) {
  nf[0] = (size_t)(c.nx + 1) * c.ny;
  nf[1] = c.ny > 1 ? (size_t)c.nx * (c.ny + 1) : 0;
  nf[2] = c.nz > 1 ? (size_t)c.nx * c.ny : 0;
}

int grhd2_gpu_set_metric_analytic(grhd2_gpu *h, const grhd2_gpu_metric_params *mp) {
  if (!h || !mp) return GRHD2_ERR_ARG;
  const grhd2_gpu_config &c = h->cfg;
  if (c.metric_kind < GRHD2_METRIC_MINKOWSKI || c.metric_kind > GRHD2_METRIC_KS || c.geom_kind < GRHD2_GEOM_CARTESIAN ||
      c.geom_kind > GRHD2_GEOM_SPHEROIDAL)
    return fail(h, GRHD2_ERR_ARG, "unknown metric kind %d or geometry kind %d", c.metric_kind, c.geom_kind);
  const bool polar = c.geom_kind == GRHD2_GEOM_SPHERICAL || c.geom_kind == GRHD2_GEOM_SPHEROIDAL;
  if (c.use_log_r && !polar)
    return fail(h, GRHD2_ERR_ARG, "a logarithmic radial grid requires spherical or spheroidal geometry");
  if (!std::isfinite(mp->bh_mass) || !std::isfinite(mp->a_spin) || !std::isfinite(mp->x_min) ||
      !std::isfinite(mp->y_min))
    return fail(h, GRHD2_ERR_ARG, "metric parameters must be finite");
  CUDA_TRY(h, cudaSetDevice(h->device));
  const MetricGrid g{{c.metric_kind, c.geom_kind, c.use_log_r ? 1 : 0, c.ny, mp->bh_mass, mp->a_spin},
                     c.nx, c.ny, mp->x_min, mp->y_min, c.dx, c.dy};
  const size_t nij = (size_t)c.nx * c.ny;
  size_t nf[3];
  face_counts(c, nf);
  int rc;
  if (!h->centre && (rc = dalloc(h, &h->centre, (size_t)NCF * nij))) return rc;
  for (int d = 0; d < 3; ++d)
    if (nf[d] && !h->face[d] && (rc = dalloc(h, &h->face[d], (size_t)NFF * nf[d]))) return rc;
  if (h->mixed) {
    if (!h->centre_f && (rc = dalloc(h, &h->centre_f, (size_t)NCF * nij))) return rc;
    for (int d = 0; d < 3; ++d)
      if (nf[d] && !h->face_f[d] && (rc = dalloc(h, &h->face_f[d], (size_t)NFF * nf[d]))) return rc;
  }
  h->metric_set = false;  // until the new tables are complete and checked
  cudaStream_t st = h->stream;
  unsigned long long *status = nullptr;
  CUDA_TRY(h, cudaMallocAsync((void **)&status, sizeof *status, st));
  CUDA_TRY(h, cudaMemsetAsync(status, 0, sizeof *status, st));
  k_metric_centre<<<nblocks((long long)nij, 128), 128, 0, st>>>(g, h->centre, status);
  if ((rc = launch_check(h))) return rc;
  for (int d = 0; d < 3; ++d) {
    if (!nf[d]) continue;
    k_metric_face<<<nblocks((long long)nf[d], 128), 128, 0, st>>>(g, d + 1, (int)nf[d], h->face[d], status);
    if ((rc = launch_check(h))) return rc;
  }
  if (h->mixed) {
    k_metric_to_float<<<nblocks((long long)(NCF * nij), 256), 256, 0, st>>>(h->centre, h->centre_f, NCF * nij);
    if ((rc = launch_check(h))) return rc;
    for (int d = 0; d < 3; ++d) {
      if (!nf[d]) continue;
      k_metric_to_float<<<nblocks((long long)(NFF * nf[d]), 256), 256, 0, st>>>(h->face[d], h->face_f[d],
                                                                               NFF * nf[d]);
      if ((rc = launch_check(h))) return rc;
    }
  }
  unsigned long long bad = 0;
  CUDA_TRY(h, cudaMemcpyAsync(&bad, status, sizeof bad, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(h, cudaFreeAsync(status, st));
  CUDA_TRY(h, cudaStreamSynchronize(st));
  if (bad & MB_ASYM) return fail(h, GRHD2_ERR_ARG, "device-built metric tables are not exactly symmetric");
  if (bad & MB_FRAME) return fail(h, GRHD2_ERR_ARG, "internal: frame gamma^dd differs from the wavespeed gamma^dd");
  h->G.centre = h->centre;
  for (int d = 0; d < 3; ++d) h->G.face[d] = h->face[d];
  h->G.centre_f = h->centre_f;
  for (int d = 0; d < 3; ++d) h->G.face_f[d] = h->face_f[d];
  h->metric_set = true;
  h->dt_valid = false;
  ++h->version;
  return GRHD2_OK;
}

int grhd2_gpu_metric_table(grhd2_gpu *h, int32_t which, double *out, size_t n, size_t *n_out) {
  if (!h) return GRHD2_ERR_ARG;
  if (which < 0 || which > 3) return fail(h, GRHD2_ERR_ARG, "metric table %d: expected 0 (centre) or 1-3 (faces)", which);
  if (!h->metric_set) return fail(h, GRHD2_ERR_STATE, "metric tables not set");
  const grhd2_gpu_config &c = h->cfg;
  size_t nf[3];
  face_counts(c, nf);
  const double *src = which == 0 ? h->centre : h->face[which - 1];
  const size_t size = which == 0 ? (size_t)NCF * c.nx * c.ny : (src ? (size_t)NFF * nf[which - 1] : 0);
  if (n_out) *n_out = size;
  if (size == 0 || (!out && n == 0)) return GRHD2_OK;
  if (!out || n < size) return fail(h, GRHD2_ERR_ARG, "metric table %d holds %zu doubles; out holds %zu", which, size, n);
  CUDA_TRY(h, cudaSetDevice(h->device));
  CUDA_TRY(h, cudaMemcpyAsync(out, src, size * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
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
    CUDA_TRY(h, cudaMemcpyAsync(h->inj, t.data(), n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));  // in the handle's stream order; the source is released
    h->G.inj = h->inj;
  }
  if (c.case_id == 8) {
    if (!b->dust_outer) return fail(h, GRHD2_ERR_ARG, "dust case needs dust_outer");
    const size_t n = (size_t)5 * c.nghost;
    std::vector<double> t(n);
    for (int g = 0; g < c.nghost; ++g)
      for (int v = 0; v < 5; ++v) t[v * c.nghost + g] = b->dust_outer[5 * g + v];
    if (!h->dust && (rc = dalloc(h, &h->dust, n))) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(h->dust, t.data(), n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));  // in the handle's stream order; the source is released
    h->G.dust = h->dust;
  }
  if (c.case_id == 5) {
    if (!b->x_c) return fail(h, GRHD2_ERR_ARG, "jet case needs x_c");
    const size_t n = (size_t)c.nx + 2 * c.nghost + 1;
    if (!h->xc && (rc = dalloc(h, &h->xc, n))) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(h->xc, b->x_c, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));  // in the handle's stream order; the source is released
    h->G.xc = h->xc;
  }
  for (int q = 0; q < 7; ++q) h->G.jet[q] = b->jet[q];
  h->bc_set = true;
  ++h->version;
  return GRHD2_OK;
}

static int upload_impl(grhd2_gpu *h, const double *up, const double *p, bool sync) {
  if (!h) return GRHD2_ERR_ARG;
  CUDA_TRY(h, cudaSetDevice(h->device));
  const GridDev &G = h->G;
  if (p) {
    CUDA_TRY(h, cudaMemcpyAsync(h->staging, p, h->n_ghosted * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (h->mixed)
      k_prims_in<float><<<nblocks(G.ncell, 256), 256, 0, h->stream>>>(G, h->staging, (float *)G.P, h->frozen[0],
                                                                     h->frozen[1], h->frozen[2]);
    else
      k_prims_in<double><<<nblocks(G.ncell, 256), 256, 0, h->stream>>>(G, h->staging, (double *)G.P, h->frozen[0],
                                                                      h->frozen[1], h->frozen[2]);
    if (int rc = launch_check(h)) return rc;
    h->prims_set = true;
  }
  if (up) {
    CUDA_TRY(h, cudaMemcpyAsync(h->staging, up, h->n_interior * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    k_cons_in<<<nblocks(G.ncell, LAYOUT_BS), LAYOUT_BS, 0, h->stream>>>(G, h->staging, G.UP);
    if (int rc = launch_check(h)) return rc;
    if (int rc = clear_carries(h, h->stream)) return rc;
    h->cons_set = true;
  }
  if (sync) CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return GRHD2_OK;
}

int grhd2_gpu_upload(grhd2_gpu *h, const double *up, const double *p) { return upload_impl(h, up, p, true); }
int grhd2_gpu_upload_async(grhd2_gpu *h, const double *up, const double *p) { return upload_impl(h, up, p, false); }

int grhd2_gpu_prim_to_cons_all(grhd2_gpu *h) {
  if (int rc = ready(h, false)) return rc;
  if (!h->prims_set) return fail(h, GRHD2_ERR_STATE, "primitives not uploaded");
  const GridDev &G = h->G;
  if (h->mixed) k_p2c_all<float><<<nblocks(G.ncell, 128), 128, 0, h->stream>>>(G, G.phys, (const float *)G.P, G.UP);
  else k_p2c_all<double><<<nblocks(G.ncell, 128), 128, 0, h->stream>>>(G, G.phys, (const double *)G.P, G.UP);
  if (int rc = launch_check(h)) return rc;
  if (int rc = clear_carries(h, h->stream)) return rc;
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
  if (int rc = self_batch(h)) return rc;
  h->hclock.mode = 0;
  h->hclock.dt_explicit = dt;
  if (int rc = write_clock(h)) return rc;
  if (int rc = batch_steps(h->self, 1, false)) return fail(h, rc, "%s", h->self->err.c_str());
  return GRHD2_OK;
}

int grhd2_gpu_run(grhd2_gpu *h, double t0, double final_time, int64_t max_steps, double *t_out, int64_t *steps_out) {
  if (int rc = ready(h, true)) return rc;
  double dt;
  if (int rc = grhd2_gpu_cfl(h, &dt)) return rc;
  if (int rc = self_batch(h)) return rc;
  // the host predicts the step count with the device clock's arithmetic (grhd2.f90:179-230)
  GridClock c{t0, final_time, dt, 0.0, 0, max_steps, 1, 0};
  c.active = t0 < final_time && max_steps != 0;
  GridClock pred = c;
  long long n = 0;
  while (pred.active) {
    pred.t = pred.t + clock_dt(pred);
    pred.steps += 1;
    pred.active = pred.t < pred.final_time && (pred.max_steps < 0 || pred.steps < pred.max_steps);
    ++n;
  }
  h->hclock = c;
  if (int rc = write_clock(h)) return rc;
  if (int rc = batch_steps(h->self, n, true)) return fail(h, rc, "%s", h->self->err.c_str());
  CUDA_TRY(h, cudaMemcpyAsync(&h->hclock, h->G.clock, sizeof(GridClock), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (int rc = check_persistent(h->self)) return fail(h, rc, "%s", h->self->err.c_str());
  if (h->hclock.steps != pred.steps || h->hclock.t != pred.t)
    return fail(h, GRHD2_ERR_STATE, "device clock (%lld steps) differs from the host prediction (%lld)",
                (long long)h->hclock.steps, (long long)pred.steps);
  if (t_out) *t_out = h->hclock.t;
  if (steps_out) *steps_out = h->hclock.steps;
  return GRHD2_OK;
}

int grhd2_gpu_calc_rhs(grhd2_gpu *h, double *rhs_host) {
  if (int rc = ready(h, false)) return rc;
  if (!h->prims_set) return fail(h, GRHD2_ERR_STATE, "primitives not uploaded");
  int rc;
  if (!h->G.RHS) {
    if ((rc = dalloc(h, &h->G.RHS, 5 * h->G.pplane))) return rc;
    ++h->version;
  }
  if ((rc = self_batch(h))) return rc;
  h->hclock.mode = 0;  // a finished run() leaves its clock inactive; the flux kernels would skip the grid
  if ((rc = write_clock(h))) return rc;
  grhd2_gpu_batch *b = h->self;
  for (const auto &grp : b->groups) {
    rc = grp.mixed ? enqueue_fluxes<float, float>(b, grp, b->stream) : enqueue_fluxes<double, double>(b, grp, b->stream);
    if (!rc)
      rc = grp.mixed ? enqueue_cells<0, float, float>(b, grp, b->stream) : enqueue_cells<0, double, double>(b, grp, b->stream);
    if (rc) return fail(h, rc, "%s", b->err.c_str());
  }
  if (rhs_host) {
    k_cons_out<<<nblocks(h->G.ncell, LAYOUT_BS), LAYOUT_BS, 0, h->stream>>>(h->G, h->G.RHS, h->staging);
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
  if (h->mixed) k_c2p_all<float><<<nblocks(G.ncell, 128), 128, 0, h->stream>>>(G, G.phys, (float *)G.P, G.UP, G.cnt);
  else k_c2p_all<double><<<nblocks(G.ncell, 128), 128, 0, h->stream>>>(G, G.phys, (double *)G.P, G.UP, G.cnt);
  if (int rc = launch_check(h)) return rc;
  if (int rc = clear_carries(h, h->stream)) return rc;
  h->prims_set = true;
  return GRHD2_OK;
}

int grhd2_gpu_set_boundary(grhd2_gpu *h) {
  if (int rc = ready(h, false)) return rc;
  if (h->cfg.case_id == 12 && (h->cfg.nz % 2) != 0)
    return fail(h, GRHD2_ERR_BOUNDARY, "CRITICAL ERROR: nz must be even for 3D Trans-Polar boundary conditions.");
  return GRHD2_OK;
}

static int download_impl(grhd2_gpu *h, double *up, double *p, bool sync) {
  if (int rc = ready(h, false)) return rc;
  const GridDev &G = h->G;
  if (p) {
    if (!h->prims_set) return fail(h, GRHD2_ERR_STATE, "primitives not uploaded");
    CUDA_TRY(h, cudaMemcpyAsync(h->staging, p, h->n_ghosted * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    const long long n = (long long)(G.nx + 2 * G.ng + 1) * (G.ny + 2 * G.ng + 1) * (G.nz + 2 * G.ng + 1);
    if (h->mixed) k_prims_out<float><<<nblocks(n, 256), 256, 0, h->stream>>>(G, (const float *)G.P, h->staging);
    else k_prims_out<double><<<nblocks(n, 256), 256, 0, h->stream>>>(G, (const double *)G.P, h->staging);
    if (int rc = launch_check(h)) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(p, h->staging, h->n_ghosted * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  }
  if (up) {
    if (!h->cons_set) return fail(h, GRHD2_ERR_STATE, "conserved state not uploaded");
    k_cons_out<<<nblocks(G.ncell, LAYOUT_BS), LAYOUT_BS, 0, h->stream>>>(G, G.UP, h->staging);
    if (int rc = launch_check(h)) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(up, h->staging, h->n_interior * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  }
  if (sync) CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return GRHD2_OK;
}

int grhd2_gpu_download(grhd2_gpu *h, double *up, double *p) { return download_impl(h, up, p, true); }
int grhd2_gpu_download_async(grhd2_gpu *h, double *up, double *p) { return download_impl(h, up, p, false); }

int grhd2_gpu_get_counters(grhd2_gpu *h, grhd2_gpu_counters *out) {
  if (!h || !out) return GRHD2_ERR_ARG;
  CUDA_TRY(h, cudaSetDevice(h->device));
  unsigned long long c[NCNT];
  CUDA_TRY(h, cudaMemcpyAsync(c, h->G.cnt, sizeof c, cudaMemcpyDeviceToHost, h->stream));
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
  CUDA_TRY(h, cudaMemsetAsync(h->G.cnt, 0, NCNT * sizeof(unsigned long long), h->stream));
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
  // scratch of this call only, from the device's stream-ordered pool on the handle's
  // stream (no device-wide synchronisation), released after the result is copied out
  double *dT = nullptr, *dq = nullptr;
  cudaStream_t st = h->stream;
  CUDA_TRY(h, cudaMallocAsync((void **)&dT, T.size() * sizeof(double), st));
  cudaError_t e = cudaMallocAsync((void **)&dq, (size_t)15 * n * sizeof(double), st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dT, T.data(), T.size() * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dq, qL, (size_t)5 * n * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && qR)
    e = cudaMemcpyAsync(dq + 5 * n, qR, (size_t)5 * n * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    if (h->mixed)
      k_riemann_faces<float><<<nblocks(n, 128), 128, 0, st>>>(h->G.phys, n, dir, dq, dq + 5 * n, dT, dq + 10 * n,
                                                              physical_only);
    else
      k_riemann_faces<double><<<nblocks(n, 128), 128, 0, st>>>(h->G.phys, n, dir, dq, dq + 5 * n, dT, dq + 10 * n,
                                                               physical_only);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(flux, dq + 10 * n, (size_t)5 * n * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(dT, st);
  if (dq) cudaFreeAsync(dq, st);
  const cudaError_t es = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = es;
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

}  // extern "C"

// ---- allocation-free face fluxes ------------------------------------------------------
// Scratch of grhd2_gpu_riemann_faces_noalloc: one fixed array per device, laid out as
// regions of GRHD2_GPU_NOALLOC_MAX_FACES entries (faces of one call are indexed 0..n-1 in
// each region).  Every region is written by the call before it is read, so nothing needs
// to start at zero.
namespace {
constexpr size_t NA_MAX = GRHD2_GPU_NOALLOC_MAX_FACES;
constexpr size_t NA_ALPHA = 0, NA_BETA = NA_ALPHA + NA_MAX, NA_GAMMA = NA_BETA + 3 * NA_MAX,
                 NA_SQG = NA_GAMMA + 9 * NA_MAX, NA_TABLE = NA_SQG + NA_MAX, NA_QL = NA_TABLE + NFF * NA_MAX,
                 NA_QR = NA_QL + 5 * NA_MAX, NA_FLUX = NA_QR + 5 * NA_MAX, NA_TOTAL = NA_FLUX + 5 * NA_MAX;
static_assert(NA_TOTAL == 50 * NA_MAX, "50 doubles per face");
// one status word after the per-face regions: nonzero when a face's frame gamma^dd differs
// from its wavespeed gamma^dd (the consistency check of build_face_table); cleared by every
// call before its table kernel runs
constexpr size_t NA_STATUS = NA_TOTAL;

static __device__ __align__(256) double g_noalloc_scratch[NA_TOTAL + 1];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
double *g_noalloc_ptr[NA_MAX_DEVICES] = {};

// per-face table of n faces (the fields build_face_table writes), built on the device
__global__ void k_face_table(int n, int dir, const double *__restrict__ alpha, const double *__restrict__ beta,
                             const double *__restrict__ gamma, const double *__restrict__ sqg, double *__restrict__ T,
                             unsigned long long *status) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n) return;
  double g[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) g[q] = gamma[9 * f + q];
  const size_t m = (size_t)n;
  T[FF_ALPHA * m + f] = alpha[f];
  T[FF_BETA_N * m + f] = beta[3 * f + (dir - 1)];
  T[FF_G11 * m + f] = g[0]; T[FF_G12 * m + f] = g[3]; T[FF_G13 * m + f] = g[6];
  T[FF_G22 * m + f] = g[4]; T[FF_G23 * m + f] = g[7]; T[FF_G33 * m + f] = g[8];
  T[FF_SQG * m + f] = sqg[f];
  const double gup_w = gamma_up_dd(g, dir);
  T[FF_GUP * m + f] = gup_w;
  double cof[9], gup;
  const bool ok = face_frame(g, dir, cof, &gup);
#pragma unroll
  for (int q = 0; q < 9; ++q) T[(FF_COF + q) * m + f] = cof[q];
  if (ok && __double_as_longlong(gup) != __double_as_longlong(gup_w)) atomicOr(status, 1ull);
  T[FF_FRAME_OK * m + f] = ok ? 1.0 : 0.0;
  T[FF_ZERO * m + f] = 0.0;
}

// device address of the scratch on the handle's device (looked up once per device)
int noalloc_scratch(grhd2_gpu *h, double **out) {
  if (h->device < 0 || h->device >= NA_MAX_DEVICES)
    return fail(h, GRHD2_ERR_ARG, "device %d is beyond the %d devices the allocation-free entry supports", h->device,
                NA_MAX_DEVICES);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[h->device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(h, GRHD2_ERR_CUDA, "cudaGetSymbolAddress of the face scratch: %s", cudaGetErrorString(e));
    g_noalloc_ptr[h->device] = (double *)p;
  }
  *out = g_noalloc_ptr[h->device];
  return GRHD2_OK;
}
}  // namespace

extern "C" {

int grhd2_gpu_riemann_faces_noalloc(grhd2_gpu *h, int n, int dir, const double *qL, const double *qR,
                                    const double *alpha, const double *beta, const double *gamma, const double *sqg,
                                    double *flux) {
  if (!h || n < 0 || dir < 1 || dir > 3 || !qL || !qR || !alpha || !beta || !gamma || !sqg || !flux)
    return fail(h, GRHD2_ERR_ARG, "invalid arguments to the allocation-free face-flux entry point");
  if ((size_t)n > NA_MAX)
    return fail(h, GRHD2_ERR_ARG, "%d faces exceed the allocation-free scratch (at most %d faces per call)", n,
                GRHD2_GPU_NOALLOC_MAX_FACES);
  if (n == 0) return GRHD2_OK;
  for (int f = 0; f < n; ++f) {
    const double *g = &gamma[9 * (size_t)f];
    if (!bit_equal(g[1], g[3]) || !bit_equal(g[2], g[6]) || !bit_equal(g[5], g[7]))
      return fail(h, GRHD2_ERR_ARG, "face metric of direction %d is not exactly symmetric at face %d", dir, f);
  }
  CUDA_TRY(h, cudaSetDevice(h->device));
  double *s = nullptr;
  if (int rc = noalloc_scratch(h, &s)) return rc;
  const size_t m = (size_t)n;
  cudaStream_t st = h->stream;
  CUDA_TRY(h, cudaMemcpyAsync(s + NA_ALPHA, alpha, m * sizeof(double), cudaMemcpyHostToDevice, st));
  CUDA_TRY(h, cudaMemcpyAsync(s + NA_BETA, beta, 3 * m * sizeof(double), cudaMemcpyHostToDevice, st));
  CUDA_TRY(h, cudaMemcpyAsync(s + NA_GAMMA, gamma, 9 * m * sizeof(double), cudaMemcpyHostToDevice, st));
  CUDA_TRY(h, cudaMemcpyAsync(s + NA_SQG, sqg, m * sizeof(double), cudaMemcpyHostToDevice, st));
  CUDA_TRY(h, cudaMemcpyAsync(s + NA_QL, qL, 5 * m * sizeof(double), cudaMemcpyHostToDevice, st));
  CUDA_TRY(h, cudaMemcpyAsync(s + NA_QR, qR, 5 * m * sizeof(double), cudaMemcpyHostToDevice, st));
  unsigned long long *status = (unsigned long long *)(s + NA_STATUS);
  CUDA_TRY(h, cudaMemsetAsync(status, 0, sizeof *status, st));
  k_face_table<<<nblocks(n, 128), 128, 0, st>>>(n, dir, s + NA_ALPHA, s + NA_BETA, s + NA_GAMMA, s + NA_SQG,
                                                s + NA_TABLE, status);
  if (int rc = launch_check(h)) return rc;
  if (h->mixed)
    k_riemann_faces<float><<<nblocks(n, 128), 128, 0, st>>>(h->G.phys, n, dir, s + NA_QL, s + NA_QR, s + NA_TABLE,
                                                            s + NA_FLUX, 0);
  else
    k_riemann_faces<double><<<nblocks(n, 128), 128, 0, st>>>(h->G.phys, n, dir, s + NA_QL, s + NA_QR, s + NA_TABLE,
                                                             s + NA_FLUX, 0);
  if (int rc = launch_check(h)) return rc;
  CUDA_TRY(h, cudaMemcpyAsync(flux, s + NA_FLUX, 5 * m * sizeof(double), cudaMemcpyDeviceToHost, st));
  unsigned long long bad = 0;
  CUDA_TRY(h, cudaMemcpyAsync(&bad, status, sizeof bad, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(h, cudaStreamSynchronize(st));
  if (bad) return fail(h, GRHD2_ERR_ARG, "internal: frame gamma^dd differs from the wavespeed gamma^dd");
  return GRHD2_OK;
}

// ---- diagnostics ------------------------------------------------------------------------
int grhd2_gpu_total_mass(grhd2_gpu *h, double *out) {
  if (!out) return fail(h, GRHD2_ERR_ARG, "out is NULL");
  if (int rc = ready(h, true)) return rc;
  if (!h->u_valid) return fail(h, GRHD2_ERR_STATE, "no step has run: the mass monitor sums u, the state at the start of the last step");
  double *part = (double *)(h->diag + (DIAG_BLOCKS + 1) * sizeof(DiagGlobal));
  k_diag_mass<<<DIAG_BLOCKS, DIAG_BS, 0, h->stream>>>(h->G, h->G.U, part);
  k_sum_final<<<1, DIAG_BS, 0, h->stream>>>(part, DIAG_BLOCKS, part + DIAG_BLOCKS);
  if (int rc = launch_check(h)) return rc;
  CUDA_TRY(h, cudaMemcpyAsync(out, part + DIAG_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return GRHD2_OK;
}

int grhd2_gpu_mdot(grhd2_gpu *h, int idx_probe, double *out) {
  if (!out) return fail(h, GRHD2_ERR_ARG, "out is NULL");
  if (int rc = ready(h, true)) return rc;
  if (idx_probe < 1 || idx_probe > h->cfg.nx)
    return fail(h, GRHD2_ERR_ARG, "CRITICAL ERROR: invalid accretion-probe index: %d", idx_probe);
  double *res = (double *)(h->diag + (DIAG_BLOCKS + 1) * sizeof(DiagGlobal));
  if (h->mixed) k_diag_mdot<float><<<1, DIAG_BS, 0, h->stream>>>(h->G, (const float *)h->G.P, h->G.UP, idx_probe - 1, res);
  else k_diag_mdot<double><<<1, DIAG_BS, 0, h->stream>>>(h->G, (const double *)h->G.P, h->G.UP, idx_probe - 1, res);
  if (int rc = launch_check(h)) return rc;
  CUDA_TRY(h, cudaMemcpyAsync(out, res, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return GRHD2_OK;
}

int grhd2_gpu_ppi_modes(grhd2_gpu *h, const double *z, double *values) {
  if (!z || !values) return fail(h, GRHD2_ERR_ARG, "z or values is NULL");
  if (int rc = ready(h, true)) return rc;
  const int nz = h->cfg.nz, MAXM = 4;
  for (int q = 0; q < 1 + 4 * MAXM; ++q) values[q] = 0.0;
  if (nz < 2) return GRHD2_OK;  // output.f90:1005: no azimuthal direction
  double *plane = (double *)(h->diag + (DIAG_BLOCKS + 1) * sizeof(DiagGlobal)) + DIAG_BLOCKS + 1;
  if (h->mixed) k_diag_azimuthal<float><<<nz, DIAG_BS, 0, h->stream>>>(h->G, (const float *)h->G.P, h->G.UP, plane);
  else k_diag_azimuthal<double><<<nz, DIAG_BS, 0, h->stream>>>(h->G, (const double *)h->G.P, h->G.UP, plane);
  if (int rc = launch_check(h)) return rc;
  std::vector<double> am(nz);
  CUDA_TRY(h, cudaMemcpyAsync(am.data(), plane, nz * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  // output.f90:1024-1047, on the host: nz terms per mode
  double c0 = 0.0, cr[4] = {0, 0, 0, 0}, ci[4] = {0, 0, 0, 0};
  for (int k = 0; k < nz; ++k) {
    c0 = c0 + am[k];
    for (int m = 1; m <= MAXM; ++m) {
      cr[m - 1] = cr[m - 1] + am[k] * std::cos((double)m * z[k]);
      ci[m - 1] = ci[m - 1] - am[k] * std::sin((double)m * z[k]);
    }
  }
  values[0] = c0;
  for (int m = 1; m <= MAXM; ++m) {
    double *v = values + 1 + 4 * (m - 1);
    v[0] = cr[m - 1];
    v[1] = ci[m - 1];
    if (c0 > DBL_MIN) {
      v[2] = std::sqrt(cr[m - 1] * cr[m - 1] + ci[m - 1] * ci[m - 1]) / c0;
      v[3] = -std::atan2(ci[m - 1], cr[m - 1]) / (double)m;
    }
  }
  return GRHD2_OK;
}

int grhd2_gpu_gw_strain(grhd2_gpu *h, const double *x, const double *y, const double *z, int use_log_r,
                        double bh_mass, double spin, double *out) {
  if (!x || !y || !z || !out) return fail(h, GRHD2_ERR_ARG, "invalid arguments to grhd2_gpu_gw_strain");
  if (int rc = ready(h, true)) return rc;
  for (int q = 0; q < 5; ++q) out[q] = 0.0;
  if (h->cfg.metric_kind == GRHD2_METRIC_MINKOWSKI || bh_mass < 0.1) return GRHD2_OK;  // output.f90:864
  // event_horizon_radius (metrics.f90:66-87)
  if (bh_mass < 0.0) return fail(h, GRHD2_ERR_ARG, "CRITICAL ERROR: black-hole mass must be non-negative.");
  const double big = std::max(1.0, std::max(bh_mass * bh_mass, spin * spin));
  const double disc = bh_mass * bh_mass - spin * spin;
  if (disc < -64.0 * DBL_EPSILON * big) return fail(h, GRHD2_ERR_ARG, "CRITICAL ERROR: Kerr spin must satisfy |a| <= M.");
  const double r_h = bh_mass + std::sqrt(disc > 0.0 ? disc : 0.0);
  const int nx = h->cfg.nx, ny = h->cfg.ny, nz = h->cfg.nz;
  std::vector<double> tab((size_t)nx + 2 * ny + 2 * nz);
  for (int i = 0; i < nx; ++i) tab[i] = use_log_r ? std::exp(x[i]) : x[i];
  for (int j = 0; j < ny; ++j) { tab[nx + j] = std::sin(y[j]); tab[nx + ny + j] = std::cos(y[j]); }
  for (int k = 0; k < nz; ++k) { tab[nx + 2 * ny + k] = std::sin(z[k]); tab[nx + 2 * ny + nz + k] = std::cos(z[k]); }
  double *base = (double *)(h->diag + (DIAG_BLOCKS + 1) * sizeof(DiagGlobal)) + DIAG_BLOCKS + 1 + nz;
  double *part = base, *res = base + 3 * DIAG_BLOCKS, *dtab = base + 3 * (DIAG_BLOCKS + 1);
  CUDA_TRY(h, cudaMemcpyAsync(dtab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  if (h->mixed)
    k_diag_gw<float><<<DIAG_BLOCKS, DIAG_BS, 0, h->stream>>>(h->G, (const float *)h->G.P, dtab, use_log_r, r_h, bh_mass,
                                                             spin, part);
  else
    k_diag_gw<double><<<DIAG_BLOCKS, DIAG_BS, 0, h->stream>>>(h->G, (const double *)h->G.P, dtab, use_log_r, r_h,
                                                              bh_mass, spin, part);
  k_sum3_final<<<1, DIAG_BS, 0, h->stream>>>(part, DIAG_BLOCKS, res);
  if (int rc = launch_check(h)) return rc;
  double I[3];
  CUDA_TRY(h, cudaMemcpyAsync(I, res, sizeof I, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));  // the host table goes out of scope
  out[0] = (I[0] - I[1]) / 1000.0;  // gw_observer_distance, output.f90:28
  out[1] = (2.0 * I[2]) / 1000.0;
  out[2] = I[0]; out[3] = I[1]; out[4] = I[2];
  return GRHD2_OK;
}

int grhd2_gpu_global_diagnostics(grhd2_gpu *h, grhd2_gpu_diagnostics *out) {
  if (!out) return fail(h, GRHD2_ERR_ARG, "out is NULL");
  if (int rc = ready(h, true)) return rc;
  DiagGlobal *part = (DiagGlobal *)h->diag;
  if (h->mixed) k_diag_global<float><<<DIAG_BLOCKS, DIAG_BS, 0, h->stream>>>(h->G, (const float *)h->G.P, h->G.UP, part);
  else k_diag_global<double><<<DIAG_BLOCKS, DIAG_BS, 0, h->stream>>>(h->G, (const double *)h->G.P, h->G.UP, part);
  k_diag_global_final<<<1, DIAG_BS, 0, h->stream>>>(part, DIAG_BLOCKS, part + DIAG_BLOCKS);
  if (int rc = launch_check(h)) return rc;
  DiagGlobal r;
  CUDA_TRY(h, cudaMemcpyAsync(&r, part + DIAG_BLOCKS, sizeof r, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  out->mass_total = r.mass; out->disk_mass = r.disk; out->angular_momentum = r.angmom;
  out->rho_min = r.rho_min; out->p_min = r.p_min; out->rho_max = r.rho_max; out->p_max = r.p_max;
  out->max_v_sq = r.vsq_max;
  out->atmosphere_cells = (int64_t)r.atmosphere;
  out->invalid_cells = (int64_t)r.invalid;
  return GRHD2_OK;
}

// ---- VTK cell data ------------------------------------------------------------------------
int grhd2_gpu_vtk_cell_data(grhd2_gpu *h, const double *r_scale, void *out_host) {
  if (!out_host) return fail(h, GRHD2_ERR_ARG, "out_host is NULL");
  if (int rc = ready(h, true)) return rc;
  const size_t field = (size_t)h->G.ncell * sizeof(double);
  int rc;
  if (!h->vtk) {  // 7 fields, device scratch kept for later frames
    if ((rc = dalloc(h, &h->vtk, 7 * (size_t)h->G.ncell + (size_t)h->cfg.nx))) return rc;
  }
  double *scale = nullptr;
  if (r_scale) {
    scale = h->vtk + 7 * (size_t)h->G.ncell;
    CUDA_TRY(h, cudaMemcpyAsync(scale, r_scale, h->cfg.nx * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  }
  unsigned long long *out = (unsigned long long *)h->vtk;
  if (h->mixed) k_vtk_cells<float><<<DIAG_BLOCKS, DIAG_BS, 0, h->stream>>>(h->G, (const float *)h->G.P, scale, out);
  else k_vtk_cells<double><<<DIAG_BLOCKS, DIAG_BS, 0, h->stream>>>(h->G, (const double *)h->G.P, scale, out);
  if ((rc = launch_check(h))) return rc;
  CUDA_TRY(h, cudaMemcpyAsync(out_host, out, 7 * field, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return GRHD2_OK;
}

// ---- checkpoint snapshots ---------------------------------------------------------------
int grhd2_gpu_snapshot_begin(grhd2_gpu *h, double *up_host) {
  if (!up_host) return fail(h, GRHD2_ERR_ARG, "up_host is NULL");
  if (int rc = ready(h, true)) return rc;
  int rc;
  if (!h->snap) {
    if ((rc = dalloc(h, &h->snap, h->n_interior))) return rc;
    CUDA_TRY(h, cudaStreamCreateWithFlags(&h->snap_stream, cudaStreamNonBlocking));
    CUDA_TRY(h, cudaEventCreateWithFlags(&h->snap_taken, cudaEventDisableTiming));
    CUDA_TRY(h, cudaEventCreateWithFlags(&h->snap_done, cudaEventDisableTiming));
  }
  // the previous snapshot's copy must have left the buffer before it is overwritten
  if (h->snap_pending) CUDA_TRY(h, cudaStreamWaitEvent(h->stream, h->snap_done, 0));
  k_cons_out<<<nblocks(h->G.ncell, LAYOUT_BS), LAYOUT_BS, 0, h->stream>>>(h->G, h->G.UP, h->snap);
  if ((rc = launch_check(h))) return rc;
  CUDA_TRY(h, cudaEventRecord(h->snap_taken, h->stream));
  CUDA_TRY(h, cudaStreamWaitEvent(h->snap_stream, h->snap_taken, 0));
  CUDA_TRY(h, cudaMemcpyAsync(up_host, h->snap, h->n_interior * sizeof(double), cudaMemcpyDeviceToHost,
                              h->snap_stream));
  CUDA_TRY(h, cudaEventRecord(h->snap_done, h->snap_stream));
  h->snap_pending = true;
  return GRHD2_OK;
}

int grhd2_gpu_snapshot_wait(grhd2_gpu *h) {
  if (!h) return GRHD2_ERR_ARG;
  if (!h->snap_pending) return GRHD2_OK;
  CUDA_TRY(h, cudaSetDevice(h->device));
  CUDA_TRY(h, cudaEventSynchronize(h->snap_done));
  h->snap_pending = false;
  return GRHD2_OK;
}

int grhd2_gpu_get_stream(grhd2_gpu *h, void **stream_out) {
  if (!h || !stream_out) return GRHD2_ERR_ARG;
  *stream_out = (void *)h->stream;
  return GRHD2_OK;
}

int grhd2_gpu_profile_step(grhd2_gpu *h, double dt, float *ms, const char **names, int cap, int *n_out) {
  if (int rc = ready(h, true)) return rc;
  if (int rc = self_batch(h)) return rc;
  h->hclock.mode = 0;
  h->hclock.dt_explicit = dt;
  if (int rc = write_clock(h)) return rc;
  if (int rc = profile_common(h->self, ms, names, cap, n_out)) return fail(h, rc, "%s", h->self->err.c_str());
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
  if (h->self) {
    destroy_batch_resources(h->self);
    destroy_lanes(h->self);
    delete h->self;
  }
  if (h->snap_stream) {
    cudaStreamSynchronize(h->snap_stream);
    cudaStreamDestroy(h->snap_stream);
  }
  if (h->snap_taken) cudaEventDestroy(h->snap_taken);
  if (h->snap_done) cudaEventDestroy(h->snap_done);
  void *bufs[] = {h->G.P, h->G.Prot[0], h->G.Prot[1], h->G.U, h->G.UP, h->G.Uc, h->G.UPc, h->G.RHS, h->G.Q, h->G.F[0], h->G.F[1],
                  h->G.F[2], h->G.cnt, h->G.clock,
                  h->centre, h->face[0], h->face[1], h->face[2], h->centre_f, h->face_f[0], h->face_f[1], h->face_f[2],
                  h->inj, h->dust, h->xc, h->frozen[0], h->frozen[1],
                  h->frozen[2], h->red, h->staging, h->diag, h->snap, h->vtk};
  // stream-ordered release: after the handle's stream (synchronised above) has drained
  for (void *b : bufs) if (b) cudaFreeAsync(b, h->stream);
  if (h->stream && h->own_stream) cudaStreamDestroy(h->stream);
  delete h;
}

// ---- batches ---------------------------------------------------------------------------
int grhd2_gpu_batch_create(grhd2_gpu **handles, int n, grhd2_gpu_batch **out) {
  if (!handles || n <= 0 || !out) return GRHD2_ERR_ARG;
  *out = nullptr;
  grhd2_gpu_batch *b = new (std::nothrow) grhd2_gpu_batch();
  if (!b) return GRHD2_ERR_NOMEM;
  *out = b;
  for (int k = 0; k < n; ++k) {
    grhd2_gpu *h = handles[k];
    if (!h) return bfail(b, GRHD2_ERR_ARG, "handle %d is NULL", k);
    if (k > 0 && (h->device != b->device || h->stream != b->stream))
      return bfail(b, GRHD2_ERR_ARG, "handle %d is on another device or stream (batched handles share one stream)", k);
    if (!h->metric_set || !(h->prims_set && h->cons_set))
      return bfail(b, GRHD2_ERR_STATE, "handle %d has no metric or state uploaded", k);
    if ((h->cfg.case_id == 7 || h->cfg.case_id == 8 || h->cfg.case_id == 5) && !h->bc_set)
      return bfail(b, GRHD2_ERR_STATE, "handle %d has no boundary data", k);
    if (k == 0) { b->device = h->device; b->stream = h->stream; }
    b->m.push_back(h);
  }
  BCUDA_TRY(b, cudaSetDevice(b->device));
  return build_batch(b);
}

int grhd2_gpu_batch_set_clock(grhd2_gpu_batch *b, int k, double t0, double final_time, int64_t max_steps) {
  if (!b || k < 0 || k >= (int)b->m.size()) return bfail(b, GRHD2_ERR_ARG, "grid index out of range");
  grhd2_gpu *h = b->m[k];
  double dt;
  if (int rc = grhd2_gpu_cfl(h, &dt)) return bfail(b, rc, "grid %d: %s", k, h->err.c_str());
  h->hclock = GridClock{t0, final_time, dt, 0.0, 0, max_steps, 1, (t0 < final_time && max_steps != 0) ? 1 : 0};
  if (int rc = write_clock(h)) return bfail(b, rc, "%s", h->err.c_str());
  return GRHD2_OK;
}

int grhd2_gpu_batch_step(grhd2_gpu_batch *b, int nsteps, int use_graph) {
  if (!b) return GRHD2_ERR_ARG;
  BCUDA_TRY(b, cudaSetDevice(b->device));
  return batch_steps(b, nsteps, use_graph != 0);
}

int grhd2_gpu_batch_cons_to_prim(grhd2_gpu_batch *b) {
  if (!b) return GRHD2_ERR_ARG;
  BCUDA_TRY(b, cudaSetDevice(b->device));
  for (size_t k = 0; k < b->m.size(); ++k) {
    grhd2_gpu *h = b->m[k];
    if (int rc = ready(h, false)) return bfail(b, rc, "grid %d: %s", (int)k, h->err.c_str());
    if (!h->cons_set) return bfail(b, GRHD2_ERR_STATE, "grid %d: conserved state not uploaded", (int)k);
  }
  if (int rc = refresh_batch(b)) return rc;
  for (const auto &grp : b->groups) {
    if (grp.nb[K_CELL] <= 0) continue;
    const unsigned nb = (unsigned)grp.nb[K_CELL];
    if (grp.mixed) k_c2p_batch<float><<<nb, CELL_BS, 0, b->stream>>>(b->d_grids, grp.d_map + grp.off[K_CELL]);
    else k_c2p_batch<double><<<nb, CELL_BS, 0, b->stream>>>(b->d_grids, grp.d_map + grp.off[K_CELL]);
    if (int rc = blaunch_check(b, "c2p_batch")) return rc;
  }
  for (grhd2_gpu *h : b->m)
    if (int rc = clear_carries(h, b->stream)) return bfail(b, rc, "%s", h->err.c_str());
  for (grhd2_gpu *h : b->m) h->prims_set = true;
  return GRHD2_OK;
}

int grhd2_gpu_batch_get_clock(grhd2_gpu_batch *b, int k, double *t, int64_t *steps, int *active) {
  if (!b || k < 0 || k >= (int)b->m.size()) return bfail(b, GRHD2_ERR_ARG, "grid index out of range");
  grhd2_gpu *h = b->m[k];
  GridClock c;
  BCUDA_TRY(b, cudaMemcpyAsync(&c, h->G.clock, sizeof c, cudaMemcpyDeviceToHost, b->stream));
  BCUDA_TRY(b, cudaStreamSynchronize(b->stream));
  if (int rc = check_persistent(b)) return rc;
  if (t) *t = c.t;
  if (steps) *steps = c.steps;
  if (active) *active = c.active;
  return GRHD2_OK;
}

int grhd2_gpu_batch_clocks(grhd2_gpu_batch *b, double *t, int64_t *steps, int *active) {
  if (!b) return GRHD2_ERR_ARG;
  BCUDA_TRY(b, cudaSetDevice(b->device));
  if (int rc = refresh_batch(b)) return rc;
  const int n = (int)b->m.size();
  std::vector<GridClock> c(n);
  k_gather_clocks<<<nblocks(n, 128), 128, 0, b->stream>>>(b->d_grids, n, b->d_clocks);
  if (int rc = blaunch_check(b, "gather_clocks")) return rc;
  BCUDA_TRY(b, cudaMemcpyAsync(c.data(), b->d_clocks, sizeof(GridClock) * n, cudaMemcpyDeviceToHost, b->stream));
  BCUDA_TRY(b, cudaStreamSynchronize(b->stream));
  if (int rc = check_persistent(b)) return rc;
  for (int g = 0; g < n; ++g) {
    if (t) t[g] = c[g].t;
    if (steps) steps[g] = c[g].steps;
    if (active) active[g] = c[g].active;
  }
  return GRHD2_OK;
}

int grhd2_gpu_batch_set_flux_variant(grhd2_gpu_batch *b, int variant) {
  if (!b) return GRHD2_ERR_ARG;
  if (variant != GRHD2_FLUX_AUTO && variant != GRHD2_FLUX_SPLIT && variant != GRHD2_FLUX_FUSED &&
      variant != GRHD2_FLUX_SPLIT_VAR)
    return bfail(b, GRHD2_ERR_ARG, "invalid flux variant %d", variant);
  BCUDA_TRY(b, cudaSetDevice(b->device));
  b->variant_request = variant;
  return build_batch(b);
}

int grhd2_gpu_batch_set_stage_kernel(grhd2_gpu_batch *b, int mode) {
  if (!b) return GRHD2_ERR_ARG;
  if (mode != GRHD2_STAGE_AUTO && mode != GRHD2_STAGE_OFF && mode != GRHD2_STAGE_ON)
    return bfail(b, GRHD2_ERR_ARG, "invalid stage-kernel mode %d", mode);
  BCUDA_TRY(b, cudaSetDevice(b->device));
  b->stage_request = mode;
  return build_batch(b);
}

int grhd2_gpu_batch_stage_kernel(grhd2_gpu_batch *b) {
  if (!b) return GRHD2_ERR_ARG;
  if (int rc = refresh_batch(b)) return rc;
  int n = 0;
  for (const auto &grp : b->groups) n += grp.stage ? 1 : 0;
  return n;
}

int grhd2_gpu_batch_set_step_mode(grhd2_gpu_batch *b, int mode) {
  if (!b) return GRHD2_ERR_ARG;
  if (mode != GRHD2_STEP_AUTO && mode != GRHD2_STEP_GRAPH && mode != GRHD2_STEP_PERSISTENT)
    return bfail(b, GRHD2_ERR_ARG, "invalid step mode %d", mode);
  BCUDA_TRY(b, cudaSetDevice(b->device));
  b->step_request = mode;
  return build_batch(b);
}

int grhd2_gpu_batch_step_mode(grhd2_gpu_batch *b) {
  if (!b) return GRHD2_ERR_ARG;
  if (int rc = refresh_batch(b)) return rc;
  return b->persistent ? GRHD2_STEP_PERSISTENT : GRHD2_STEP_GRAPH;
}

int grhd2_gpu_batch_set_tile(grhd2_gpu_batch *b, int tx) {
  if (!b) return GRHD2_ERR_ARG;
  if (tx != 0 && tx != 32 && tx != 64 && tx != 128 && tx != 256)
    return bfail(b, GRHD2_ERR_ARG, "tile extent %d must be 0 (automatic), 32, 64, 128 or 256", tx);
  BCUDA_TRY(b, cudaSetDevice(b->device));
  b->tile_request = (unsigned)tx;
  return build_batch(b);
}

int grhd2_gpu_batch_autotune(grhd2_gpu_batch *b, int reps, int *variants, int *tiles, int cap, int *n_out) {
  if (!b || reps <= 0) return bfail(b, GRHD2_ERR_ARG, "invalid arguments to autotune");
  BCUDA_TRY(b, cudaSetDevice(b->device));
  b->variant_request = GRHD2_FLUX_AUTO;
  b->tile_request = 0;
  b->forced.clear();
  if (int rc = build_batch(b)) return rc;
  const int n = (int)b->m.size();
  // tuning launches count reconstruction clamps and HLLC fallbacks: save and restore
  std::vector<unsigned long long> saved((size_t)n * NCNT);
  for (int g = 0; g < n; ++g)
    BCUDA_TRY(b, cudaMemcpyAsync(&saved[(size_t)g * NCNT], b->m[g]->G.cnt, NCNT * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, b->stream));
  BCUDA_TRY(b, cudaStreamSynchronize(b->stream));
  std::vector<GridDev> hg(n);
  for (int g = 0; g < n; ++g) hg[g] = b->m[g]->G;
  cudaEvent_t e0, e1;
  BCUDA_TRY(b, cudaEventCreate(&e0));
  BCUDA_TRY(b, cudaEventCreate(&e1));
  // In a step the face kernels find little of their input in L2 (the other kernels of the
  // step evict it); timing repeated launches would favour whichever variant reuses the most.
  // Each timed repetition therefore starts after a write larger than L2.
  const size_t flush_bytes = (size_t)160 << 20;
  void *flush = nullptr;
  if (cudaMalloc(&flush, flush_bytes) != cudaSuccess) {
    cudaGetLastError();
    flush = nullptr;  // tune without flushing
  }
  int rc = 0, k = 0;
  const int ngroups = (int)b->groups.size();
  for (int gi = 0; gi < ngroups && !rc; ++gi) {
    for (int d = 1; d <= 3 && !rc; ++d) {
      if (b->groups[gi].nb[K_FLUX_X + d - 1] <= 0) continue;
      float best = 0.0f;
      FluxChoice best_c{DEFAULT_VARIANT, DEFAULT_TX};
      bool first = true;
      for (int v : {GRHD2_FLUX_SPLIT, GRHD2_FLUX_SPLIT_VAR, GRHD2_FLUX_FUSED}) {
        for (unsigned tx : {32u, 64u, 128u}) {
          b->forced[{gi, d}] = FluxChoice{v, tx};
          if ((rc = build_batch(b))) break;
          const Group &grp = b->groups[gi];
          auto run = [&]() {
            return grp.mixed ? enqueue_dir<float, float>(b, grp, d, v, b->stream)
                             : enqueue_dir<double, double>(b, grp, d, v, b->stream);
          };
          if ((rc = run())) break;  // warm-up
          float t = 0.0f;
          for (int r = 0; r < reps && !rc; ++r) {
            if (flush) cudaMemsetAsync(flush, r & 0xff, flush_bytes, b->stream);
            cudaEventRecord(e0, b->stream);
            rc = run();
            cudaEventRecord(e1, b->stream);
            cudaError_t e = cudaEventSynchronize(e1);
            if (e != cudaSuccess) { rc = bfail(b, GRHD2_ERR_CUDA, "autotune: %s", cudaGetErrorString(e)); break; }
            float tr = 0.0f;
            cudaEventElapsedTime(&tr, e0, e1);
            t += tr;
          }
          if (rc) break;
          if (first || t < best) { best = t; best_c = FluxChoice{v, tx}; first = false; }
        }
        if (rc) break;
      }
      if (rc) break;
      b->forced[{gi, d}] = best_c;
      {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune[tune_key(b->groups[gi], hg, d)] = best_c;
      }
      if (k < cap) {
        if (variants) variants[k] = best_c.variant;
        if (tiles) tiles[k] = (int)best_c.tx;
      }
      ++k;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (flush) {
    cudaStreamSynchronize(b->stream);
    cudaFree(flush);
  }
  b->forced.clear();  // the choices now come from the cache
  int rc2 = build_batch(b);
  for (int g = 0; g < n; ++g)
    cudaMemcpyAsync(b->m[g]->G.cnt, &saved[(size_t)g * NCNT], NCNT * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                    b->stream);
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (rc) return rc;
  if (rc2) return rc2;
  if (e != cudaSuccess) return bfail(b, GRHD2_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
  if (n_out) *n_out = k;
  return GRHD2_OK;
}

int grhd2_gpu_batch_profile_step(grhd2_gpu_batch *b, float *ms, const char **names, int cap, int *n_out) {
  if (!b) return GRHD2_ERR_ARG;
  return profile_common(b, ms, names, cap, n_out);
}

const char *grhd2_gpu_batch_last_error(const grhd2_gpu_batch *b) { return b ? b->err.c_str() : "NULL batch"; }

void grhd2_gpu_batch_destroy(grhd2_gpu_batch *b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  destroy_batch_resources(b);
  destroy_lanes(b);
  delete b;
}

}  // extern "C"
