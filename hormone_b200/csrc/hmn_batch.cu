// hmn_batch.cu -- many independent simulations of uneven sizes on one GPU.
//
// A batch owns one device memory pool; each admitted simulation gets its
// state, its primitive planes and its geometry from the pool (admission is
// by footprint: hmn_batch_add fails with HMN_ENOMEM when the pool has no
// room) and a descriptor in a device array.  A batch step runs, for all
// simulations at once, the step of src/main/hormone.f90:126-147 on each
// simulation's own clock: CFL reduction, dt with the clamps, rktype fused
// RK stages and the time advance -- one persistent launch per phase and
// tile kind, captured in a CUDA graph that is replayed for every step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/hormone_gpu.h"
#include "hmn_internal.h"

using namespace hmn;

namespace {

struct SlotInfo {
  bool used = false;
  size_t off = 0, bytes = 0;
  int kind = -1;
  bool mag = false, glm = false;
  int nvar = 0;
  int n[3] = {1, 1, 1};
  int ntiles = 0;
};

struct Klass {
  int kind;
  bool mag, glm;
  int first, count;  // range in the item list
  int grid;          // persistent CTAs of the stage launches
  bool dynamic;      // stage launches take items from the shared counter
};

constexpr size_t kAlign = 256;
size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

}  // namespace

struct hmn_batch {
  int max_sims = 0;
  int precision = 0;
  int rktype = 3;
  char* pool = nullptr;
  size_t pool_bytes = 0;
  std::vector<std::pair<size_t, size_t>> free_list;  // (offset, size), sorted by offset
  SimDesc* d_sims = nullptr;
  std::vector<SimDesc> h_sims;
  std::vector<SlotInfo> slots;
  int2* d_items = nullptr;
  size_t items_cap = 0;
  std::vector<Klass> classes;
  bool dirty = true;
  cudaStream_t st = nullptr;
  int nsm = 148;
  int blocks_per_sm[3] = {0, 0, 0};  // per tile kind; 0: occupancy-derived persistent grid
  int tile_id[3] = {0, 2, 4};         // tile of each kind (batch_tile_variants)
  int sweep[3] = {HMN_SWEEP_STATIC, HMN_SWEEP_STATIC, HMN_SWEEP_STATIC};  // item order and split per kind
  int* d_queue = nullptr;             // {next item, CTAs finished} of a dynamic stage launch
  cudaGraphExec_t graph = nullptr;
  long long launches = 0;
  double* stage_h = nullptr;
  size_t stage_h_bytes = 0;
};

static int cuda_fail(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return HMN_OK;
  fprintf(stderr, "hormone_b200 batch: %s: %s\n", what, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? HMN_ENOMEM : HMN_ECUDA;
}
#define BCK(call, what)                       \
  do {                                        \
    cudaError_t _e = (call);                  \
    if (_e != cudaSuccess) return cuda_fail(_e, what); \
  } while (0)

static size_t sim_bytes(const int n[3], int nvar) {
  const size_t plane = (size_t)n[0] * n[1] * n[2];
  size_t b = 0;
  b += 3 * align_up((size_t)nvar * plane * sizeof(double));  // U[0..2]
  b += 2 * align_up((size_t)10 * plane * sizeof(double));    // P[0..1]
  for (int a = 0; a < 3; a++) b += align_up((size_t)kGeoArrays * (n[a] + 4) * sizeof(double));
  return b;
}

static bool pool_alloc(hmn_batch* b, size_t bytes, size_t* off) {
  for (size_t i = 0; i < b->free_list.size(); i++) {
    auto& f = b->free_list[i];
    if (f.second >= bytes) {
      *off = f.first;
      f.first += bytes;
      f.second -= bytes;
      if (f.second == 0) b->free_list.erase(b->free_list.begin() + i);
      return true;
    }
  }
  return false;
}

static void pool_free(hmn_batch* b, size_t off, size_t bytes) {
  b->free_list.push_back({off, bytes});
  std::sort(b->free_list.begin(), b->free_list.end());
  std::vector<std::pair<size_t, size_t>> merged;
  for (auto& f : b->free_list) {
    if (!merged.empty() && merged.back().first + merged.back().second == f.first)
      merged.back().second += f.second;
    else
      merged.push_back(f);
  }
  b->free_list.swap(merged);
}

extern "C" size_t hmn_batch_footprint(const hmn_grid* grid, const hmn_params* par) {
  if (!grid || !par) return 0;
  int dim = 0;
  for (int a = 0; a < 3; a++) dim += grid->n[a] > 1;
  const bool glm = par->mag_on && dim > 1;
  const int nvar = 5 + (par->mag_on ? 3 : 0) + (glm ? 1 : 0);
  return sim_bytes(grid->n, nvar);
}

extern "C" int hmn_batch_create(size_t pool_bytes, int max_sims, int precision, int rktype, hmn_batch** out) {
  if (!out || max_sims < 1 || pool_bytes < kAlign || (precision != 0 && precision != 1) || rktype < 1 || rktype > 3)
    return HMN_EINVAL;
  *out = nullptr;
  hmn_batch* b = new (std::nothrow) hmn_batch();
  if (!b) return HMN_ENOMEM;
  b->max_sims = max_sims;
  b->precision = precision;
  b->rktype = rktype;
  b->pool_bytes = align_up(pool_bytes);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->pool, b->pool_bytes);
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_sims, (size_t)max_sims * sizeof(SimDesc));
  if (e == cudaSuccess) e = cudaMemset(b->d_sims, 0, (size_t)max_sims * sizeof(SimDesc));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_queue, 2 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(b->d_queue, 0, 2 * sizeof(int));
  if (e != cudaSuccess) {
    int rc = cuda_fail(e, "batch create");
    hmn_batch_destroy(b);
    return rc;
  }
  b->h_sims.assign(max_sims, SimDesc());
  memset(b->h_sims.data(), 0, (size_t)max_sims * sizeof(SimDesc));
  b->slots.assign(max_sims, SlotInfo());
  b->free_list.push_back({0, b->pool_bytes});
  *out = b;
  return HMN_OK;
}

extern "C" int hmn_batch_destroy(hmn_batch* b) {
  if (!b) return HMN_EINVAL;
  if (b->st) cudaStreamSynchronize(b->st);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  cudaFree(b->pool);
  cudaFree(b->d_sims);
  cudaFree(b->d_items);
  cudaFree(b->d_queue);
  if (b->stage_h) cudaFreeHost(b->stage_h);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
  return HMN_OK;
}

// geometry arrays of one axis exactly as hmn_create derives them
static void axis_geometry(const hmn_grid* grid, int a, double* base) {
  const int L = grid->n[a] + 4;
  const double *x = grid->x[a], *xi = grid->xi[a];
  for (int s = 0; s < kGeoArrays * L; s++) base[s] = 0.0;
  for (int s = 0; s < L; s++) {
    base[0 * L + s] = x[s];
    base[1 * L + s] = grid->dx[a][s];
    base[2 * L + s] = grid->idx[a][s];
    base[3 * L + s] = grid->dxi[a][s];
    base[4 * L + s] = grid->idxi[a][s];
  }
  for (int s = 1; s < L; s++) base[5 * L + s] = x[s] - xi[s - 1];
  for (int s = 0; s < L; s++) base[6 * L + s] = xi[s] - x[s];
  for (int s = 1; s + 1 < L; s++) {
    base[7 * L + s] = (x[s + 1] - x[s]) / (xi[s] - x[s]);
    base[8 * L + s] = (x[s] - x[s - 1]) / (x[s] - xi[s - 1]);
    base[9 * L + s] = x[s + 1] - x[s];
    base[10 * L + s] = x[s] - x[s - 1];
    base[11 * L + s] = grid->idx[a][s] + grid->idx[a][s + 1];
    base[12 * L + s] = 1.0 / base[9 * L + s];
    base[13 * L + s] = base[9 * L + s] / base[10 * L + s];
    base[14 * L + s] = 1.0 / base[11 * L + s];
  }
}

static int ensure_stage(hmn_batch* b, size_t bytes) {
  if (b->stage_h_bytes >= bytes) return HMN_OK;
  if (b->stage_h) cudaFreeHost(b->stage_h);
  b->stage_h = nullptr;
  b->stage_h_bytes = 0;
  BCK(cudaMallocHost((void**)&b->stage_h, bytes), "pinned staging");
  b->stage_h_bytes = bytes;
  return HMN_OK;
}

extern "C" int hmn_batch_add(hmn_batch* b, const hmn_grid* grid, const hmn_params* par, const double* u,
                             const double* const prim[9], double time, double t_end, int* sim) {
  if (!b || !grid || !par || !u || !sim) return HMN_EINVAL;
  if (grid->ghost != 0 || par->gravswitch != 0 || par->rktype != b->rktype || par->limiter < 0 ||
      par->limiter > 2 || par->nspc != 0)
    return HMN_EBADCFG;
  int solve[3], dim = 0;
  for (int a = 0; a < 3; a++) {
    if (grid->n[a] < 1) return HMN_EINVAL;
    solve[a] = grid->n[a] > 1;
    dim += solve[a];
    if (solve[a]) {
      if (grid->n[a] < 2) return HMN_EBADCFG;
      for (int io = 0; io < 2; io++)
        for (int sv = 0; sv < 2; sv++)
          if (grid->bc[a][io][sv] < 0 || grid->bc[a][io][sv] > 5) return HMN_EBADCFG;  // codes 0-5
    }
  }
  const int kind = batch_tile_kind(solve);
  if (kind < 0) return HMN_EBADCFG;
  int slot = -1;
  for (int s = 0; s < b->max_sims; s++)
    if (!b->slots[s].used) {
      slot = s;
      break;
    }
  if (slot < 0) return HMN_ENOMEM;
  const bool mag = par->mag_on != 0, glm = mag && dim > 1;
  const int nvar = 5 + (mag ? 3 : 0) + (glm ? 1 : 0);
  const size_t bytes = sim_bytes(grid->n, nvar);
  size_t off;
  if (!pool_alloc(b, bytes, &off)) return HMN_ENOMEM;  // admission by footprint
  SlotInfo& si = b->slots[slot];
  si.used = true;
  si.off = off;
  si.bytes = bytes;
  si.kind = kind;
  si.mag = mag;
  si.glm = glm;
  si.nvar = nvar;
  for (int a = 0; a < 3; a++) si.n[a] = grid->n[a];
  SimDesc& S = b->h_sims[slot];
  memset(&S, 0, sizeof(S));
  const size_t plane = (size_t)grid->n[0] * grid->n[1] * grid->n[2];
  char* p = b->pool + off;
  for (int q = 0; q < 3; q++) {
    S.U[q] = (double*)p;
    p += align_up((size_t)nvar * plane * sizeof(double));
  }
  for (int q = 0; q < 2; q++) {
    S.P[q] = (double*)p;
    p += align_up((size_t)10 * plane * sizeof(double));
  }
  // geometry
  size_t geo_total = 0;
  for (int a = 0; a < 3; a++) geo_total += (size_t)kGeoArrays * (grid->n[a] + 4);
  int rc = ensure_stage(b, std::max(geo_total, (size_t)10 * plane) * sizeof(double));
  if (rc) {
    pool_free(b, off, bytes);
    si.used = false;
    return rc;
  }
  BCK(cudaStreamSynchronize(b->st), "sync");
  {
    double* h = b->stage_h;
    for (int a = 0; a < 3; a++) {
      const int L = grid->n[a] + 4;
      axis_geometry(grid, a, h);
      double* dbase = (double*)p;
      BCK(cudaMemcpyAsync(dbase, h, (size_t)kGeoArrays * L * sizeof(double), cudaMemcpyHostToDevice, b->st), "geo");
      BCK(cudaStreamSynchronize(b->st), "sync");
      AxisGeo& g = S.G.g[a];
      g.x = dbase + 0 * L;
      g.dx = dbase + 1 * L;
      g.idx = dbase + 2 * L;
      g.dxi = dbase + 3 * L;
      g.idxi = dbase + 4 * L;
      g.hl = dbase + 5 * L;
      g.hr = dbase + 6 * L;
      g.mcf = dbase + 7 * L;
      g.mcb = dbase + 8 * L;
      g.ga = dbase + 9 * L;
      g.gb = dbase + 10 * L;
      g.isum = dbase + 11 * L;
      g.rga = dbase + 12 * L;
      g.gab = dbase + 13 * L;
      g.risum = dbase + 14 * L;
      p += align_up((size_t)kGeoArrays * L * sizeof(double));
    }
  }
  for (int a = 0; a < 3; a++) {
    S.G.n[a] = grid->n[a];
    S.G.solve[a] = solve[a];
  }
  memcpy(S.G.bc, grid->bc, sizeof(S.G.bc));
  int tile[3];
  batch_tile_shape(b->tile_id[kind], tile);
  for (int a = 0; a < 3; a++) S.tiles[a] = (grid->n[a] + tile[a] - 1) / tile[a];
  si.ntiles = S.tiles[0] * S.tiles[1] * S.tiles[2];
  S.plane = plane;
  S.pcur = 0;
  S.nvar = nvar;
  S.limiter = par->limiter;
  S.rktype = par->rktype;
  S.glm = glm;
  S.active = 1;
  S.gamma = par->gamma;
  S.gm1 = par->gamma - 1.0;
  S.damp = std::exp(-par->alpha9wave * par->courant);
  S.phifac = 1.0;
  S.sc.min_dti_bits = 0x7ff0000000000000ULL;
  S.sc.cfmax_bits = 0ULL;
  S.sc.time = time;
  S.sc.t_out = t_end;
  S.sc.t_end = t_end;
  S.sc.courant = par->courant;
  S.sc.outstyle = 1;
  S.sc.endstyle = 1;
  // state: u and the primitives as the reference holds them after start-up
  BCK(cudaMemcpyAsync(S.U[0], u, (size_t)nvar * plane * sizeof(double), cudaMemcpyHostToDevice, b->st), "upload u");
  if (prim) {
    for (int q = 0; q < 9; q++) {
      if (prim[q])
        BCK(cudaMemcpyAsync(S.P[0] + q * plane, prim[q], plane * sizeof(double), cudaMemcpyHostToDevice, b->st),
            "upload prim");
      else
        BCK(cudaMemsetAsync(S.P[0] + q * plane, 0, plane * sizeof(double), b->st), "memset");
    }
    BCK(launch_prim_init(S.P[0], plane, mag, (int)std::min<size_t>((plane + 255) / 256, (size_t)b->nsm * 8), b->st),
        "prim init");
  } else {
    BCK(launch_prim_from_u(S.U[0], S.P[0], plane, mag, glm, (int)std::min<size_t>((plane + 255) / 256, (size_t)b->nsm * 8),
                           b->st),
        "prim");
  }
  b->launches += 1;
  BCK(cudaMemcpyAsync(b->d_sims + slot, &S, sizeof(SimDesc), cudaMemcpyHostToDevice, b->st), "descriptor");
  BCK(cudaStreamSynchronize(b->st), "sync");
  b->dirty = true;
  *sim = slot;
  return HMN_OK;
}

extern "C" int hmn_batch_remove(hmn_batch* b, int sim) {
  if (!b || sim < 0 || sim >= b->max_sims || !b->slots[sim].used) return HMN_EINVAL;
  BCK(cudaStreamSynchronize(b->st), "sync");
  SlotInfo& si = b->slots[sim];
  pool_free(b, si.off, si.bytes);
  si = SlotInfo();
  SimDesc& S = b->h_sims[sim];
  memset(&S, 0, sizeof(S));
  BCK(cudaMemcpyAsync(b->d_sims + sim, &S, sizeof(SimDesc), cudaMemcpyHostToDevice, b->st), "descriptor");
  BCK(cudaStreamSynchronize(b->st), "sync");
  b->dirty = true;
  return HMN_OK;
}

// pull every descriptor (clocks, done flags, errors) to the host mirror
static int pull(hmn_batch* b) {
  BCK(cudaMemcpyAsync(b->h_sims.data(), b->d_sims, (size_t)b->max_sims * sizeof(SimDesc), cudaMemcpyDeviceToHost,
                      b->st),
      "poll");
  BCK(cudaStreamSynchronize(b->st), "sync");
  return HMN_OK;
}

// Hold (held[s] = 1) or release simulations: a held simulation is left out
// of every step (its clock, state and CFL partials stay as they are) until
// it is released, so a scheduler can advance some simulations alone.
extern "C" int hmn_batch_set_held(hmn_batch* b, const int* held) {
  if (!b || !held) return HMN_EINVAL;
  int rc = pull(b);
  if (rc) return rc;
  bool changed = false;
  for (int s = 0; s < b->max_sims; s++) {
    const int h = b->slots[s].used && held[s] ? 1 : 0;
    if (b->h_sims[s].held != h) changed = true;
    b->h_sims[s].held = h;
  }
  if (!changed) return HMN_OK;
  BCK(cudaMemcpyAsync(b->d_sims, b->h_sims.data(), (size_t)b->max_sims * sizeof(SimDesc), cudaMemcpyHostToDevice,
                      b->st),
      "descriptor");
  BCK(cudaStreamSynchronize(b->st), "sync");
  b->dirty = true;
  return HMN_OK;
}

static int rebuild(hmn_batch* b) {
  // work list: active, unfinished simulations grouped by (tile kind, mag, glm)
  std::vector<int2> items;
  b->classes.clear();
  for (int kind = 0; kind < 3; kind++)  // the tile kinds of batch_tile_kind
    for (int m = 0; m < 3; m++) {
      const bool mag = m > 0, glm = m == 2;
      const int sweep = b->sweep[kind];
      Klass k{kind, mag, glm, (int)items.size(), 0, 0, sweep == HMN_SWEEP_DYNAMIC};
      std::vector<int> sims;
      int most = 0;
      for (int s = 0; s < b->max_sims; s++) {
        const SlotInfo& si = b->slots[s];
        if (!si.used || si.kind != kind || si.mag != mag || si.glm != glm || b->h_sims[s].sc.done ||
            b->h_sims[s].held)
          continue;
        sims.push_back(s);
        most = std::max(most, si.ntiles);
      }
      if (sweep == HMN_SWEEP_INTERLEAVED) {  // tile t of every simulation, then tile t + 1
        for (int t = 0; t < most; t++)
          for (int s : sims)
            if (t < b->slots[s].ntiles) items.push_back(make_int2(s, t));
      } else {
        if (sweep == HMN_SWEEP_DYNAMIC)  // the largest simulations first
          std::stable_sort(sims.begin(), sims.end(),
                           [b](int x, int y) { return b->slots[x].ntiles > b->slots[y].ntiles; });
        for (int s : sims)
          for (int t = 0; t < b->slots[s].ntiles; t++) items.push_back(make_int2(s, t));
      }
      k.count = (int)items.size() - k.first;
      if (k.count) {
        // occupancy queries run here, outside any stream capture
        int per = b->blocks_per_sm[kind];
        if (per <= 0) per = batch_stage_blocks_per_sm(b->tile_id[kind], mag, glm, b->precision);
        k.grid = (int)std::min<long long>((long long)per * b->nsm, k.count);
        b->classes.push_back(k);
      }
    }
  if (items.size() > b->items_cap) {
    cudaFree(b->d_items);
    b->d_items = nullptr;
    b->items_cap = std::max(items.size(), (size_t)1024);
    BCK(cudaMalloc((void**)&b->d_items, b->items_cap * sizeof(int2)), "items");
  }
  if (!items.empty())
    BCK(cudaMemcpyAsync(b->d_items, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice, b->st),
        "items");
  BCK(cudaStreamSynchronize(b->st), "sync");
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->dirty = false;
  return HMN_OK;
}

static int enqueue_step(hmn_batch* b, long long* nlaunch) {
  for (const Klass& k : b->classes) {
    BCK(launch_batch_cfl(b->d_sims, b->d_items + k.first, k.count, b->tile_id[k.kind], k.mag,
                         std::min(k.count, b->nsm * 4),
                         b->st),
        "batch cfl");
    (*nlaunch)++;
  }
  BCK(launch_batch_finalize(b->d_sims, b->max_sims, b->st), "batch finalize");
  (*nlaunch)++;
  for (int s = 1; s <= b->rktype; s++)
    for (const Klass& k : b->classes) {
      BCK(launch_batch_stage(b->d_sims, b->d_items + k.first, k.count, b->tile_id[k.kind], k.mag, k.glm, s,
                             b->rktype,
                             b->precision, k.grid, k.dynamic ? b->d_queue : nullptr, b->st),
          "batch stage");
      (*nlaunch)++;
    }
  BCK(launch_batch_advance(b->d_sims, b->max_sims, b->st), "batch advance");
  (*nlaunch)++;
  return HMN_OK;
}

extern "C" int hmn_batch_step(hmn_batch* b, int nsteps) {
  if (!b || nsteps < 0) return HMN_EINVAL;
  if (b->dirty) {
    int rc = pull(b);
    if (rc) return rc;
    rc = rebuild(b);
    if (rc) return rc;
  }
  if (b->classes.empty() || nsteps == 0) return HMN_OK;
  long long per_step = 0;
  if (!b->graph) {
    // capture one step; replaying it advances every simulation by one step
    cudaGraph_t g;
    BCK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal), "capture");
    int rc = enqueue_step(b, &per_step);
    cudaError_t e = cudaStreamEndCapture(b->st, &g);
    if (rc) return rc;
    BCK(e, "capture end");
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    BCK(e, "graph instantiate");
  } else {
    // launches per step equal those of the captured sequence
    per_step = (long long)b->classes.size() * (1 + b->rktype) + 2;
  }
  for (int s = 0; s < nsteps; s++) BCK(cudaGraphLaunch(b->graph, b->st), "graph launch");
  b->launches += per_step * nsteps;
  return HMN_OK;
}

extern "C" int hmn_batch_poll(hmn_batch* b, double* time, int* tn, int* done, int* err) {
  if (!b) return HMN_EINVAL;
  int rc = pull(b);
  if (rc) return rc;
  bool any_done = false;
  for (int s = 0; s < b->max_sims; s++) {
    const SimDesc& S = b->h_sims[s];
    if (time) time[s] = S.sc.time;
    if (tn) tn[s] = S.sc.tn;
    if (done) done[s] = b->slots[s].used ? S.sc.done : 0;
    if (err) err[s] = S.sc.err_code;
    if (b->slots[s].used && S.sc.done) any_done = true;
  }
  // drop finished simulations from the work list at the next step: the list
  // is rebuilt only when its tile count differs from that of the used,
  // unfinished and not held simulations (the set rebuild() lists), so a
  // finished simulation left in its slot does not force a rebuild and graph
  // re-capture at every poll
  if (any_done) {
    size_t live = 0;
    for (const Klass& k : b->classes) live += k.count;
    size_t want = 0;
    for (int s = 0; s < b->max_sims; s++)
      if (b->slots[s].used && !b->h_sims[s].sc.done && !b->h_sims[s].held) want += b->slots[s].ntiles;
    if (want != live) b->dirty = true;
  }
  return HMN_OK;
}

extern "C" int hmn_batch_download(hmn_batch* b, int sim, double* u, double* const prim[9]) {
  if (!b || sim < 0 || sim >= b->max_sims || !b->slots[sim].used) return HMN_EINVAL;
  int rc = pull(b);
  if (rc) return rc;
  const SimDesc& S = b->h_sims[sim];
  const SlotInfo& si = b->slots[sim];
  if (u)
    BCK(cudaMemcpyAsync(u, S.U[0], (size_t)si.nvar * S.plane * sizeof(double), cudaMemcpyDeviceToHost, b->st),
        "download u");
  if (prim) {
    // primitives of the current state; phi carries the pending phidamp factor
    const double* Pc = S.P[S.pcur];
    for (int q = 0; q < 9; q++)
      if (prim[q])
        BCK(cudaMemcpyAsync(prim[q], Pc + q * S.plane, S.plane * sizeof(double), cudaMemcpyDeviceToHost, b->st),
            "download prim");
    BCK(cudaStreamSynchronize(b->st), "sync");
    if (prim[8] && S.phifac != 1.0)
      for (size_t c = 0; c < S.plane; c++) prim[8][c] = prim[8][c] * S.phifac;
  }
  BCK(cudaStreamSynchronize(b->st), "sync");
  return S.sc.err_code;
}

extern "C" int hmn_batch_set_schedule(hmn_batch* b, int kind, int tile_id, int blocks_per_sm) {
  if (!b || kind < 0 || kind > 2 || blocks_per_sm < 0) return HMN_EINVAL;
  int ids[4], nv = batch_tile_variants(kind, ids);
  bool ok = false;
  for (int v = 0; v < nv; v++) ok = ok || ids[v] == tile_id;
  if (!ok) return HMN_EINVAL;
  BCK(cudaStreamSynchronize(b->st), "sync");
  b->blocks_per_sm[kind] = blocks_per_sm;
  if (tile_id != b->tile_id[kind]) {
    b->tile_id[kind] = tile_id;
    int tile[3];
    batch_tile_shape(tile_id, tile);
    int rc = pull(b);
    if (rc) return rc;
    for (int s = 0; s < b->max_sims; s++) {
      SlotInfo& si = b->slots[s];
      if (!si.used || si.kind != kind) continue;
      SimDesc& S = b->h_sims[s];
      for (int a = 0; a < 3; a++) S.tiles[a] = (si.n[a] + tile[a] - 1) / tile[a];
      si.ntiles = S.tiles[0] * S.tiles[1] * S.tiles[2];
      BCK(cudaMemcpyAsync(&b->d_sims[s].tiles, S.tiles, sizeof(S.tiles), cudaMemcpyHostToDevice, b->st), "tiles");
    }
    BCK(cudaStreamSynchronize(b->st), "sync");
  }
  b->dirty = true;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return HMN_OK;
}

extern "C" int hmn_batch_set_sweep(hmn_batch* b, int kind, int sweep) {
  if (!b || kind < 0 || kind > 2 || sweep < HMN_SWEEP_STATIC || sweep > HMN_SWEEP_DYNAMIC) return HMN_EINVAL;
  BCK(cudaStreamSynchronize(b->st), "sync");
  if (sweep == b->sweep[kind]) return HMN_OK;
  b->sweep[kind] = sweep;
  b->dirty = true;  // the next step rebuilds the work list and its graph
  return HMN_OK;
}

extern "C" long long hmn_batch_launch_count(hmn_batch* b) { return b ? b->launches : -1; }

extern "C" int hmn_batch_sync(hmn_batch* b) {
  if (!b) return HMN_EINVAL;
  BCK(cudaStreamSynchronize(b->st), "sync");
  return HMN_OK;
}

extern "C" void* hmn_batch_stream(hmn_batch* b) { return b ? (void*)b->st : nullptr; }
