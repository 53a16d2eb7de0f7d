// hmn_capi.cu -- the C ABI of include/hormone_gpu.h: context, device memory,
// host<->device layout conversion and the launch sequence of one step
// (src/main/hormone.f90:126-147).
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstddef>
#include <new>
#include <vector>

#include "../../include/hormone_gpu.h"
#include "hmn_internal.h"


using namespace hmn;

constexpr int kRunGraphSteps = 16;

struct hmn_ctx {
  int n[3];
  int solve[3];
  int dim, mag, glm, nvar, ghost;
  int bc[3][2][2];
  hmn_params par;
  size_t plane;
  double* buf[3];            // conserved-state RK buffers: [0] = U^n (A), [1] = B, [2] = C
  double* pbuf[2];           // primitive planes (10 each), ping-pong across stages
  int pcur;                  // primitive buffer of the current state
  double* geo;               // 3 axes x kGeoArrays x (n+4)
  double* gphi[2];           // gravitational potential ping-pong
  double* gpsi[2];
  double* gorg[2];
  int gcur;                  // current potential buffer
  double* prim_out;          // device scratch for downloads (10 planes)
  double* stage_h;           // pinned staging for ghosted host layouts
  size_t stage_h_bytes;
  DevScalars* sc;            // device scalars
  DevScalars* sc_h;          // pinned mirror
  GridDev G;
  cudaStream_t st;
  double phifac;             // pending phidamp factor of the phi slot
  int tile[3], tiles[3];
  long long launches;
  double grvtime, cgrav_old;
  double dtg_unit;
  int nsm;
  TmaMaps tmaps[2];          // tensor maps of pbuf[0], pbuf[1] for TMA staging of 3-D tiles
  int tma_ok;
  double* zsend[2];          // slab decomposition: caller's send buffers (low, high z face)
  // push exchange: this slab's halo buffers [low, high][parity] and the
  // neighbours' buffers its stages store into [low neighbour, high][parity];
  // zpar is the parity holding the halos of the current state
  const double* zrecv[2][2];
  double* zpush[2][2];
  int zpush_on, zpar;
  double* gsend[2];          // slab decomposition with gravity: caller's potential send buffers
  // the gravity sub-cycles planned by the last hmn_gravity_begin: cycles
  // left, the next RK sub-stage, the cycle's step, speed and psi damping
  int gv_left, gv_g;
  double gv_dtgrav, gv_cgrav, gv_damp;
  double* dir[3][2];         // Dirichlet ghost values per face (device)
  double* fb;                // boundary code 10: the inner x3 face's flux (device, 9 + nspc)
  double* spcorg;            // passive scalars times density at RK stage 1
  double* xi1_h;             // host copies of the grid arrays the metric set-up needs
  double* axis_h;            // x, dx, dxi, idx of the three axes, (n+4) each
  double* hgc;               // spherical Laplacian coefficients: 8 planes
  double* gin;               // potential beyond r = xi1s after the last boundary pass (n1*n2)
  double xi1s;
  // hmn_run's device loop as a CUDA graph of kRunGraphSteps steps, valid for
  // the primitive-buffer parity and phidamp factor it was captured with
  unsigned int* small_bar;   // grid barrier of the persistent small-grid loop (2 words, lazily)
  int hg_uni, hg_urcn_ok;    // uniform Cartesian grid: the gravity stage's constant Laplacian weights
  double hg_c0, hg_cm[3], hg_cp[3], hg_cn, hg_rcn;
  cudaGraphExec_t run_exec;
  int run_pcur;
  double run_phifac;
  long long run_launches;    // kernel launches one replay makes
  double* sphbuf;            // spherical metric factors (SphGeo arrays)
  double* sincbuf;           // spherical: sin of the theta centres (device, from js-2), or nullptr
  double* evobuf;            // evo_output partials and totals (device)
  // asynchronous checkpoint: device snapshot -> pinned staging on a copy stream
  cudaStream_t cst;
  cudaEvent_t ck_snap, ck_done;
  double* ck_dev;            // nvar u planes, 9 primitive planes, grvphi, grvpsi
  double* ck_h;              // pinned host staging of the same
  int ck_pending;
  double* ck_u;              // destinations given to hmn_checkpoint_begin
  double* ck_prim[9];
  double* ck_gphi;
  double* ck_gpsi;
  double* ck_spc;
};

static int cuda_fail(hmn_ctx* c, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return HMN_OK;
  fprintf(stderr, "hormone_b200: %s: %s\n", what, cudaGetErrorString(e));
  (void)c;
  return e == cudaErrorMemoryAllocation ? HMN_ENOMEM : HMN_ECUDA;
}

#define CK(call, what)                         \
  do {                                         \
    cudaError_t _e = (call);                   \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, what); \
  } while (0)

// cuTensorMapEncodeTiled from the driver, found through the runtime (no -lcuda)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// Tensor maps of one set of primitive planes, seen as a 4-D tensor
// (x, y, z, plane) of doubles, with the three box shapes of a 3-D tile's
// stencil region.  Needs every stride to be a multiple of 16 bytes (nx even).
static bool encode_region_maps(const double* P, const int n[3], size_t plane, const int tile[3], TmaMaps* out) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn || n[0] % 2 != 0) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)n[0], (cuuint64_t)n[1], (cuuint64_t)n[2], 10};
  const cuuint64_t strides[3] = {(cuuint64_t)n[0] * 8, (cuuint64_t)n[0] * n[1] * 8, (cuuint64_t)plane * 8};
  const cuuint32_t boxes[3][4] = {{(cuuint32_t)tile[0] + 4, (cuuint32_t)tile[1], (cuuint32_t)tile[2], 1},
                                  {(cuuint32_t)tile[0], 2, (cuuint32_t)tile[2], 1},
                                  {(cuuint32_t)tile[0], (cuuint32_t)tile[1], 2, 1}};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  for (int b = 0; b < 3; b++) {
    CUresult r = fn(&out->box[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(P), dims, strides,
                    boxes[b], estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
  }
  return true;
}

// TMA staging of 3-D tiles (grids with an even x extent).  On by default for
// the mixed form (2.6 % faster at 256^3); off for FP64, whose TMA variant
// spills more under the 96-register cap of its 640-thread CTA and runs 7 %
// slower.  HMN_TMA=1 / HMN_TMA=0 force it on / off.
static void setup_tma(hmn_ctx* ctx) {
  ctx->tma_ok = 0;
  bool want = ctx->par.precision == 1;
  const char* env = getenv("HMN_TMA");
  if (env && env[0]) want = env[0] != '0';
  if (!want) return;
  if (!(ctx->solve[0] && ctx->solve[1] && ctx->solve[2]) || ctx->par.nspc > 0) return;
  bool ok = true;
  for (int b = 0; b < 2 && ok; b++)
    ok = encode_region_maps(ctx->pbuf[b], ctx->n, ctx->plane, ctx->tile, &ctx->tmaps[b]);
  ctx->tma_ok = ok ? 1 : 0;
}

// the stage tile of this grid (stage_tile), again once the coordinate
// system is known: spherical grids take the smaller 3-D tile
static void retile(hmn_ctx* ctx) {
  stage_tile(ctx->solve, ctx->par.precision, ctx->par.nspc, ctx->tile, ctx->G.sph.on && ctx->G.sph.crd == 2);
  for (int a = 0; a < 3; a++) ctx->tiles[a] = (ctx->n[a] + ctx->tile[a] - 1) / ctx->tile[a];
  setup_tma(ctx);
}

static size_t ghosted_index(const hmn_ctx* c, int i, int j, int k) {
  const int g = c->ghost;
  const size_t sx = (size_t)c->n[0] + 2 * g, sy = (size_t)c->n[1] + 2 * g;
  return (size_t)(i + g) + sx * ((size_t)(j + g) + sy * (size_t)(k + g));
}

static size_t ghosted_plane(const hmn_ctx* c) {
  const int g = c->ghost;
  return ((size_t)c->n[0] + 2 * g) * ((size_t)c->n[1] + 2 * g) * ((size_t)c->n[2] + 2 * g);
}

static int ensure_stage(hmn_ctx* ctx, size_t bytes) {
  if (ctx->stage_h_bytes >= bytes) return HMN_OK;
  if (ctx->stage_h) cudaFreeHost(ctx->stage_h);
  ctx->stage_h = nullptr;
  ctx->stage_h_bytes = 0;
  CK(cudaMallocHost((void**)&ctx->stage_h, bytes), "cudaMallocHost");
  ctx->stage_h_bytes = bytes;
  return HMN_OK;
}

// copy nplanes host planes (ghosted or packed) into contiguous device planes
static int to_device(hmn_ctx* ctx, double* dst, const double* src, int nplanes, size_t src_plane_stride) {
  const size_t P = ctx->plane;
  if (ctx->ghost == 0) {
    for (int q = 0; q < nplanes; q++)
      CK(cudaMemcpyAsync(dst + q * P, src + q * src_plane_stride, P * sizeof(double), cudaMemcpyHostToDevice,
                         ctx->st),
         "upload");
    return HMN_OK;
  }
  int rc = ensure_stage(ctx, (size_t)nplanes * P * sizeof(double));
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->st), "sync");
  size_t o = 0;
  for (int q = 0; q < nplanes; q++)
    for (int k = 0; k < ctx->n[2]; k++)
      for (int j = 0; j < ctx->n[1]; j++)
        for (int i = 0; i < ctx->n[0]; i++) ctx->stage_h[o++] = src[q * src_plane_stride + ghosted_index(ctx, i, j, k)];
  CK(cudaMemcpyAsync(dst, ctx->stage_h, (size_t)nplanes * P * sizeof(double), cudaMemcpyHostToDevice, ctx->st),
     "upload");
  CK(cudaStreamSynchronize(ctx->st), "sync");
  return HMN_OK;
}

static int to_host(hmn_ctx* ctx, double* dst, const double* src, int nplanes, size_t dst_plane_stride) {
  const size_t P = ctx->plane;
  if (ctx->ghost == 0) {
    for (int q = 0; q < nplanes; q++)
      CK(cudaMemcpyAsync(dst + q * dst_plane_stride, src + q * P, P * sizeof(double), cudaMemcpyDeviceToHost,
                         ctx->st),
         "download");
    CK(cudaStreamSynchronize(ctx->st), "sync");
    return HMN_OK;
  }
  int rc = ensure_stage(ctx, (size_t)nplanes * P * sizeof(double));
  if (rc) return rc;
  CK(cudaMemcpyAsync(ctx->stage_h, src, (size_t)nplanes * P * sizeof(double), cudaMemcpyDeviceToHost, ctx->st),
     "download");
  CK(cudaStreamSynchronize(ctx->st), "sync");
  size_t o = 0;
  for (int q = 0; q < nplanes; q++)
    for (int k = 0; k < ctx->n[2]; k++)
      for (int j = 0; j < ctx->n[1]; j++)
        for (int i = 0; i < ctx->n[0]; i++) dst[q * dst_plane_stride + ghosted_index(ctx, i, j, k)] = ctx->stage_h[o++];
  return HMN_OK;
}

// a slab of a z-decomposed grid with at least one neighbouring slab
static bool slab_exchanges(const hmn_ctx* ctx) { return ctx->G.zhalo[0] || ctx->G.zhalo[1]; }

static int blocks_for(const hmn_ctx* ctx) {
  size_t b = (ctx->plane + 255) / 256;
  size_t cap = (size_t)ctx->nsm * 8;
  return (int)(b < cap ? (b ? b : 1) : cap);
}

extern "C" int hmn_create(const hmn_grid* grid, const hmn_params* par, hmn_ctx** out) {
  if (!grid || !par || !out) return HMN_EINVAL;
  *out = nullptr;
  for (int a = 0; a < 3; a++) {
    if (grid->n[a] < 1) return HMN_EINVAL;
    if (!grid->x[a] || !grid->xi[a] || !grid->dx[a] || !grid->dxi[a] || !grid->idx[a] || !grid->idxi[a])
      return HMN_EINVAL;
  }
  if (grid->ghost != 0 && grid->ghost != 2) return HMN_EINVAL;
  if (par->rktype < 1 || par->rktype > 3 || par->limiter < 0 || par->limiter > 2) return HMN_EBADCFG;
  if (par->gravswitch != 0 && par->gravswitch != 3) return HMN_EBADCFG;
  if (par->precision != 0 && par->precision != 1) return HMN_EBADCFG;
  // passive scalars: at most 8, FP64 form only
  if (par->nspc < 0 || par->nspc > 8 || (par->nspc > 0 && par->precision != 0)) return HMN_EBADCFG;
  hmn_ctx* ctx = new (std::nothrow) hmn_ctx();
  if (!ctx) return HMN_ENOMEM;
  memset(ctx, 0, sizeof(*ctx));
  ctx->par = *par;
  ctx->ghost = grid->ghost;
  ctx->dim = 0;
  for (int a = 0; a < 3; a++) {
    ctx->n[a] = grid->n[a];
    ctx->solve[a] = grid->n[a] > 1;
    ctx->dim += ctx->solve[a];
  }
  memcpy(ctx->bc, grid->bc, sizeof(ctx->bc));
  for (int a = 0; a < 3; a++) {
    if (!ctx->solve[a]) continue;
    for (int io = 0; io < 2; io++)
      for (int sv = 0; sv < 2; sv++) {
        const int code = ctx->bc[a][io][sv];
        // code 10 exists only at the inner x3 face, for scalars and vectors alike (fluxboundary.f90:22-28)
        const bool flux10 = code == 10 && a == 2 && io == 0 && ctx->bc[2][0][0] == 10 && ctx->bc[2][0][1] == 10;
        if (!((code >= 0 && code <= 5) || code == 9 || flux10)) {
          delete ctx;
          return HMN_EBADCFG;
        }
      }
    if (ctx->n[a] < 2) {
      delete ctx;
      return HMN_EBADCFG;
    }
  }
  if (par->gravswitch == 3 && ctx->dim < 2) {  // 3-D Cartesian, or spherical (r, theta) / 3-D (hmn_set_metric)
    delete ctx;
    return HMN_EBADCFG;
  }
  ctx->mag = par->mag_on != 0;
  ctx->glm = ctx->mag && ctx->dim > 1;
  ctx->nvar = 5 + (ctx->mag ? 3 : 0) + (ctx->glm ? 1 : 0);
  ctx->plane = (size_t)ctx->n[0] * ctx->n[1] * ctx->n[2];
  ctx->phifac = 1.0;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    int rc = cuda_fail(ctx, e, "device setup");
    delete ctx;
    return rc;
  }
  // geometry arrays (host derivation, single IEEE operations)
  const int kA = kGeoArrays;
  size_t geo_len = 0;
  for (int a = 0; a < 3; a++) geo_len += (size_t)kA * (ctx->n[a] + 4);
  std::vector<double> geo(geo_len, 0.0);
  size_t off = 0;
  size_t offs[3];
  for (int a = 0; a < 3; a++) {
    const int n = ctx->n[a], L = n + 4;
    offs[a] = off;
    double* base = geo.data() + off;
    const double *x = grid->x[a], *xi = grid->xi[a];
    for (int s = 0; s < L; s++) {
      base[0 * L + s] = x[s];
      base[1 * L + s] = grid->dx[a][s];
      base[2 * L + s] = grid->idx[a][s];
      base[3 * L + s] = grid->dxi[a][s];
      base[4 * L + s] = grid->idxi[a][s];
    }
    for (int s = 1; s < L; s++) base[5 * L + s] = x[s] - xi[s - 1];  // hl
    for (int s = 0; s < L; s++) base[6 * L + s] = xi[s] - x[s];      // hr
    for (int s = 1; s + 1 < L; s++) {
      base[7 * L + s] = (x[s + 1] - x[s]) / (xi[s] - x[s]);          // mcf
      base[8 * L + s] = (x[s] - x[s - 1]) / (x[s] - xi[s - 1]);      // mcb
      base[9 * L + s] = x[s + 1] - x[s];                              // ga
      base[10 * L + s] = x[s] - x[s - 1];                             // gb
      base[11 * L + s] = grid->idx[a][s] + grid->idx[a][s + 1];       // isum
      base[12 * L + s] = 1.0 / base[9 * L + s];                       // rga
      base[13 * L + s] = base[9 * L + s] / base[10 * L + s];          // gab
      base[14 * L + s] = 1.0 / base[11 * L + s];                      // risum
    }
    off += (size_t)kA * L;
  }
  ctx->xi1_h = (double*)malloc((size_t)(ctx->n[0] + 4) * sizeof(double));
  ctx->axis_h = (double*)malloc((size_t)4 * (ctx->n[0] + ctx->n[1] + ctx->n[2] + 12) * sizeof(double));
  if (!ctx->xi1_h || !ctx->axis_h) {
    free(ctx->xi1_h);
    free(ctx->axis_h);
    cudaStreamDestroy(ctx->st);
    delete ctx;
    return HMN_ENOMEM;
  }
  memcpy(ctx->xi1_h, grid->xi[0], (size_t)(ctx->n[0] + 4) * sizeof(double));
  {
    double* h = ctx->axis_h;
    for (int a = 0; a < 3; a++) {
      const size_t L = (size_t)ctx->n[a] + 4;
      const double* src[4] = {grid->x[a], grid->dx[a], grid->dxi[a], grid->idx[a]};
      for (int q = 0; q < 4; q++, h += L) memcpy(h, src[q], L * sizeof(double));
    }
  }
  size_t bytes = ctx->plane * sizeof(double);
  int nplanes = 9;  // every RK buffer can also hold the 9 primitive planes
  e = cudaMalloc((void**)&ctx->geo, geo_len * sizeof(double));
  for (int b = 0; b < 3 && e == cudaSuccess; b++) e = cudaMalloc((void**)&ctx->buf[b], nplanes * bytes);
  for (int b = 0; b < 2 && e == cudaSuccess; b++)
    e = cudaMalloc((void**)&ctx->pbuf[b], (size_t)(10 + par->nspc) * bytes);
  if (e == cudaSuccess && par->nspc > 0) e = cudaMalloc((void**)&ctx->spcorg, (size_t)par->nspc * bytes);
  if (e == cudaSuccess) e = cudaMalloc((void**)&ctx->prim_out, 10 * bytes);
  if (e == cudaSuccess) e = cudaMalloc((void**)&ctx->sc, sizeof(DevScalars));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&ctx->sc_h, sizeof(DevScalars));
  if (e == cudaSuccess && par->gravswitch == 3) {
    for (int b = 0; b < 2 && e == cudaSuccess; b++) {
      e = cudaMalloc((void**)&ctx->gphi[b], bytes);
      if (e == cudaSuccess) e = cudaMalloc((void**)&ctx->gpsi[b], bytes);
      if (e == cudaSuccess) e = cudaMalloc((void**)&ctx->gorg[b], bytes);
    }
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->geo, geo.data(), geo_len * sizeof(double), cudaMemcpyHostToDevice, ctx->st);
  if (e == cudaSuccess) {
    for (int b = 0; b < 3 && e == cudaSuccess; b++) e = cudaMemsetAsync(ctx->buf[b], 0, nplanes * bytes, ctx->st);
    for (int b = 0; b < 2 && e == cudaSuccess; b++)
      e = cudaMemsetAsync(ctx->pbuf[b], 0, (size_t)(10 + par->nspc) * bytes, ctx->st);
    for (int b = 0; b < 2 && e == cudaSuccess && par->gravswitch == 3; b++) {
      e = cudaMemsetAsync(ctx->gphi[b], 0, bytes, ctx->st);
      if (e == cudaSuccess) e = cudaMemsetAsync(ctx->gpsi[b], 0, bytes, ctx->st);
    }
  }
  if (e != cudaSuccess) {
    int rc = cuda_fail(ctx, e, "allocation");
    hmn_destroy(ctx);
    return rc;
  }
  // device scalars
  DevScalars s;
  memset(&s, 0, sizeof(s));
  s.min_dti_bits = 0x7ff0000000000000ULL;
  s.cfmax_bits = 0ULL;
  s.courant = par->courant;
  s.HGfac = par->HGfac;
  s.hgcfl = par->hgcfl;
  s.outstyle = par->outstyle;
  s.endstyle = par->endstyle;
  s.gravswitch = par->gravswitch;
  s.maxtngrv = par->maxtngrv;
  // tools.f90:160-183: dtg_unit = min over cells of dtgrav_cell(cgrav=1)
  if (par->gravswitch == 3) {
    double m = INFINITY;
    const double off0 = ctx->solve[0] ? 1.0 : 0.0, off1 = ctx->solve[1] ? 1.0 : 0.0, off2 = ctx->solve[2] ? 1.0 : 0.0;
    for (int k = 0; k < ctx->n[2]; k++)
      for (int j = 0; j < ctx->n[1]; j++)
        for (int i = 0; i < ctx->n[0]; i++) {
          const double d1 = grid->dxi[0][i + 2], d2 = grid->dxi[1][j + 2], d3 = grid->dxi[2][k + 2];
          const double dvol = d1 * d2 * d3;
          const double s1 = d2 * d3 + d2 * d3, s2 = d1 * d3 + d1 * d3, s3 = d1 * d2 + d1 * d2;
          const double v = dvol / (1.0 * (off0 * s1 + off1 * s2 + off2 * s3));
          m = v < m ? v : m;
        }
    s.dtg_unit = m;
    ctx->dtg_unit = m;
  }
  *ctx->sc_h = s;
  e = cudaMemcpyAsync(ctx->sc, ctx->sc_h, sizeof(DevScalars), cudaMemcpyHostToDevice, ctx->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
  if (e != cudaSuccess) {
    int rc = cuda_fail(ctx, e, "init");
    hmn_destroy(ctx);
    return rc;
  }
  // GridDev with device pointers
  GridDev& G = ctx->G;
  for (int a = 0; a < 3; a++) {
    G.n[a] = ctx->n[a];
    G.solve[a] = ctx->solve[a];
    const int L = ctx->n[a] + 4;
    const double* base = ctx->geo + offs[a];
    G.g[a].x = base + 0 * L;
    G.g[a].dx = base + 1 * L;
    G.g[a].idx = base + 2 * L;
    G.g[a].dxi = base + 3 * L;
    G.g[a].idxi = base + 4 * L;
    G.g[a].hl = base + 5 * L;
    G.g[a].hr = base + 6 * L;
    G.g[a].mcf = base + 7 * L;
    G.g[a].mcb = base + 8 * L;
    G.g[a].ga = base + 9 * L;
    G.g[a].gb = base + 10 * L;
    G.g[a].isum = base + 11 * L;
    G.g[a].rga = base + 12 * L;
    G.g[a].gab = base + 13 * L;
    G.g[a].risum = base + 14 * L;
  }
  memcpy(G.bc, ctx->bc, sizeof(G.bc));
  // a Cartesian grid uniform along every axis gives every cell the same
  // Laplacian weights in the gravity stage: form them once, in the kernel's
  // operation order (hg_stage_kernel)
  ctx->hg_uni = 1;
  for (int a = 0; a < 3; a++) {
    const int n = ctx->n[a];
    for (int s = 2; s <= n + 2; s++)
      if (grid->dx[a][s] != grid->dx[a][2] || grid->idx[a][s] != grid->idx[a][2]) ctx->hg_uni = 0;
    for (int s = 2; s <= n + 1; s++)
      if (grid->dxi[a][s] != grid->dxi[a][2]) ctx->hg_uni = 0;
  }
  if (ctx->hg_uni) {
    const double dxi0 = grid->dxi[0][2], dxi1 = grid->dxi[1][2], dxi2 = grid->dxi[2][2];
    const double i0 = grid->idx[0][2], i1 = grid->idx[1][2], i2 = grid->idx[2][2];
    ctx->hg_c0 = -((i0 + i0) * dxi1 * dxi2 + (i1 + i1) * dxi0 * dxi2 + (i2 + i2) * dxi0 * dxi1);
    const double ayz = dxi1 * dxi2, axz = dxi0 * dxi2, axy = dxi0 * dxi1;
    ctx->hg_cm[0] = ayz / grid->dx[0][2];
    ctx->hg_cp[0] = ayz / grid->dx[0][3];
    ctx->hg_cm[1] = axz / grid->dx[1][2];
    ctx->hg_cp[1] = axz / grid->dx[1][3];
    ctx->hg_cm[2] = axy / grid->dx[2][2];
    ctx->hg_cp[2] = axy / grid->dx[2][3];
    ctx->hg_cn = dxi0 * dxi1 * dxi2;
    ctx->hg_rcn = 1.0 / ctx->hg_cn;
    const double m = std::fabs(ctx->hg_cn);
    ctx->hg_urcn_ok = m >= std::ldexp(1.0, -500) && m < std::ldexp(1.0, 501);
  }
  G.idx_rn = 1;
  for (int a = 0; a < 3; a++)
    for (int s = 2; s < ctx->n[a] + 3; s++) {
      const double dx = grid->dx[a][s], m = std::fabs(dx);
      if (!(grid->idx[a][s] == 1.0 / dx) || !(m >= std::ldexp(1.0, -500)) || !(m < std::ldexp(1.0, 501)))
        G.idx_rn = 0;
    }
  stage_tile(ctx->solve, par->precision, par->nspc, ctx->tile);
  for (int a = 0; a < 3; a++) ctx->tiles[a] = (ctx->n[a] + ctx->tile[a] - 1) / ctx->tile[a];
  setup_tma(ctx);
  *out = ctx;
  return HMN_OK;
}

extern "C" int hmn_destroy(hmn_ctx* ctx) {
  if (!ctx) return HMN_EINVAL;
  if (ctx->st) cudaStreamSynchronize(ctx->st);
  if (ctx->ck_pending) cudaEventSynchronize(ctx->ck_done);
  if (ctx->cst) cudaStreamDestroy(ctx->cst);
  if (ctx->ck_snap) cudaEventDestroy(ctx->ck_snap);
  if (ctx->ck_done) cudaEventDestroy(ctx->ck_done);
  cudaFree(ctx->ck_dev);
  if (ctx->ck_h) cudaFreeHost(ctx->ck_h);
  for (int b = 0; b < 3; b++) cudaFree(ctx->buf[b]);
  for (int b = 0; b < 2; b++) cudaFree(ctx->pbuf[b]);
  cudaFree(ctx->spcorg);
  cudaFree(ctx->small_bar);
  for (int a = 0; a < 3; a++)
    for (int io = 0; io < 2; io++) cudaFree(ctx->dir[a][io]);
  cudaFree(ctx->fb);
  for (int b = 0; b < 2; b++) {
    cudaFree(ctx->gphi[b]);
    cudaFree(ctx->gpsi[b]);
    cudaFree(ctx->gorg[b]);
  }
  if (ctx->run_exec) cudaGraphExecDestroy(ctx->run_exec);
  cudaFree(ctx->geo);
  cudaFree(ctx->sphbuf);
  cudaFree(ctx->sincbuf);
  cudaFree(ctx->evobuf);
  cudaFree(ctx->hgc);
  cudaFree(ctx->gin);
  free(ctx->xi1_h);
  free(ctx->axis_h);
  cudaFree(ctx->prim_out);
  cudaFree(ctx->sc);
  if (ctx->sc_h) cudaFreeHost(ctx->sc_h);
  if (ctx->stage_h) cudaFreeHost(ctx->stage_h);
  if (ctx->st) cudaStreamDestroy(ctx->st);
  delete ctx;
  return HMN_OK;
}

// the captured device loop bakes in the grid description: drop it whenever
// that changes
static void drop_run_graph(hmn_ctx* ctx) {
  if (ctx->run_exec) cudaGraphExecDestroy(ctx->run_exec);
  ctx->run_exec = nullptr;
}

// host copy of axis a's array q (0 x, 1 dx, 2 dxi, 3 idx), offset +2
static const double* host_axis(const hmn_ctx* ctx, int a, int q) {
  const double* h = ctx->axis_h;
  for (int b = 0; b < a; b++) h += (size_t)4 * (ctx->n[b] + 4);
  return h + (size_t)q * (ctx->n[a] + 4) + 2;
}

// setup_grv_hyperbolic (gravity_hyperbolic.f90:336-405) on a spherical grid:
// lap_coeff(0..3) and the normalisation lap_coeff(-1) at coefficient index
// (i,j,k) >= -1, in the reference's operation order (the axisymmetric form
// for one phi cell, the 3-D form otherwise; Robin outer radius, gbtype 1)
static void sph_lap_coeffs(const hmn_ctx* ctx, const double* sinc, const double* sini, int i, int j, int k,
                           double c[5]) {
  const double *x1 = host_axis(ctx, 0, 0), *dx1 = host_axis(ctx, 0, 1), *dxi1 = host_axis(ctx, 0, 2);
  const double *dx2 = host_axis(ctx, 1, 1), *dxi2 = host_axis(ctx, 1, 2);
  const double *dx3 = host_axis(ctx, 2, 1), *dxi3 = host_axis(ctx, 2, 2), *idx3 = host_axis(ctx, 2, 3);
  const double* xi1 = ctx->xi1_h + 2;
  const int gie = ctx->n[0] - 1, gje = ctx->n[1] - 1;
  const double a = xi1[i], b = xi1[i - 1];
  if (ctx->n[2] == 1) {  // :336-363
    c[0] = -((a * a / dx1[i + 1] + b * b / dx1[i]) * sinc[j] * dxi2[j] +
             (sini[j] / dx2[j + 1] + sini[j - 1] / dx2[j]) * dxi1[i]);
    c[1] = a * a * sinc[j] * dxi2[j] / dx1[i + 1];
    c[2] = sini[j] * dxi1[i] / dx2[j + 1];
    c[3] = 0.0;
    if (i == 0 && ctx->xi1s > 0.0) c[0] = c[0] + b * b * sinc[j] * dxi2[j] / dx1[i];
    if (i == gie) {
      c[0] = c[0] + c[1] * x1[i] / x1[i + 1];
      c[1] = 0.0;
    }
    if (j == gje) {
      c[0] = c[0] + c[2];
      c[2] = 0.0;
    }
    c[4] = x1[i] * x1[i] * sinc[j] * dxi1[i] * dxi2[j];
  } else {  // :367-400
    c[0] = -((a * a / dx1[i + 1] + b * b / dx1[i]) * sinc[j] * dxi2[j] * dxi3[k] +
             (sini[j] / dx2[j + 1] + sini[j - 1] / dx2[j]) * dxi1[i] * dxi3[k] +
             (idx3[k] + idx3[k + 1]) * dxi1[i] * dxi2[j]);
    c[1] = a * a * sinc[j] * dxi2[j] * dxi3[k] / dx1[i + 1];
    c[2] = sini[j] * dxi1[i] * dxi3[k] / dx2[j + 1];
    c[3] = dxi1[i] * dxi2[j] / dx3[k + 1];
    if (j == gje) {
      c[0] = c[0] + c[2];
      c[2] = 0.0;
    }
    if (i == 0 && ctx->xi1s > 0.0) c[0] = c[0] + b * b * sinc[j] * dxi2[j] * dxi3[k] / dx1[i];
    if (i == gie) {
      c[0] = c[0] + c[1] * x1[i] / x1[i + 1];
      c[1] = 0.0;
    }
    c[4] = x1[i] * x1[i] * sinc[j] * dxi1[i] * dxi2[j] * dxi3[k];
  }
}

// metric.f90:53-100 for cylindrical coordinates with one phi cell (the
// axisymmetric R-z form; a solved phi axis is refused because gridset
// reads an unset width dxi2(js-2) for its ghost centres); no gravity or
// passive scalars
static int set_cylindrical(hmn_ctx* ctx, const hmn_metric* mt) {
  if (!mt || !mt->detg1 || !mt->idetg1 || !mt->sx1) return HMN_EINVAL;
  if (ctx->n[1] != 1 || ctx->par.gravswitch != 0 || ctx->par.nspc != 0 || !ctx->solve[0]) return HMN_EBADCFG;
  const int L1 = ctx->n[0] + 4;
  std::vector<double> h((size_t)6 * L1, 0.0);
  double *g1 = h.data(), *ig1 = g1 + L1, *s1 = ig1 + L1, *ar2 = s1 + 3 * L1;
  const double* xi = ctx->xi1_h;
  for (int s = 0; s < L1; s++) {
    g1[s] = mt->detg1[s];
    ig1[s] = mt->idetg1[s];
    s1[s] = mt->sx1[s];
    if (s > 0) ar2[s] = xi[s] * xi[s] - xi[s - 1] * xi[s - 1];
  }
  cudaFree(ctx->sphbuf);  // sized for this coordinate system
  ctx->sphbuf = nullptr;
  CK(cudaMalloc((void**)&ctx->sphbuf, h.size() * sizeof(double)), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->sphbuf, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->st), "metric");
  CK(cudaStreamSynchronize(ctx->st), "metric");
  SphGeo M{};
  const double* b = ctx->sphbuf;
  M.detg1 = b;
  M.idetg1 = b + L1;
  M.sx1 = b + 2 * L1;
  M.ar2 = b + 5 * L1;
  M.fac_j = 4.0;
  M.fac_k = 1.0;
  M.crd = 1;
  M.on = 1;
  ctx->G.sph = M;
  return HMN_OK;
}

// metric.f90:102-151 for spherical polar coordinates: the caller's 1-D
// factors plus the radial and polar products the kernels form the 2-D and
// 3-D factors from (same single IEEE operations as the reference); with
// self-gravity the Laplacian coefficient planes and the spherical dtg_unit.
extern "C" int hmn_set_metric(hmn_ctx* ctx, int crdnt, const hmn_metric* mt) {
  if (!ctx) return HMN_EINVAL;
  drop_run_graph(ctx);
  if (crdnt == 0) {
    ctx->G.sph = SphGeo{};
    retile(ctx);
    return HMN_OK;
  }
  if (crdnt == 1) return set_cylindrical(ctx, mt);
  if (crdnt != 2) return HMN_EBADCFG;
  if (!mt || !mt->detg1 || !mt->idetg1 || !mt->sx1 || !mt->sini || !mt->cosi || !mt->scot) return HMN_EINVAL;
  // single grids without passive scalars (either precision); r solved; self-gravity
  // on (r, theta) grids with one phi cell or on 3-D grids
  if (ctx->par.nspc != 0 || !ctx->solve[0]) return HMN_EBADCFG;
  const bool grav = ctx->par.gravswitch == 3;
  if (grav && (!ctx->solve[1] || !mt->sinc || !mt->sisin)) return HMN_EBADCFG;
  const int L1 = ctx->n[0] + 4, L2 = ctx->n[1] + 4;
  std::vector<double> h((size_t)6 * L1 + (size_t)5 * L2, 0.0);
  double *g1 = h.data(), *ig1 = g1 + L1, *s1 = ig1 + L1, *vr = s1 + L1, *hr2 = vr + L1, *ar2 = hr2 + L1;
  double *si = ar2 + L1, *ra2 = si + L2, *cd = ra2 + L2, *sc = cd + L2, *ss = sc + L2;
  const double* xi = ctx->xi1_h;
  for (int s = 0; s < L1; s++) {
    g1[s] = mt->detg1[s];
    ig1[s] = mt->idetg1[s];
    s1[s] = mt->sx1[s];
    hr2[s] = 0.5 * (xi[s] * xi[s]);
    if (s > 0) {
      vr[s] = (xi[s] * xi[s] * xi[s] - xi[s - 1] * xi[s - 1] * xi[s - 1]) / 3.0;
      ar2[s] = xi[s] * xi[s] - xi[s - 1] * xi[s - 1];
    }
  }
  for (int s = 0; s < L2; s++) {
    si[s] = mt->sini[s];
    sc[s] = mt->scot[s];
    ss[s] = mt->sisin ? mt->sisin[s] : 0.0;
    if (s > 0) {
      ra2[s] = 1.0 / (-mt->cosi[s] + mt->cosi[s - 1]);
      cd[s] = mt->cosi[s - 1] - mt->cosi[s];
    }
  }
  cudaFree(ctx->sphbuf);  // sized for this coordinate system
  ctx->sphbuf = nullptr;
  CK(cudaMalloc((void**)&ctx->sphbuf, h.size() * sizeof(double)), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->sphbuf, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->st), "metric");
  CK(cudaStreamSynchronize(ctx->st), "metric");
  SphGeo& M = ctx->G.sph;
  const double* b = ctx->sphbuf;
  M.detg1 = b;
  M.idetg1 = b + L1;
  M.sx1 = b + 2 * L1;
  M.vr = b + 3 * L1;
  M.hr2 = b + 4 * L1;
  M.ar2 = b + 5 * L1;
  M.sini = b + 6 * L1;
  M.ra2 = M.sini + L2;
  M.cd = M.sini + 2 * L2;
  M.scot = M.sini + 3 * L2;
  M.sisin = M.sini + 4 * L2;
  M.fac_j = ctx->n[1] == 1 ? 2.0 : 1.0;
  M.fac_k = ctx->n[2] == 1 ? 4.0 : 1.0;
  M.crd = 2;
  M.on = 1;
  retile(ctx);
  cudaFree(ctx->sincbuf);  // the angular-momentum weights of hmn_evo
  ctx->sincbuf = nullptr;
  if (mt->sinc) {
    CK(cudaMalloc((void**)&ctx->sincbuf, (size_t)L2 * sizeof(double)), "cudaMalloc");
    CK(cudaMemcpyAsync(ctx->sincbuf, mt->sinc, (size_t)L2 * sizeof(double), cudaMemcpyHostToDevice, ctx->st),
       "metric");
    CK(cudaStreamSynchronize(ctx->st), "metric");
  }
  ctx->xi1s = xi[1];  // xi1(is-1)
  if (grav) {
    // the Laplacian's 8 planes per cell: c0, the -x/+x/-y/+y/-z/+z weights, the normalisation
    const int n0 = ctx->n[0], n1 = ctx->n[1], n2 = ctx->n[2];
    const size_t P = ctx->plane;
    std::vector<double> lc((size_t)8 * P);
    const double *sinc = mt->sinc + 2, *sini = mt->sini + 2;
    for (int k = 0; k < n2; k++)
      for (int j = 0; j < n1; j++)
        for (int i = 0; i < n0; i++) {
          const size_t c = (size_t)i + (size_t)n0 * ((size_t)j + (size_t)n1 * k);
          double cc[5], cx[5], cy[5], cz[5];
          sph_lap_coeffs(ctx, sinc, sini, i, j, k, cc);
          sph_lap_coeffs(ctx, sinc, sini, i - 1, j, k, cx);
          sph_lap_coeffs(ctx, sinc, sini, i, j - 1, k, cy);
          sph_lap_coeffs(ctx, sinc, sini, i, j, k - 1, cz);
          const double v[8] = {cc[0], cx[1], cc[1], cy[2], cc[2], cz[3], cc[3], cc[4]};
          for (int q = 0; q < 8; q++) lc[(size_t)q * P + c] = v[q];
        }
    if (!ctx->hgc) CK(cudaMalloc((void**)&ctx->hgc, lc.size() * sizeof(double)), "cudaMalloc");
    if (!ctx->gin) CK(cudaMalloc((void**)&ctx->gin, (size_t)n1 * n2 * sizeof(double)), "cudaMalloc");
    CK(cudaMemcpyAsync(ctx->hgc, lc.data(), lc.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->st),
       "metric");
    CK(cudaMemsetAsync(ctx->gin, 0, (size_t)n1 * n2 * sizeof(double), ctx->st), "metric");
    // tools.f90:160-183 with dtgrav_cell on the spherical dvol and face areas (metric.f90:117-130)
    const double *dxi2 = host_axis(ctx, 1, 2), *dxi3 = host_axis(ctx, 2, 2);
    const double off0 = 1.0, off1 = 1.0, off2 = ctx->solve[2] ? 1.0 : 0.0;
    const double fj = M.fac_j, fk = M.fac_k;
    double m = INFINITY;
    for (int k = 0; k < n2; k++)
      for (int j = 0; j < n1; j++)
        for (int i = 0; i < n0; i++) {
          const double a = xi[i + 2], bb = xi[i + 1];
          const double cdj = mt->cosi[j + 1] - mt->cosi[j + 2];
          const double dvol = (a * a * a - bb * bb * bb) / 3.0 * cdj * dxi3[k] * fj * fk;
          const double sa1 = 0.5 * (bb * bb) * cdj * dxi3[k] * fj * fk + 0.5 * (a * a) * cdj * dxi3[k] * fj * fk;
          const double sa2 = 0.5 * mt->sini[j + 1] * (a * a - bb * bb) * dxi3[k] * fk +
                             0.5 * mt->sini[j + 2] * (a * a - bb * bb) * dxi3[k] * fk;
          const double sa3 = 0.5 * (a * a - bb * bb) * dxi2[j] * fj + 0.5 * (a * a - bb * bb) * dxi2[j] * fj;
          const double v = dvol / (1.0 * (off0 * sa1 + off1 * sa2 + off2 * sa3));
          m = v < m ? v : m;
        }
    ctx->dtg_unit = m;
    CK(cudaMemcpyAsync(&ctx->sc->dtg_unit, &ctx->dtg_unit, sizeof(double), cudaMemcpyHostToDevice, ctx->st),
       "metric");
    CK(cudaStreamSynchronize(ctx->st), "metric");
  }
  return HMN_OK;
}

extern "C" int hmn_upload(hmn_ctx* ctx, const double* u, const double* const prim[9], const double* grvphi,
                          const double* grvpsi) {
  if (!ctx) return HMN_EINVAL;
  const size_t gp = ghosted_plane(ctx);
  int rc;
  if (u) {
    rc = to_device(ctx, ctx->buf[0], u, ctx->nvar, gp);
    if (rc) return rc;
    ctx->phifac = 1.0;
  }
  double* Pc = ctx->pbuf[ctx->pcur];
  if (prim) {
    // the primitives as the reference holds them after initialcondition;
    // eint as pressure -> internalenergy derives it (eos.f90:805-842)
    const size_t P = ctx->plane;
    for (int q = 0; q < 9; q++) {
      if (prim[q]) {
        rc = to_device(ctx, Pc + q * P, prim[q], 1, gp);
        if (rc) return rc;
      } else {
        CK(cudaMemsetAsync(Pc + q * P, 0, P * sizeof(double), ctx->st), "memset");
      }
    }
    CK(launch_prim_init(Pc, ctx->plane, ctx->mag, blocks_for(ctx), ctx->st), "prim init");
    ctx->launches += 1;
    ctx->phifac = 1.0;
  } else if (u) {
    CK(launch_prim_from_u(ctx->buf[0], Pc, ctx->plane, ctx->mag, ctx->glm, blocks_for(ctx), ctx->st), "prim");
    ctx->launches += 1;
  }
  if (grvphi && ctx->par.gravswitch == 3) {
    rc = to_device(ctx, ctx->gphi[ctx->gcur], grvphi, 1, gp);
    if (rc) return rc;
  }
  if (grvpsi && ctx->par.gravswitch == 3) {
    rc = to_device(ctx, ctx->gpsi[ctx->gcur], grvpsi, 1, gp);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(ctx->st), "sync");
  return HMN_OK;
}

// pull the scalars and the error word; returns the error code if any kernel recorded one
static int fetch_scalars(hmn_ctx* ctx) {
  CK(cudaMemcpyAsync(ctx->sc_h, ctx->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->st), "scalars");
  CK(cudaStreamSynchronize(ctx->st), "sync");
  if (ctx->sc_h->err_code) return ctx->sc_h->err_code;
  return HMN_OK;
}

static int push_times(hmn_ctx* ctx, double time, double t_out, double t_end) {
  // only the three time fields change; write them individually
  double tv[3] = {time, t_out, t_end};
  static_assert(offsetof(DevScalars, t_out) == offsetof(DevScalars, time) + sizeof(double), "layout");
  static_assert(offsetof(DevScalars, t_end) == offsetof(DevScalars, time) + 2 * sizeof(double), "layout");
  double* dst = &ctx->sc->time;
  CK(cudaMemcpyAsync(dst, tv, sizeof(tv), cudaMemcpyHostToDevice, ctx->st), "times");
  CK(cudaMemsetAsync(&ctx->sc->done, 0, sizeof(int), ctx->st), "times");
  CK(cudaStreamSynchronize(ctx->st), "sync");
  return HMN_OK;
}

static int enqueue_cfl(hmn_ctx* ctx) {
  CK(launch_cfl(ctx->G, ctx->pbuf[ctx->pcur], ctx->plane, ctx->par.gamma, ctx->sc, ctx->mag, blocks_for(ctx),
                ctx->st),
     "cfl");
  ctx->launches += 2;
  return HMN_OK;
}

extern "C" int hmn_timestep(hmn_ctx* ctx, double time, double t_out, double t_end, double* dt, double* ch) {
  if (!ctx) return HMN_EINVAL;
  if (slab_exchanges(ctx)) return HMN_EBADCFG;  // dt is a reduction over all slabs
  int rc = push_times(ctx, time, t_out, t_end);
  if (rc) return rc;
  rc = enqueue_cfl(ctx);
  if (rc) return rc;
  rc = fetch_scalars(ctx);
  if (dt) *dt = ctx->sc_h->dt;
  if (ch) *ch = ctx->sc_h->ch;
  return rc;
}

static void rk_coeff(int iter, int type, double* faco, double* fact, double* facn) {
  // rungekutta.f90:146-183
  if (type == 3) {
    if (iter == 1) { *faco = 1.0; *fact = 1.0; *facn = 0.0; }
    else if (iter == 2) { *faco = 0.75; *fact = 0.25; *facn = *fact; }
    else { *faco = 1.0 / 3.0; *fact = 2.0 / 3.0; *facn = *fact; }
  } else if (type == 2) {
    if (iter == 1) { *faco = 1.0; *fact = 1.0; *facn = 0.0; }
    else { *faco = 0.5; *fact = 0.5; *facn = *fact; }
  } else {
    *faco = 1.0; *fact = 1.0; *facn = 0.0;
  }
}

// RK stage s (1..rktype) of the current step; the last stage also does the
// step's buffer bookkeeping
// The arguments of RK stage s (1-based) on the state in primitive buffer
// pcur: buffer roles, RK coefficients, scalars (hydro.f90:35-41).
static StageArgs stage_args(hmn_ctx* ctx, int s, int pcur) {
  const int rk = ctx->par.rktype;
  StageArgs a;
  memset(&a, 0, sizeof(a));
  rk_coeff(s, rk, &a.faco, &a.fact, &a.facn);
  a.uorg = ctx->buf[0];
  a.pin = ctx->pbuf[pcur];
  a.pout = ctx->pbuf[1 - pcur];
  if (s == 1) {
    a.phifac = ctx->phifac;
    a.ucur = ctx->buf[0];
    a.uout = ctx->buf[1];
  } else if (s == 2) {
    a.ucur = ctx->buf[1];
    a.uout = rk == 2 ? ctx->buf[0] : ctx->buf[2];
    a.phifac = 1.0;
  } else {
    a.ucur = ctx->buf[2];
    a.uout = ctx->buf[0];
    a.phifac = 1.0;
  }
  a.gphi = ctx->par.gravswitch == 3 ? ctx->gphi[ctx->gcur] : nullptr;
  a.sc = ctx->sc;
  a.plane = ctx->plane;
  a.gamma = ctx->par.gamma;
  a.gm1 = ctx->par.gamma - 1.0;
  a.limiter = ctx->par.limiter;
  a.nvar = ctx->nvar;
  for (int d = 0; d < 3; d++) {
    a.tile[d] = ctx->tile[d];
    a.tiles[d] = ctx->tiles[d];
  }
  a.stage = s;
  a.nspc = ctx->par.nspc;
  a.spcorg = ctx->spcorg;
  return a;
}

static int enqueue_stage(hmn_ctx* ctx, int s) {
  const int rk = ctx->par.rktype;
  for (int a = 0; a < 3; a++)
    for (int io = 0; io < 2; io++)
      if (ctx->solve[a] && (ctx->bc[a][io][0] >= 9 || ctx->bc[a][io][1] >= 9) && !ctx->G.dir[a][io])
        return HMN_EBADCFG;  // codes 9 and 10 need hmn_set_dirichlet first
  if (ctx->solve[2] && ctx->bc[2][0][0] == 10 && !ctx->fb) return HMN_EBADCFG;  // and hmn_set_flux_boundary
  {
    StageArgs a = stage_args(ctx, s, ctx->pcur);
    if (ctx->zpush_on) {  // read the halos of this parity, store into the other
      ctx->G.zhalo[0] = ctx->zrecv[0][ctx->zpar];
      ctx->G.zhalo[1] = ctx->zrecv[1][ctx->zpar];
      a.push[0] = ctx->zpush[0][ctx->zpar ^ 1];
      a.push[1] = ctx->zpush[1][ctx->zpar ^ 1];
    }
    const TmaMaps* tm = ctx->tma_ok ? &ctx->tmaps[ctx->pcur] : nullptr;
    if (ctx->par.precision == 1)
      CK(launch_stage_mixed(ctx->G, a, ctx->mag, ctx->glm, tm, ctx->st), "stage");
    else
      CK(launch_stage(ctx->G, a, ctx->mag, ctx->glm, tm, ctx->st), "stage");
    ctx->launches += 1;
    ctx->pcur = 1 - ctx->pcur;
    if (ctx->zpush_on) ctx->zpar ^= 1;
  }
  if (s == rk) {
    if (rk == 1) {
      double* t = ctx->buf[0];
      ctx->buf[0] = ctx->buf[1];
      ctx->buf[1] = t;
    }
    ctx->phifac = 1.0;
  }
  return HMN_OK;
}

static int enqueue_hydro(hmn_ctx* ctx) {
  for (int s = 1; s <= ctx->par.rktype; s++) {
    int rc = enqueue_stage(ctx, s);
    if (rc) return rc;
  }
  return HMN_OK;
}

extern "C" int hmn_hydro_step(hmn_ctx* ctx) {
  if (!ctx) return HMN_EINVAL;
  if (slab_exchanges(ctx)) return HMN_EBADCFG;  // the halos must be exchanged between stages
  return enqueue_hydro(ctx);
}

// ---------------------------------------------------------------------------
// boundary code 9: ghost values given by the host (d0, p0, v10.., b10.., spc0
// of module physval, boundarycondition.f90:104-115,196-212)

extern "C" int hmn_set_dirichlet(hmn_ctx* ctx, int axis, int side, const double* vals) {
  if (!ctx || !vals || axis < 0 || axis > 2 || side < 0 || side > 1) return HMN_EINVAL;
  const int oa0 = axis == 0 ? 1 : 0, oa1 = axis == 2 ? 1 : 2;
  const size_t m = (size_t)(8 + ctx->par.nspc) * 2 * (size_t)ctx->n[oa0] * ctx->n[oa1];
  if (!ctx->dir[axis][side]) CK(cudaMalloc((void**)&ctx->dir[axis][side], m * sizeof(double)), "dirichlet");
  CK(cudaMemcpyAsync(ctx->dir[axis][side], vals, m * sizeof(double), cudaMemcpyHostToDevice, ctx->st),
     "dirichlet");
  CK(cudaStreamSynchronize(ctx->st), "sync");
  drop_run_graph(ctx);
  ctx->G.dir[axis][side] = ctx->dir[axis][side];
  return HMN_OK;
}

// boundary code 10 (fluxboundary.f90:42-87): the flux through the inner x3
// face, 9 conserved slots and then the scalars; the reference sets it for
// the wind-tunnel inflow
extern "C" int hmn_set_flux_boundary(hmn_ctx* ctx, int axis, int side, const double* flux) {
  if (!ctx || !flux) return HMN_EINVAL;
  if (axis != 2 || side != 0 || ctx->bc[2][0][0] != 10) return HMN_EBADCFG;
  const size_t m = (size_t)(9 + ctx->par.nspc);
  if (!ctx->fb) CK(cudaMalloc((void**)&ctx->fb, (9 + 8) * sizeof(double)), "flux boundary");
  CK(cudaMemcpyAsync(ctx->fb, flux, m * sizeof(double), cudaMemcpyHostToDevice, ctx->st), "flux boundary");
  CK(cudaStreamSynchronize(ctx->st), "sync");
  drop_run_graph(ctx);
  ctx->G.fb = ctx->G.zhalo[0] ? nullptr : ctx->fb;  // a slab above the first has no such face
  return HMN_OK;
}

// ---------------------------------------------------------------------------
// slab decomposition along z (mpi_domain.F90's role for this path)

extern "C" size_t hmn_slab_halo_bytes(const hmn_ctx* ctx) {
  if (!ctx) return 0;
  return (size_t)(10 + ctx->par.nspc) * 2 * (size_t)ctx->n[0] * ctx->n[1] * sizeof(double);
}

extern "C" int hmn_set_slab(hmn_ctx* ctx, double* send_lo, double* send_hi, const double* recv_lo,
                            const double* recv_hi, int wrap_lo, int wrap_hi) {
  if (!ctx) return HMN_EINVAL;
  if (!ctx->solve[2] || ctx->n[2] < 2 || (ctx->par.gravswitch != 0 && ctx->G.sph.on)) return HMN_EBADCFG;
  if ((recv_lo && !send_lo) || (recv_hi && !send_hi)) return HMN_EINVAL;
  ctx->zsend[0] = send_lo;
  ctx->zsend[1] = send_hi;
  drop_run_graph(ctx);
  ctx->G.zhalo[0] = recv_lo;
  ctx->G.zhalo[1] = recv_hi;
  ctx->G.fb = recv_lo ? nullptr : ctx->fb;  // code 10 lives on the grid's inner z face only
  ctx->G.zwrap[0] = recv_lo && wrap_lo ? 1 : 0;
  ctx->G.zwrap[1] = recv_hi && wrap_hi ? 1 : 0;
  return HMN_OK;
}

extern "C" size_t hmn_slab_gravity_halo_bytes(const hmn_ctx* ctx) {
  if (!ctx) return 0;
  return (size_t)ctx->n[0] * ctx->n[1] * sizeof(double);
}

// Slab decomposition with hyperbolic self-gravity: the potential's layer
// beyond each neighbouring z face comes from the neighbour (its bottom or
// top layer, exchanged by the caller before every gravity sub-stage and
// once after the last) for the Laplacian and for the force of the hydro
// stages.  After hmn_set_slab, on the faces it gave halos for.
extern "C" int hmn_set_slab_gravity(hmn_ctx* ctx, double* send_lo, double* send_hi, const double* recv_lo,
                                    const double* recv_hi) {
  if (!ctx) return HMN_EINVAL;
  if (ctx->par.gravswitch != 3 || ctx->G.sph.on || ctx->zpush_on) return HMN_EBADCFG;
  if ((recv_lo != nullptr) != (ctx->G.zhalo[0] != nullptr) || (recv_hi != nullptr) != (ctx->G.zhalo[1] != nullptr) ||
      (recv_lo && !send_lo) || (recv_hi && !send_hi))
    return HMN_EINVAL;
  ctx->gsend[0] = send_lo;
  ctx->gsend[1] = send_hi;
  ctx->G.ghalo[0] = recv_lo;
  ctx->G.ghalo[1] = recv_hi;
  drop_run_graph(ctx);
  return HMN_OK;
}

// the potential's halo faces match the primitives' (a slab with gravity
// exchanges both)
static bool gravity_halos_set(const hmn_ctx* ctx) {
  return (ctx->G.zhalo[0] == nullptr || ctx->G.ghalo[0] != nullptr) &&
         (ctx->G.zhalo[1] == nullptr || ctx->G.ghalo[1] != nullptr);
}

extern "C" int hmn_pack_gravity_halos(hmn_ctx* ctx) {
  if (!ctx) return HMN_EINVAL;
  if (ctx->par.gravswitch != 3) return HMN_EBADCFG;
  const size_t layer = (size_t)ctx->n[0] * ctx->n[1];
  const double* phi = ctx->gphi[ctx->gcur];
  if (ctx->gsend[0])
    CK(cudaMemcpyAsync(ctx->gsend[0], phi, layer * sizeof(double), cudaMemcpyDeviceToDevice, ctx->st), "pack");
  if (ctx->gsend[1])
    CK(cudaMemcpyAsync(ctx->gsend[1], phi + (size_t)(ctx->n[2] - 1) * layer, layer * sizeof(double),
                       cudaMemcpyDeviceToDevice, ctx->st),
       "pack");
  return HMN_OK;
}

extern "C" int hmn_gravity_unit(hmn_ctx* ctx, double* dtg_unit) {
  if (!ctx || !dtg_unit) return HMN_EINVAL;
  *dtg_unit = ctx->dtg_unit;
  return HMN_OK;
}

// the grid-wide dtg_unit (tools.f90:160-183 is a minimum over all cells):
// slabs of one grid set the minimum over the slabs
extern "C" int hmn_set_gravity_unit(hmn_ctx* ctx, double dtg_unit) {
  if (!ctx || !(dtg_unit > 0.0)) return HMN_EINVAL;
  ctx->dtg_unit = dtg_unit;
  CK(cudaMemcpyAsync(&ctx->sc->dtg_unit, &ctx->dtg_unit, sizeof(double), cudaMemcpyHostToDevice, ctx->st),
     "gravity unit");
  CK(cudaStreamSynchronize(ctx->st), "gravity unit");
  drop_run_graph(ctx);
  return HMN_OK;
}

// Push exchange between z slabs: each stage's kernel stores its two bottom
// and two top layers into the neighbours' halo buffers as it writes them
// (on several GPUs the buffers are the neighbours' memory: the exchange
// rides inside the stage).  Buffers alternate by stage parity, so a stage
// never overwrites halos a neighbour may still be reading; between stages
// every slab must have finished the previous one (the caller's barrier).
extern "C" int hmn_set_slab_push(hmn_ctx* ctx, const double* const recv_lo[2], const double* const recv_hi[2],
                                 double* const push_lo[2], double* const push_hi[2], int wrap_lo, int wrap_hi) {
  if (!ctx || !recv_lo || !recv_hi || !push_lo || !push_hi) return HMN_EINVAL;
  if (!ctx->solve[0] || !ctx->solve[1] || !ctx->solve[2] || ctx->n[2] < 2 || ctx->par.gravswitch != 0 ||
      ctx->G.sph.on)
    return HMN_EBADCFG;  // 3-D Cartesian grids
  for (int q = 0; q < 2; q++)
    if ((recv_lo[q] == nullptr) != (push_lo[q] == nullptr) || (recv_hi[q] == nullptr) != (push_hi[q] == nullptr))
      return HMN_EINVAL;
  for (int q = 0; q < 2; q++) {
    ctx->zrecv[0][q] = recv_lo[q];
    ctx->zrecv[1][q] = recv_hi[q];
    ctx->zpush[0][q] = push_lo[q];
    ctx->zpush[1][q] = push_hi[q];
  }
  ctx->zpush_on = 1;
  ctx->zpar = 0;
  ctx->zsend[0] = ctx->zsend[1] = nullptr;
  drop_run_graph(ctx);
  ctx->G.zhalo[0] = recv_lo[0];
  ctx->G.zhalo[1] = recv_hi[0];
  ctx->G.fb = recv_lo[0] ? nullptr : ctx->fb;
  ctx->G.zwrap[0] = recv_lo[0] && wrap_lo ? 1 : 0;
  ctx->G.zwrap[1] = recv_hi[0] && wrap_hi ? 1 : 0;
  return HMN_OK;
}

// push mode: store the current state's boundary layers into the neighbours'
// halo buffers of the current parity (after an upload, before the first stage)
static int push_current_halos(hmn_ctx* ctx) {
  CK(launch_pack_zhalos(ctx->pbuf[ctx->pcur], ctx->n, 10 + ctx->par.nspc, ctx->zpush[0][ctx->zpar],
                        ctx->zpush[1][ctx->zpar], blocks_for(ctx), ctx->st),
     "push halos");
  ctx->launches += 1;
  return HMN_OK;
}

extern "C" int hmn_pack_halos(hmn_ctx* ctx) {
  if (!ctx) return HMN_EINVAL;
  if (ctx->zpush_on) return push_current_halos(ctx);
  if (!slab_exchanges(ctx)) return HMN_OK;  // a single slab has nothing to send
  CK(launch_pack_zhalos(ctx->pbuf[ctx->pcur], ctx->n, 10 + ctx->par.nspc, ctx->zsend[0], ctx->zsend[1],
                        blocks_for(ctx), ctx->st),
     "pack halos");
  ctx->launches += 1;
  return HMN_OK;
}

extern "C" int hmn_hydro_stage(hmn_ctx* ctx, int stage) {
  if (!ctx || stage < 1 || stage > ctx->par.rktype) return HMN_EINVAL;
  if (ctx->par.gravswitch == 3 && !gravity_halos_set(ctx)) return HMN_EBADCFG;  // the force needs them
  return enqueue_stage(ctx, stage);
}

extern "C" int hmn_cfl_local(hmn_ctx* ctx, double time, double t_out, double t_end) {
  if (!ctx) return HMN_EINVAL;
  int rc = push_times(ctx, time, t_out, t_end);
  if (rc) return rc;
  CK(launch_cfl_cells(ctx->G, ctx->pbuf[ctx->pcur], ctx->plane, ctx->par.gamma, ctx->sc, ctx->mag,
                      blocks_for(ctx), ctx->st),
     "cfl");
  ctx->launches += 1;
  return HMN_OK;
}

extern "C" int hmn_cfl_partials(hmn_ctx* ctx, double** min_dti, double** cfmax) {
  if (!ctx) return HMN_EINVAL;
  static_assert(sizeof(unsigned long long) == sizeof(double), "bit patterns");
  if (min_dti) *min_dti = reinterpret_cast<double*>(&ctx->sc->min_dti_bits);
  if (cfmax) *cfmax = reinterpret_cast<double*>(&ctx->sc->cfmax_bits);
  return HMN_OK;
}

extern "C" int hmn_cfl_finalize(hmn_ctx* ctx, double* dt, double* ch) {
  if (!ctx) return HMN_EINVAL;
  CK(launch_cfl_finalize(ctx->sc, ctx->st), "cfl");
  ctx->launches += 1;
  int rc = fetch_scalars(ctx);
  if (dt) *dt = ctx->sc_h->dt;
  if (ch) *ch = ctx->sc_h->ch;
  return rc;
}

extern "C" int hmn_phidamp(hmn_ctx* ctx) {
  if (!ctx) return HMN_EINVAL;
  ctx->phifac = ctx->phifac * std::exp(-ctx->par.alpha9wave * ctx->par.courant);  // source.f90:253
  return HMN_OK;
}

// hg_boundary_conditions on a spherical grid: of the ghost images only the
// one beyond r = xi1s enters the Laplacian with a non-zero weight, and it
// keeps the value of this pass through the next call's sub-cycles
// (gravity_hyperbolic.f90:186-190); the stage kernels form the others.
static int sph_gravity_boundary(hmn_ctx* ctx) {
  if (!ctx->G.sph.on || !ctx->gin) return HMN_OK;
  CK(cudaMemcpy2DAsync(ctx->gin, sizeof(double), ctx->gphi[ctx->gcur], (size_t)ctx->n[0] * sizeof(double),
                       sizeof(double), (size_t)ctx->n[1] * ctx->n[2], cudaMemcpyDeviceToDevice, ctx->st),
     "gravity boundary");
  return HMN_OK;
}

// Plan the sub-cycles of gravity_hyperbolic.f90:19-60 for the step
// [time, time + dt]: *nsub = tngrav x grktype sub-stages (0 at tn = 0, where
// grav_init_other only sets the clock).
extern "C" int hmn_gravity_begin(hmn_ctx* ctx, double time, double dt, int tn, int* nsub) {
  if (!ctx || !nsub) return HMN_EINVAL;
  *nsub = 0;
  ctx->gv_left = 0;
  if (ctx->par.gravswitch != 3) return HMN_OK;
  if (!ctx->G.sph.on && ctx->dim != 3) return HMN_EBADCFG;  // the Cartesian solver is 3-D
  if (!gravity_halos_set(ctx)) return HMN_EBADCFG;
  if (tn == 0) {
    ctx->grvtime = time;
    return HMN_OK;
  }
  // cgrav and dtgrav of the last hmn_timestep
  int rc = fetch_scalars(ctx);
  if (rc) return rc;
  const double cgrav = ctx->sc_h->cgrav;
  const double dtgrav = ctx->sc_h->dtgrav;
  const int tngrav = (int)std::ceil((time + dt - ctx->grvtime) / dtgrav);  // gravity_hyperbolic.f90:33-34
  if (tngrav < 1) return HMN_OK;
  ctx->gv_dtgrav = (time + dt - ctx->grvtime) / (double)tngrav;
  ctx->gv_cgrav = cgrav;
  ctx->gv_left = tngrav;
  ctx->gv_g = 1;
  *nsub = tngrav * ctx->par.grktype;
  return HMN_OK;
}

// The next RK sub-stage of the planned sub-cycles (hyperbolic_gravity_step,
// gravity_hyperbolic.f90:62-110); the last sub-stage of a cycle advances the
// gravity clock.
extern "C" int hmn_gravity_substage(hmn_ctx* ctx) {
  if (!ctx) return HMN_EINVAL;
  if (ctx->gv_left < 1) return HMN_EBADCFG;
  const int g = ctx->gv_g;
  const double cgrav = ctx->gv_cgrav, dtgrav = ctx->gv_dtgrav;
  if (g == 1) ctx->gv_damp = std::exp(-(1.0 - ctx->cgrav_old / cgrav + ctx->par.alphagrv * ctx->par.hgcfl));
  double faco, fact, facn;
  rk_coeff(g, ctx->par.grktype, &faco, &fact, &facn);
  HGArgs a;
  memset(&a, 0, sizeof(a));
  a.phi_in = ctx->gphi[ctx->gcur];
  a.psi_in = ctx->gpsi[ctx->gcur];
  a.phi_out = ctx->gphi[1 - ctx->gcur];
  a.psi_out = ctx->gpsi[1 - ctx->gcur];
  a.org_phi = ctx->gorg[0];
  a.org_psi = ctx->gorg[1];
  a.dens = ctx->pbuf[ctx->pcur];  // density plane of the state at the gravity call
  a.plane = ctx->plane;
  a.faco = faco;
  a.facn = facn;
  a.fdc = fact * dtgrav * cgrav;
  a.fourpiG = 4.0 * M_PI * ctx->par.G;
  a.damp = ctx->gv_damp;
  a.stage1 = g == 1;
  a.last = g == ctx->par.grktype;
  a.sc = ctx->sc;
  a.lc = ctx->hgc;
  a.gin = ctx->gin;
  a.uni = ctx->hg_uni && !ctx->G.sph.on;
  a.urcn_ok = ctx->hg_urcn_ok;
  a.uc0 = ctx->hg_c0;
  for (int d = 0; d < 3; d++) {
    a.ucm[d] = ctx->hg_cm[d];
    a.ucp[d] = ctx->hg_cp[d];
  }
  a.ucn = ctx->hg_cn;
  a.urcn = ctx->hg_rcn;
  if (ctx->G.sph.on)
    CK(launch_hg_stage_sph(ctx->G, a, ctx->st), "hg stage");
  else
    CK(launch_hg_stage(ctx->G, a, blocks_for(ctx), ctx->st), "hg stage");
  ctx->launches += 1;
  ctx->gcur = 1 - ctx->gcur;
  if (g == ctx->par.grktype) {
    ctx->grvtime = ctx->grvtime + dtgrav;
    ctx->cgrav_old = cgrav;
    ctx->gv_left -= 1;
    ctx->gv_g = 1;
  } else {
    ctx->gv_g = g + 1;
  }
  return HMN_OK;
}

extern "C" int hmn_gravity_step(hmn_ctx* ctx, double time, double dt, int tn) {
  if (!ctx) return HMN_EINVAL;
  if (ctx->par.gravswitch != 3) return HMN_OK;
  if (ctx->G.ghalo[0] || ctx->G.ghalo[1]) return HMN_EBADCFG;  // a slab exchanges between sub-stages
  int nsub = 0;
  int rc = hmn_gravity_begin(ctx, time, dt, tn, &nsub);
  if (rc) return rc;
  if (tn != 0 && nsub == 0) return HMN_OK;
  for (int l = 0; l < nsub; l++) {
    rc = hmn_gravity_substage(ctx);
    if (rc) return rc;
  }
  return sph_gravity_boundary(ctx);
}

// evo_output (output.f90:147-275): the grid's totals of the current state,
// summed per block and then over blocks in a fixed order.
extern "C" int hmn_evo(hmn_ctx* ctx, double out[10]) {
  if (!ctx || !out) return HMN_EINVAL;
  const int nb = blocks_for(ctx);
  if (!ctx->evobuf)
    CK(cudaMalloc((void**)&ctx->evobuf, ((size_t)ctx->nsm * 8 + 1) * kEvoQ * sizeof(double)), "cudaMalloc");
  double* tot = ctx->evobuf + (size_t)nb * kEvoQ;
  const double* gphi = ctx->par.gravswitch == 3 ? ctx->gphi[ctx->gcur] : nullptr;
  CK(launch_evo(ctx->G, ctx->pbuf[ctx->pcur], ctx->plane, gphi, ctx->G.sph.crd == 2 ? ctx->sincbuf : nullptr,
                ctx->evobuf, nb, tot, ctx->st),
     "evo");
  ctx->launches += 2;
  double h[kEvoQ];
  CK(cudaMemcpyAsync(h, tot, sizeof(h), cudaMemcpyDeviceToHost, ctx->st), "evo");
  CK(cudaStreamSynchronize(ctx->st), "evo");
  // Mtot, Etot, Eitot, Ektot = 0.5 sum, Egtot, Mbound, Ebound, Jbound, Ebtot = 0.5 sum, Jtot
  for (int q = 0; q < kEvoQ; q++) out[q] = h[q];
  out[3] = 0.5 * h[3];
  out[8] = 0.5 * h[8];
  return HMN_OK;
}

extern "C" int hmn_set_gravity_clock(hmn_ctx* ctx, double grvtime, double cgrav_old) {
  if (!ctx) return HMN_EINVAL;
  ctx->grvtime = grvtime;
  ctx->cgrav_old = cgrav_old;
  return HMN_OK;
}

extern "C" int hmn_gravity_clock(hmn_ctx* ctx, double* grvtime, double* cgrav_old) {
  if (!ctx) return HMN_EINVAL;
  if (grvtime) *grvtime = ctx->grvtime;
  if (cgrav_old) *cgrav_old = ctx->cgrav_old;
  return HMN_OK;
}

extern "C" int hmn_download(hmn_ctx* ctx, double* u, double* const prim[9], double* grvphi, double* grvpsi) {
  if (!ctx) return HMN_EINVAL;
  const size_t gp = ghosted_plane(ctx);
  int rc;
  if (u) {
    rc = to_host(ctx, u, ctx->buf[0], ctx->nvar, gp);
    if (rc) return rc;
  }
  if (prim) {
    CK(launch_prim_out(ctx->pbuf[ctx->pcur], ctx->plane, ctx->phifac, ctx->par.gamma - 1.0, ctx->prim_out,
                       ctx->prim_out + 9 * ctx->plane, blocks_for(ctx), ctx->st),
       "prim");
    ctx->launches += 1;
    for (int q = 0; q < 9; q++) {
      if (!prim[q]) continue;
      rc = to_host(ctx, prim[q], ctx->prim_out + q * ctx->plane, 1, gp);
      if (rc) return rc;
    }
  }
  if (grvphi && ctx->par.gravswitch == 3) {
    rc = to_host(ctx, grvphi, ctx->gphi[ctx->gcur], 1, gp);
    if (rc) return rc;
  }
  if (grvpsi && ctx->par.gravswitch == 3) {
    rc = to_host(ctx, grvpsi, ctx->gpsi[ctx->gcur], 1, gp);
    if (rc) return rc;
  }
  return fetch_scalars(ctx);
}

// ---------------------------------------------------------------------------
// asynchronous checkpoint (the data of output.f90:697-795 write_bin)

static int ck_planes(const hmn_ctx* ctx) { return ctx->nvar + 9 + 2 + ctx->par.nspc; }

static int ck_ensure(hmn_ctx* ctx) {
  if (ctx->ck_dev) return HMN_OK;
  const size_t bytes = (size_t)ck_planes(ctx) * ctx->plane * sizeof(double);
  CK(cudaStreamCreateWithFlags(&ctx->cst, cudaStreamNonBlocking), "checkpoint stream");
  CK(cudaEventCreateWithFlags(&ctx->ck_snap, cudaEventDisableTiming), "checkpoint event");
  CK(cudaEventCreateWithFlags(&ctx->ck_done, cudaEventDisableTiming), "checkpoint event");
  CK(cudaMalloc((void**)&ctx->ck_dev, bytes), "checkpoint buffer");
  CK(cudaMallocHost((void**)&ctx->ck_h, bytes), "checkpoint staging");
  return HMN_OK;
}

extern "C" int hmn_checkpoint_wait(hmn_ctx* ctx) {
  if (!ctx) return HMN_EINVAL;
  if (!ctx->ck_pending) return HMN_OK;
  CK(cudaEventSynchronize(ctx->ck_done), "checkpoint copy");
  ctx->ck_pending = 0;
  const size_t P = ctx->plane;
  const size_t gp = ghosted_plane(ctx);
  auto place = [&](double* dst, const double* src, int nplanes) {
    if (!dst) return;
    if (ctx->ghost == 0) {
      memcpy(dst, src, (size_t)nplanes * P * sizeof(double));
      return;
    }
    size_t o = 0;
    for (int q = 0; q < nplanes; q++)
      for (int k = 0; k < ctx->n[2]; k++)
        for (int j = 0; j < ctx->n[1]; j++)
          for (int i = 0; i < ctx->n[0]; i++) dst[q * gp + ghosted_index(ctx, i, j, k)] = src[o++];
  };
  place(ctx->ck_u, ctx->ck_h, ctx->nvar);
  for (int q = 0; q < 9; q++) place(ctx->ck_prim[q], ctx->ck_h + (size_t)(ctx->nvar + q) * P, 1);
  place(ctx->ck_gphi, ctx->ck_h + (size_t)(ctx->nvar + 9) * P, 1);
  place(ctx->ck_gpsi, ctx->ck_h + (size_t)(ctx->nvar + 10) * P, 1);
  if (ctx->ck_spc) {  // species fastest, as hmn_download_scalars
    const int ns = ctx->par.nspc;
    const double* src = ctx->ck_h + (size_t)(ctx->nvar + 11) * P;
    size_t o = 0;
    for (int k = 0; k < ctx->n[2]; k++)
      for (int j = 0; j < ctx->n[1]; j++)
        for (int i = 0; i < ctx->n[0]; i++, o++) {
          const size_t g = ghosted_index(ctx, i, j, k);
          for (int n = 0; n < ns; n++) ctx->ck_spc[(size_t)ns * g + n] = src[(size_t)n * P + o];
        }
  }
  return HMN_OK;
}

extern "C" int hmn_checkpoint_begin(hmn_ctx* ctx, double* u, double* const prim[9], double* grvphi,
                                    double* grvpsi, double* spc) {
  if (!ctx) return HMN_EINVAL;
  int rc = hmn_checkpoint_wait(ctx);  // one checkpoint in flight at a time
  if (rc) return rc;
  rc = ck_ensure(ctx);
  if (rc) return rc;
  const size_t P = ctx->plane;
  double* const du = ctx->ck_dev;
  double* const dp = ctx->ck_dev + (size_t)ctx->nvar * P;
  double* const dg = ctx->ck_dev + (size_t)(ctx->nvar + 9) * P;
  // device snapshot on the step stream, ordered after the work enqueued so far
  if (u) CK(cudaMemcpyAsync(du, ctx->buf[0], (size_t)ctx->nvar * P * sizeof(double), cudaMemcpyDeviceToDevice,
                            ctx->st), "checkpoint snapshot");
  CK(launch_prim_out(ctx->pbuf[ctx->pcur], P, ctx->phifac, ctx->par.gamma - 1.0, dp, nullptr, blocks_for(ctx),
                     ctx->st),
     "checkpoint snapshot");
  ctx->launches += 1;
  const bool grav = ctx->par.gravswitch == 3;
  if (grav && grvphi)
    CK(cudaMemcpyAsync(dg, ctx->gphi[ctx->gcur], P * sizeof(double), cudaMemcpyDeviceToDevice, ctx->st),
       "checkpoint snapshot");
  if (grav && grvpsi)
    CK(cudaMemcpyAsync(dg + P, ctx->gpsi[ctx->gcur], P * sizeof(double), cudaMemcpyDeviceToDevice, ctx->st),
       "checkpoint snapshot");
  const int ns = ctx->par.nspc;
  double* const dsp = ctx->ck_dev + (size_t)(ctx->nvar + 11) * P;
  if (spc && ns > 0)
    CK(cudaMemcpyAsync(dsp, ctx->pbuf[ctx->pcur] + 10 * P, (size_t)ns * P * sizeof(double),
                       cudaMemcpyDeviceToDevice, ctx->st),
       "checkpoint snapshot");
  CK(cudaEventRecord(ctx->ck_snap, ctx->st), "checkpoint event");
  // device -> host on the copy stream while later steps run on the step stream
  CK(cudaStreamWaitEvent(ctx->cst, ctx->ck_snap, 0), "checkpoint wait");
  if (u) CK(cudaMemcpyAsync(ctx->ck_h, du, (size_t)ctx->nvar * P * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->cst), "checkpoint copy");
  CK(cudaMemcpyAsync(ctx->ck_h + (size_t)ctx->nvar * P, dp, 9 * P * sizeof(double), cudaMemcpyDeviceToHost,
                     ctx->cst),
     "checkpoint copy");
  if (grav && (grvphi || grvpsi))
    CK(cudaMemcpyAsync(ctx->ck_h + (size_t)(ctx->nvar + 9) * P, dg, 2 * P * sizeof(double),
                       cudaMemcpyDeviceToHost, ctx->cst),
       "checkpoint copy");
  if (spc && ns > 0)
    CK(cudaMemcpyAsync(ctx->ck_h + (size_t)(ctx->nvar + 11) * P, dsp, (size_t)ns * P * sizeof(double),
                       cudaMemcpyDeviceToHost, ctx->cst),
       "checkpoint copy");
  CK(cudaEventRecord(ctx->ck_done, ctx->cst), "checkpoint event");
  // the next snapshot overwrites ck_dev only after this copy (hmn_checkpoint_wait above)
  ctx->ck_u = u;
  for (int q = 0; q < 9; q++) ctx->ck_prim[q] = prim ? prim[q] : nullptr;
  ctx->ck_gphi = grav ? grvphi : nullptr;
  ctx->ck_gpsi = grav ? grvpsi : nullptr;
  ctx->ck_spc = ns > 0 ? spc : nullptr;
  ctx->ck_pending = 1;
  return HMN_OK;
}

// passive scalars: caller layout spc(1:nspc, i, j, k) (species fastest) with
// the context's ghost layers <-> device planes NP.. of the primitive buffer
extern "C" int hmn_upload_scalars(hmn_ctx* ctx, const double* spc) {
  if (!ctx || !spc) return HMN_EINVAL;
  const int ns = ctx->par.nspc;
  if (ns == 0) return HMN_OK;
  const size_t P = ctx->plane;
  int rc = ensure_stage(ctx, (size_t)ns * P * sizeof(double));
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->st), "sync");
  size_t o = 0;
  for (int k = 0; k < ctx->n[2]; k++)
    for (int j = 0; j < ctx->n[1]; j++)
      for (int i = 0; i < ctx->n[0]; i++, o++) {
        const size_t g = ghosted_index(ctx, i, j, k);
        for (int n = 0; n < ns; n++) ctx->stage_h[(size_t)n * P + o] = spc[(size_t)ns * g + n];
      }
  CK(cudaMemcpyAsync(ctx->pbuf[ctx->pcur] + 10 * P, ctx->stage_h, (size_t)ns * P * sizeof(double),
                     cudaMemcpyHostToDevice, ctx->st),
     "upload");
  CK(cudaStreamSynchronize(ctx->st), "sync");
  return HMN_OK;
}

extern "C" int hmn_download_scalars(hmn_ctx* ctx, double* spc) {
  if (!ctx || !spc) return HMN_EINVAL;
  const int ns = ctx->par.nspc;
  if (ns == 0) return HMN_OK;
  const size_t P = ctx->plane;
  int rc = ensure_stage(ctx, (size_t)ns * P * sizeof(double));
  if (rc) return rc;
  CK(cudaMemcpyAsync(ctx->stage_h, ctx->pbuf[ctx->pcur] + 10 * P, (size_t)ns * P * sizeof(double),
                     cudaMemcpyDeviceToHost, ctx->st),
     "download");
  CK(cudaStreamSynchronize(ctx->st), "sync");
  size_t o = 0;
  for (int k = 0; k < ctx->n[2]; k++)
    for (int j = 0; j < ctx->n[1]; j++)
      for (int i = 0; i < ctx->n[0]; i++, o++) {
        const size_t g = ghosted_index(ctx, i, j, k);
        for (int n = 0; n < ns; n++) spc[(size_t)ns * g + n] = ctx->stage_h[(size_t)n * P + o];
      }
  return HMN_OK;
}

extern "C" int hmn_download_pressure(hmn_ctx* ctx, double* p) {
  if (!ctx || !p) return HMN_EINVAL;
  CK(launch_prim_out(ctx->pbuf[ctx->pcur], ctx->plane, ctx->phifac, ctx->par.gamma - 1.0, ctx->prim_out,
                     ctx->prim_out + 9 * ctx->plane, blocks_for(ctx), ctx->st),
     "prim");
  ctx->launches += 1;
  return to_host(ctx, p, ctx->prim_out + 9 * ctx->plane, 1, ghosted_plane(ctx));
}

// one whole step on the device (hormone.f90:126-147) with device-resident time
static int enqueue_step(hmn_ctx* ctx) {
  int rc = enqueue_cfl(ctx);
  if (rc) return rc;
  rc = enqueue_hydro(ctx);
  if (rc) return rc;
  if (ctx->glm) ctx->phifac = std::exp(-ctx->par.alpha9wave * ctx->par.courant);
  CK(launch_advance(ctx->sc, ctx->st), "advance");
  ctx->launches += 1;
  return HMN_OK;
}

// Grids of at most this many cells step in one persistent launch
// (hmn_small.cu) instead of a chain of six launches per step.
constexpr size_t kSmallCells = 65536;

static bool small_run_ok(hmn_ctx* ctx) {
  const char* e = getenv("HMN_SMALL");  // HMN_SMALL=0 keeps the per-phase launches
  if (e && e[0] == '0') return false;
  return ctx->par.precision == 0 && ctx->par.nspc == 0 && (ctx->par.rktype == 2 || ctx->par.rktype == 3) &&
         !ctx->zpush_on && ctx->plane <= kSmallCells && small_run_supported(ctx->tile, ctx->G.sph.on != 0);
}

// Up to max_steps steps of the device loop in persistent launches of at
// most 4096 steps each; the clock, dt and end test stay on the device.
static int run_small(hmn_ctx* ctx, int max_steps) {
  for (int a = 0; a < 3; a++)
    for (int io = 0; io < 2; io++)
      if (ctx->solve[a] && (ctx->bc[a][io][0] >= 9 || ctx->bc[a][io][1] >= 9) && !ctx->G.dir[a][io])
        return HMN_EBADCFG;  // codes 9 and 10 need hmn_set_dirichlet first
  if (ctx->solve[2] && ctx->bc[2][0][0] == 10 && !ctx->fb) return HMN_EBADCFG;
  if (!ctx->small_bar) CK(cudaMalloc((void**)&ctx->small_bar, 2 * sizeof(unsigned int)), "barrier");
  const int rk = ctx->par.rktype;
  SmallRun R;
  memset(&R, 0, sizeof(R));
  for (int p = 0; p < 2; p++)
    for (int s = 1; s <= rk; s++) R.st[p][s - 1] = stage_args(ctx, s, (ctx->pcur + p + s - 1) & 1);
  R.sc = ctx->sc;
  R.bar = ctx->small_bar;
  R.damp = ctx->glm ? std::exp(-ctx->par.alpha9wave * ctx->par.courant) : 1.0;
  R.phifac0 = ctx->phifac;
  R.rk = rk;
  R.ntiles = ctx->tiles[0] * ctx->tiles[1] * ctx->tiles[2];
  const int tn0 = ctx->sc_h->tn, pcur0 = ctx->pcur;
  int left = max_steps;
  while (left > 0) {
    R.nsteps = left < 4096 ? left : 4096;
    const int tn_before = ctx->sc_h->tn;
    int grid = 0;
    // the barrier's arrival counter starts every launch at zero
    CK(cudaMemsetAsync(ctx->small_bar, 0, sizeof(unsigned int), ctx->st), "barrier");
    CK(launch_small_run(ctx->G, R, ctx->mag != 0, ctx->glm != 0, ctx->G.sph.on != 0, ctx->tile, ctx->st, &grid),
       "small run");
    ctx->launches += 1;
    const int rc = fetch_scalars(ctx);
    if (rc) {
      ctx->pcur = (pcur0 + rk * (ctx->sc_h->tn - tn0)) & 1;
      return rc;
    }
    const int ran = ctx->sc_h->tn - tn_before;
    if (ran > 0) R.phifac0 = R.damp;  // the next launch's first step follows a step of this one
    // the parity of the primitive buffer moves with the steps that ran
    for (int p = 0; p < 2; p++)
      for (int s = 1; s <= rk; s++)
        R.st[p][s - 1] = stage_args(ctx, s, (pcur0 + rk * (ctx->sc_h->tn - tn0) + p + s - 1) & 1);
    if (ctx->sc_h->err_code || ctx->sc_h->done || ran < R.nsteps) break;
    left -= R.nsteps;
  }
  ctx->pcur = (pcur0 + rk * (ctx->sc_h->tn - tn0)) & 1;
  if (ctx->sc_h->tn > tn0) ctx->phifac = R.damp;
  return HMN_OK;
}

// kRunGraphSteps steps of the device loop as one graph launch.  Steps are
// launch-bound on small grids (a few microseconds of work per kernel); the
// graph removes the per-launch host cost.  The step count is even so that
// an RK3 graph ends on the primitive buffer it starts on.
static int run_graph_steps(hmn_ctx* ctx) {
  if (!ctx->run_exec || ctx->run_pcur != ctx->pcur || ctx->run_phifac != ctx->phifac) {
    drop_run_graph(ctx);
    const int pcur = ctx->pcur;
    const double phifac = ctx->phifac;
    const long long launches = ctx->launches;
    CK(cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeThreadLocal), "graph capture");
    int rc = HMN_OK;
    for (int s = 0; s < kRunGraphSteps && rc == HMN_OK; s++) rc = enqueue_step(ctx);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->st, &g);
    if (rc == HMN_OK && e == cudaSuccess && ctx->pcur == pcur && ctx->phifac == phifac)
      e = cudaGraphInstantiate(&ctx->run_exec, g, 0);
    else if (rc == HMN_OK)
      rc = HMN_ECUDA;
    if (g) cudaGraphDestroy(g);
    ctx->run_launches = ctx->launches - launches;
    ctx->launches = launches;
    ctx->pcur = pcur;
    ctx->phifac = phifac;
    if (rc) return rc;
    if (e != cudaSuccess) {
      ctx->run_exec = nullptr;
      return cuda_fail(ctx, e, "graph instantiate");
    }
    ctx->run_pcur = pcur;
    ctx->run_phifac = phifac;
  }
  CK(cudaGraphLaunch(ctx->run_exec, ctx->st), "graph launch");
  ctx->launches += ctx->run_launches;
  return HMN_OK;
}

extern "C" int hmn_run(hmn_ctx* ctx, double* time, double t_end, int max_steps, int* steps) {
  if (!ctx || !time) return HMN_EINVAL;
  if (slab_exchanges(ctx)) return HMN_EBADCFG;
  if (ctx->par.gravswitch == 3) {
    // the sub-cycle count depends on each step's dt: step on the host clock
    int done = 0;
    double t = *time;
    while (done < max_steps && t < t_end) {
      double dt, ch;
      int rc = hmn_timestep(ctx, t, t_end, t_end, &dt, &ch);
      if (rc) return rc;
      rc = hmn_gravity_step(ctx, t, dt, 1);
      if (rc) return rc;
      rc = enqueue_hydro(ctx);
      if (rc) return rc;
      if (ctx->glm) ctx->phifac = std::exp(-ctx->par.alpha9wave * ctx->par.courant);
      t = t + dt;
      done++;
    }
    *time = t;
    if (steps) *steps = done;
    return fetch_scalars(ctx);
  }
  int rc = push_times(ctx, *time, t_end, t_end);
  if (rc) return rc;
  rc = fetch_scalars(ctx);
  if (rc) return rc;
  const int tn0 = ctx->sc_h->tn;
  const int pcur0 = ctx->pcur;
  if (small_run_ok(ctx)) {
    rc = run_small(ctx, max_steps);
    if (rc) return rc;
    *time = ctx->sc_h->time;
    if (steps) *steps = ctx->sc_h->tn - tn0;
    return HMN_OK;
  }
  int done = 0;
  const bool graphs = ctx->par.rktype != 1;  // rktype 1 swaps buffers on the host after each step
  const int chunk = graphs ? kRunGraphSteps : 1;
  while (done < max_steps) {
    int n = max_steps - done < chunk ? max_steps - done : chunk;
    // the first step of a call runs plain: it settles the phidamp factor
    // the later steps share
    if (graphs && done > 0 && n == kRunGraphSteps) {
      rc = run_graph_steps(ctx);
      if (rc) return rc;
    } else {
      if (done == 0 && graphs) n = 1;
      for (int s = 0; s < n; s++) {
        rc = enqueue_step(ctx);
        if (rc) return rc;
      }
    }
    done += n;
    rc = fetch_scalars(ctx);
    // steps enqueued after the end time was reached did nothing on the device (every kernel
    // returns once `done` is set), but enqueue_hydro flipped the primitive buffer for them:
    // take the buffer parity from the steps that actually ran (each stage writes the other one)
    ctx->pcur = (pcur0 + ctx->par.rktype * (ctx->sc_h->tn - tn0)) & 1;
    if (rc) return rc;
    if (ctx->sc_h->time >= t_end) break;
  }
  *time = ctx->sc_h->time;
  if (steps) *steps = ctx->sc_h->tn - tn0;  // steps that ran before the end time was reached
  return HMN_OK;
}

extern "C" int hmn_last_error(hmn_ctx* ctx, int* code, int* i, int* j, int* k, int* sim) {
  if (!ctx) return HMN_EINVAL;
  int rc = fetch_scalars(ctx);
  (void)rc;
  if (code) *code = ctx->sc_h->err_code;
  if (i) *i = ctx->sc_h->err_i;
  if (j) *j = ctx->sc_h->err_j;
  if (k) *k = ctx->sc_h->err_k;
  if (sim) *sim = 0;
  return HMN_OK;
}

extern "C" long long hmn_launch_count(hmn_ctx* ctx) { return ctx ? ctx->launches : -1; }

extern "C" int hmn_sync(hmn_ctx* ctx) {
  if (!ctx) return HMN_EINVAL;
  CK(cudaStreamSynchronize(ctx->st), "sync");
  return HMN_OK;
}

extern "C" void* hmn_stream(hmn_ctx* ctx) { return ctx ? (void*)ctx->st : nullptr; }
