// hmn_noalloc.cu -- hmn_timestep_noalloc: the CFL timestep for callers that
// cannot allocate device memory.
//
// Some host programs cannot call cudaMalloc at the point where they need a
// timestep: a Fortran step loop whose device memory is owned by another
// runtime's pool allocator that it must not bypass, or a caller that budgets
// every byte of device memory up front and forbids allocation after start-up.
// Such callers cannot create an hmn_ctx (hmn_create allocates).  This entry point takes
// the conserved state already on the device and writes dt, ch and a status
// word to caller-owned device memory; the only other device memory it touches
// is the file-scope scratch array below.  The CUDA runtime loads this
// library's device code on a GPU lazily, at its first use there, and that
// load is when the array is allocated; from then on the GPU holds it until
// the process exits.  So the first call on each device allocates (it loads
// the code and looks up the array's address) and belongs in the caller's
// start-up, before the point after which it may not allocate.
//
// Every call copies the caller's host arrays of cell widths into the
// scratch with cudaMemcpyAsync.  Host arrays are usually pageable, and a
// pageable copy cannot be recorded into a CUDA graph, so the entry point is
// not to be called while its stream is being captured.
//
// Scratch layout (doubles): the cell widths dxi of the three axes (at most
// kNoallocMaxAxis+4 values each), then one (min dti, max cf) pair per block
// of the reduction.  A grid with more than kNoallocMaxAxis cells along any
// axis is rejected with HMN_EINVAL.  All calls share the array and it keeps
// the last call's contents; every slot a call reads is written earlier in
// the same call, so nothing carries over.  Calls that overlap on the GPU
// (two streams, or two host threads without ordering) race on the array and
// must be serialised by the caller.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>

#include "../../include/hormone_gpu.h"
#include "hmn_math.cuh"

namespace {

constexpr int kNoallocMaxAxis = 4096;                // cells per axis
constexpr int kNoallocBlocks = 1024;                 // reduction blocks
constexpr int kNoallocAxisLen = kNoallocMaxAxis + 4;  // dxi values per axis
constexpr int kNoallocWords = 3 * kNoallocAxisLen + 2 * kNoallocBlocks;  // 14,348 doubles = 114,784 bytes

static __device__ __align__(256) double g_noalloc_scratch[kNoallocWords];

// Device address of g_noalloc_scratch per device.  In host code the symbol
// name is only a host-side stand-in, so the first call on each device looks
// the address up with cudaGetSymbolAddress (that device current) and later
// calls reuse it.
constexpr int kMaxDevices = 64;
static double* g_scratch_ptr[kMaxDevices] = {nullptr};

struct NoallocGrid {
  int n[3];
  int solve[3];
  const double* dxi[3];  // into the scratch, offset +2 as the hmn_grid arrays
};

template <bool MAG>
__global__ void __launch_bounds__(256) noalloc_cfl_kernel(const NoallocGrid G, const double* u, size_t plane,
                                                          double gamma, double* partial) {
  using namespace hmn;
  const double gm1 = gamma - 1.0;
  double my_dti = __longlong_as_double(0x7ff0000000000000LL);
  double my_cf = 0.0;
  double bad = 0.0;
  const double off0 = G.solve[0] ? 1.0 : 0.0, off1 = G.solve[1] ? 1.0 : 0.0, off2 = G.solve[2] ? 1.0 : 0.0;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < plane; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % G.n[0]);
    const int j = (int)((c / G.n[0]) % G.n[1]);
    const int k = (int)(c / ((size_t)G.n[0] * G.n[1]));
    // primitive variables as rungekutta.f90:205-229 derives them
    const double d = u[c];
    const double v1 = u[plane + c] / d, v2 = u[2 * plane + c] / d, v3 = u[3 * plane + c] / d;
    const double e = u[4 * plane + c];
    double b1 = 0.0, b2 = 0.0, b3 = 0.0;
    if (MAG) {
      b1 = u[5 * plane + c];
      b2 = u[6 * plane + c];
      b3 = u[7 * plane + c];
    }
    const double eint = get_eint<MAG>(e, d, v1, v2, v3, b1, b2, b3);
    if (eint <= 0.0 || d <= 0.0) {
      bad = 1.0;
      continue;
    }
    // dti_cell (timestep.f90:125-183) for eostype 0
    const double cs = sqrt(gamma * (gm1 * eint) / d);
    double cf1, cf2, cf3;
    if (MAG) {
      cf1 = get_cf(d, cs, b1, b2, b3) + fabs(v1);
      cf2 = get_cf(d, cs, b2, b1, b3) + fabs(v2);
      cf3 = get_cf(d, cs, b3, b1, b2) + fabs(v3);
    } else {
      cf1 = cs + fabs(v1);
      cf2 = cs + fabs(v2);
      cf3 = cs + fabs(v3);
    }
    const double dxi1 = G.dxi[0][i + 2], dxi2 = G.dxi[1][j + 2], dxi3 = G.dxi[2][k + 2];
    const double dvol = dxi1 * dxi2 * dxi3;
    const double sa1 = dxi2 * dxi3, sa2 = dxi1 * dxi3, sa3 = dxi1 * dxi2;
    const double dti = dvol / (cf1 * off0 * (sa1 + sa1) + cf2 * off1 * (sa2 + sa2) + cf3 * off2 * (sa3 + sa3));
    my_cf = fmax2(my_cf, fmax2(fmax2(cf1, cf2), cf3));
    my_dti = fmin2(my_dti, dti);
  }
  for (int o = 16; o > 0; o >>= 1) {
    my_dti = fmin2(my_dti, __shfl_xor_sync(0xffffffffu, my_dti, o));
    my_cf = fmax2(my_cf, __shfl_xor_sync(0xffffffffu, my_cf, o));
    bad = fmax2(bad, __shfl_xor_sync(0xffffffffu, bad, o));
  }
  __shared__ double rd[8], rc[8], rb[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    rd[wid] = my_dti;
    rc[wid] = my_cf;
    rb[wid] = bad;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
      rd[0] = fmin2(rd[0], rd[w]);
      rc[0] = fmax2(rc[0], rc[w]);
      rb[0] = fmax2(rb[0], rb[w]);
    }
    // a failed cell marks the block's cf slot negative
    partial[2 * blockIdx.x] = rd[0];
    partial[2 * blockIdx.x + 1] = rb[0] > 0.0 ? -1.0 : rc[0];
  }
}

// dt with the output/end clamps of timestep.f90:74-89 from the block partials.
__global__ void noalloc_finalize_kernel(const double* partial, int nblocks, double courant, double time,
                                        double t_out, double t_end, int outstyle, int endstyle, double* out) {
  using namespace hmn;
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double mind = __longlong_as_double(0x7ff0000000000000LL), cfmax = 0.0;
  bool bad = false;
  for (int b = 0; b < nblocks; b++) {
    mind = fmin2(mind, partial[2 * b]);
    const double c = partial[2 * b + 1];
    if (c < 0.0) bad = true;
    cfmax = fmax2(cfmax, c);
  }
  double dt = courant * mind;
  if (outstyle == 1) {
    double t_ref = t_out;
    if (endstyle == 1) t_ref = fmin2(t_out, t_end);
    if (t_ref - time - dt > 0.0 && t_ref - time - 2.0 * dt < 0.0)
      dt = 0.5 * (t_ref - time);
    else
      dt = fmin2(dt, t_out - time);
  }
  if (endstyle == 1) dt = fmin2(dt, t_end - time);
  out[0] = dt;
  out[1] = cfmax;
  out[2] = bad ? (double)HMN_ENEG_EINT : 0.0;
}

int scratch_address(double** ptr) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return HMN_ECUDA;
  if (!g_scratch_ptr[dev]) {
    double* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      fprintf(stderr, "hmn_timestep_noalloc: cudaGetSymbolAddress: %s\n", cudaGetErrorString(e));
      return HMN_ECUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *ptr = g_scratch_ptr[dev];
  return HMN_OK;
}

}  // namespace

extern "C" int hmn_timestep_noalloc(const hmn_grid* grid, const hmn_params* par, const double* u_dev, double time,
                                    double t_out, double t_end, double* out_dev, void* stream) {
  if (!grid || !par || !u_dev || !out_dev) return HMN_EINVAL;
  if (par->gravswitch != 0) return HMN_EBADCFG;  // the gravity wave speed needs the context's state
  if (grid->ghost != 0) {                        // u_dev is read as packed interior planes
    fprintf(stderr, "hmn_timestep_noalloc: u_dev must be packed (grid->ghost = 0, got %d)\n", grid->ghost);
    return HMN_EINVAL;
  }
  NoallocGrid G;
  size_t plane = 1;
  for (int a = 0; a < 3; a++) {
    if (grid->n[a] < 1 || !grid->dxi[a]) return HMN_EINVAL;
    if (grid->n[a] > kNoallocMaxAxis) {
      fprintf(stderr,
              "hmn_timestep_noalloc: axis %d has %d cells; the static scratch holds at most %d cells per axis\n", a,
              grid->n[a], kNoallocMaxAxis);
      return HMN_EINVAL;
    }
    G.n[a] = grid->n[a];
    G.solve[a] = grid->n[a] > 1;
    plane *= (size_t)grid->n[a];
  }
  double* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  for (int a = 0; a < 3; a++) {
    double* dst = scratch + a * kNoallocAxisLen;
    cudaError_t e = cudaMemcpyAsync(dst, grid->dxi[a], (size_t)(grid->n[a] + 4) * sizeof(double),
                                    cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return HMN_ECUDA;
    G.dxi[a] = dst;
  }
  double* partial = scratch + 3 * kNoallocAxisLen;
  size_t want = (plane + 255) / 256;
  const int nblocks = (int)(want < (size_t)kNoallocBlocks ? (want ? want : 1) : kNoallocBlocks);
  if (par->mag_on)
    noalloc_cfl_kernel<true><<<nblocks, 256, 0, st>>>(G, u_dev, plane, par->gamma, partial);
  else
    noalloc_cfl_kernel<false><<<nblocks, 256, 0, st>>>(G, u_dev, plane, par->gamma, partial);
  if (cudaGetLastError() != cudaSuccess) return HMN_ECUDA;
  noalloc_finalize_kernel<<<1, 32, 0, st>>>(partial, nblocks, par->courant, time, t_out, t_end, par->outstyle,
                                            par->endstyle, out_dev);
  if (cudaGetLastError() != cudaSuccess) return HMN_ECUDA;
  return HMN_OK;
}
