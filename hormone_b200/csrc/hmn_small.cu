// hmn_small.cu -- whole steps of a small grid in one persistent launch.
//
// On a grid of a few thousand cells a step (CFL reduction, dt, rktype
// fused stages, time advance: hormone.f90:126-155) is a chain of six
// dependent kernels, each holding the GPU for a few microseconds of one
// cell's dependent arithmetic; a CUDA graph removes the host's launch cost
// but not the chain.  Here one cooperative launch runs up to `nsteps`
// steps: its CTAs sweep the grid's tiles in every phase and meet at a grid
// barrier between phases.  The phases are the device functions of the
// per-phase kernels (hmn_stage.cuh), so the result is bitwise theirs; the
// last RK stage of a step also reduces the CFL quantities of the state it
// writes (the values the next step's cfl_kernel would read back), and one
// thread advances the clock and forms the next dt, so a step is four grid
// barriers: one per stage and one for the clock.
//
// Coherence: inside one launch, a CTA reads cells that other CTAs wrote in
// the previous phase (halos, the scalars of the dt finalisation), and an
// SM's L1 is not coherent with the others.  This translation unit is
// therefore compiled with -Xptxas -dlcm=cg: its global loads are cached in
// L2 only.  The barrier is one arrival counter in global memory, zeroed by
// the host before every launch and never reset inside it: a CTA's n-th
// barrier (n from 0) is passed once the counter reaches (n + 1) x the grid,
// so the last CTA to arrive learns from its own atomic that it need not
// wait, and the others see that count on their next poll.  Release and
// acquire fences order the phases' memory; a CTA that waits longer than a
// second records HMN_ETIMEOUT and the launch returns.
#include <cuda_runtime.h>

#include "hmn_internal.h"
#include "hmn_stage.cuh"

namespace hmn {
namespace {

constexpr unsigned long long kBarrierWaitNs = 1000000000ull;

// All CTAs of the launch meet here for the nb-th time (nb counts this CTA's
// barriers from 0 and is advanced here); false (with HMN_ETIMEOUT recorded)
// if the others did not arrive within kBarrierWaitNs.
__device__ __forceinline__ bool grid_sync(unsigned int* bar, DevScalars* sc, unsigned int& nb) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int target = (nb + 1u) * gridDim.x;
    __threadfence();  // this CTA's writes before its arrival
    int good = 1;
    if (atomicAdd(bar, 1u) + 1u != target) {
      volatile unsigned int* cnt = bar;
      const unsigned long long t0 = global_ns();
      while (*cnt < target) {
        if (global_ns() - t0 > kBarrierWaitNs) {
          record_error(sc, kETIMEOUT, -1, -1, -1);
          good = 0;
          break;
        }
      }
    }
    __threadfence();  // the others' writes before this CTA's next reads
    ok = good;
  }
  __syncthreads();
  nb++;
  return ok != 0;
}

// Re-arm the CFL reduction slots (as finalize_dt leaves them).
__device__ __forceinline__ void rearm_cfl(DevScalars* sc) {
  sc->min_dti_bits = 0x7ff0000000000000ULL;
  sc->cfmax_bits = 0ULL;
}

template <bool MAG, bool GLM, class TL, bool SPH>
__global__ void __launch_bounds__(TL::NT, 1)
    small_run_kernel(const __grid_constant__ GridDev G, const __grid_constant__ SmallRun R) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SmemT<TL>& sm = *reinterpret_cast<SmemT<TL>*>(smem_raw);
  DevScalars* sc = R.sc;
  if (*(volatile int*)&sc->done) return;
  unsigned int nb = 0;  // barriers passed (the same count in every CTA)
  {  // CFL reduction and dt of the state entering the first step (cfl_kernel, cfl_finalize_kernel)
    const StageArgs& A0 = R.st[0][0];
    double my_dti = __longlong_as_double(0x7ff0000000000000LL), my_cf = 0.0;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < A0.plane;
         c += (size_t)gridDim.x * blockDim.x) {
      const int i = (int)(c % G.n[0]);
      const int j = (int)((c / G.n[0]) % G.n[1]);
      const int k = (int)(c / ((size_t)G.n[0] * G.n[1]));
      double dti, cfm;
      if (!cfl_cell<MAG>(G, A0.pin, A0.plane, A0.gamma, c, i, j, k, sc, dti, cfm)) continue;
      my_cf = fmax2(my_cf, cfm);
      my_dti = fmin2(my_dti, dti);
    }
    cfl_block_reduce(my_dti, my_cf, sc);
  }
  if (!grid_sync(R.bar, sc, nb)) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) finalize_dt(sc);
  if (!grid_sync(R.bar, sc, nb)) return;
  int par = 0;
  for (int step = 0; step < R.nsteps; step++) {
    // the fused RK stages (stage_kernel); the last one also reduces the
    // CFL quantities of the state it writes, which the next step's dt needs
    for (int s = 0; s < R.rk; s++) {
      StageArgs A = R.st[par][s];
      if (s == 0) A.phifac = step == 0 ? R.phifac0 : R.damp;
      if (s + 1 < R.rk) {
        for (int t = blockIdx.x; t < R.ntiles; t += gridDim.x) {
          stage_tile_exact<MAG, GLM, TL, SPH>(G, A, sm, t, nullptr);
          __syncthreads();
        }
      } else {
        double my_dti = __longlong_as_double(0x7ff0000000000000LL), my_cf = 0.0;
        for (int t = blockIdx.x; t < R.ntiles; t += gridDim.x) {
          stage_tile_exact<MAG, GLM, TL, SPH, false, true>(G, A, sm, t, nullptr, &my_dti, &my_cf);
          __syncthreads();
        }
        cfl_block_reduce(my_dti, my_cf, sc);
      }
      if (!grid_sync(R.bar, sc, nb)) return;
    }
    // the time advance (advance_kernel) and, while the run goes on, the next
    // step's dt from the reduction above (cfl_finalize_kernel)
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      sc->time = sc->time + sc->dt;
      sc->tn = sc->tn + 1;
      if (sc->endstyle == 1 && sc->time >= sc->t_end) sc->done = 1;
      if (sc->done)
        rearm_cfl(sc);
      else
        finalize_dt(sc);
    }
    if (!grid_sync(R.bar, sc, nb)) return;
    if (*(volatile int*)&sc->done) return;  // every CTA reads it after the same barrier
    par ^= R.rk & 1;  // an odd number of stages leaves the state in the other primitive buffer
  }
}

template <bool MAG, bool GLM, class TL, bool SPH>
cudaError_t launch_t(const GridDev& G, const SmallRun& R, cudaStream_t st, int* grid_out) {
  constexpr int smem = (int)sizeof(SmemT<TL>);
  auto fn = small_run_kernel<MAG, GLM, TL, SPH>;
  static int per_sm = -1;
  if (per_sm < 0) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, TL::NT, smem);
    if (e != cudaSuccess) return e;
  }
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const int resident = per_sm * nsm;
  if (resident < 1) return cudaErrorNotSupported;
  const int grid = R.ntiles < resident ? R.ntiles : resident;
  GridDev g = G;
  SmallRun r = R;
  void* args[] = {(void*)&g, (void*)&r};
  e = cudaLaunchCooperativeKernel((const void*)fn, dim3(grid), dim3(TL::NT), args, (size_t)smem, st);
  if (grid_out) *grid_out = grid;
  return e;
}

template <class TL, bool SPH>
cudaError_t launch_mag(const GridDev& G, const SmallRun& R, bool mag, bool glm, cudaStream_t st, int* grid) {
  if (!mag) return launch_t<false, false, TL, SPH>(G, R, st, grid);
  constexpr bool multi = TL::TY > 1 || TL::TZ > 1;
  if (glm != multi) return cudaErrorNotSupported;  // GLM exactly on MHD grids of 2 or 3 dimensions
  return launch_t<true, multi, TL, SPH>(G, R, st, grid);
}

}  // namespace

int small_run_supported(const int tile[3], bool sph) {
  if (tile[0] == 256 && tile[1] == 1 && tile[2] == 1) return 1;
  if (tile[0] == 16 && tile[1] == 16 && tile[2] == 1) return 1;
  if (tile[0] == 8 && tile[1] == 8 && tile[2] == 8) return sph ? 0 : 1;
  return 0;
}

cudaError_t launch_small_run(const GridDev& G, const SmallRun& R, bool mag, bool glm, bool sph, const int tile[3],
                             cudaStream_t st, int* grid) {
  if (tile[0] == 256 && tile[1] == 1 && tile[2] == 1) {
    if (sph) return launch_mag<Tile<256, 1, 1, 288, 2>, true>(G, R, mag, glm, st, grid);
    return launch_mag<Tile<256, 1, 1, 288, 2>, false>(G, R, mag, glm, st, grid);
  }
  if (tile[0] == 16 && tile[1] == 16 && tile[2] == 1) {
    if (sph) return launch_mag<Tile<16, 16, 1, 288, 2>, true>(G, R, mag, glm, st, grid);
    return launch_mag<Tile<16, 16, 1, 288, 2>, false>(G, R, mag, glm, st, grid);
  }
  if (tile[0] == 8 && tile[1] == 8 && tile[2] == 8 && !sph)
    return launch_mag<Tile<8, 8, 8, 640, 1>, false>(G, R, mag, glm, st, grid);
  return cudaErrorNotSupported;
}

}  // namespace hmn
